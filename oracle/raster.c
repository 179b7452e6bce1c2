/* Headless G-buffer restatement (test infrastructure only).  The reference draws depth32float (reversed Z,
 * infinite far plane) and an rgba16float shading normal with a graphics pipeline (src/core/gbuffer.ts:82-103).
 * There is no graphics stack here, so the G-buffer is defined as one primary-ray sample per pixel centre:
 *   ray   : origin = eye, direction = worldAt(px, 1) - eye (the point on the near plane, frame.ts:22-26)
 *   hit   : Moller-Trumbore against every triangle whose clipped screen box (one pixel of margin) holds the pixel;
 *           w = t * dot(dir, fwd) must be >= near (the near plane clips), depth = near / w
 *   depth : the largest depth wins (reversed Z, 'greater'); equal depths keep the smaller triangle index
 *   normal: normalize(interpolated vertex normal) * (front ? 1 : -1), front = the eye on the side of the triangle's
 *           counter-clockwise face (gbuffer.ts:94-95), rounded to f16 as the texture stores it; w = 0.
 * The CUDA raster implements the same definition. */
#include <stdlib.h>
#include "gi_oracle.h"
#include "orc_math.h"

enum { F_VP = 0, F_IVP = 16, F_EYE = 80, F_FWD = 84, F_SIZE = 100 };

static v3 world_at(const float *F, int32_t px, int32_t py, float d) {
  float nx = ((float)px + 0.5f) * F[F_SIZE + 2] * 2.0f - 1.0f;
  float ny = 1.0f - ((float)py + 0.5f) * F[F_SIZE + 3] * 2.0f;
  const float *m = F + F_IVP;
  float h[4];
  for (int i = 0; i < 4; i++) h[i] = m[i] * nx + m[4 + i] * ny + m[8 + i] * d + m[12 + i] * 1.0f;
  return V(h[0] / h[3], h[1] / h[3], h[2] / h[3]);
}

/* Moller-Trumbore.  Returns 1 and (t, u, v) on a hit with t > 0. */
static int ray_tri(v3 o, v3 dir, v3 a, v3 b, v3 c, float *t, float *u, float *v) {
  v3 e1 = sub(b, a), e2 = sub(c, a);
  v3 pv = cross(dir, e2);
  float det = dot(e1, pv);
  if (det == 0.0f) return 0;
  float inv = 1.0f / det;
  v3 tv = sub(o, a);
  float uu = dot(tv, pv) * inv;
  if (uu < 0.0f || uu > 1.0f) return 0;
  v3 qv = cross(tv, e1);
  float vv = dot(dir, qv) * inv;
  if (vv < 0.0f || uu + vv > 1.0f) return 0;
  float tt = dot(e2, qv) * inv;
  if (!(tt > 0.0f)) return 0;
  *t = tt; *u = uu; *v = vv;
  return 1;
}

/* Screen box of the triangle clipped to w >= near, one pixel of margin, clamped; returns 0 when empty. */
static int screen_box(const float *F, uint32_t W, uint32_t H, v3 p[3], int32_t box[4]) {
  const float *m = F + F_VP;
  float near = F[F_EYE + 3];
  float cl[3][4];
  for (int k = 0; k < 3; k++)
    for (int i = 0; i < 4; i++) cl[k][i] = m[i] * p[k].x + m[4 + i] * p[k].y + m[8 + i] * p[k].z + m[12 + i] * 1.0f;
  float pts[8][2];
  int np = 0;
  for (int k = 0; k < 3; k++) {
    const float *a = cl[k], *b = cl[(k + 1) % 3];
    int ina = a[3] >= near, inb = b[3] >= near;
    if (ina) { pts[np][0] = a[0] / a[3]; pts[np][1] = a[1] / a[3]; np++; }
    if (ina != inb) {
      float t = (a[3] - near) / (a[3] - b[3]);
      float x = a[0] + (b[0] - a[0]) * t, y = a[1] + (b[1] - a[1]) * t;
      pts[np][0] = x / near; pts[np][1] = y / near; np++;
    }
  }
  if (np == 0) return 0;
  float x0 = 1e30f, x1 = -1e30f, y0 = 1e30f, y1 = -1e30f;
  for (int k = 0; k < np; k++) {
    float sx = (pts[k][0] * 0.5f + 0.5f) * (float)W, sy = (0.5f - pts[k][1] * 0.5f) * (float)H;
    x0 = fminf_(x0, sx); x1 = fmaxf_(x1, sx); y0 = fminf_(y0, sy); y1 = fmaxf_(y1, sy);
  }
  if (!(x1 >= -1.0f) || !(y1 >= -1.0f) || !(x0 <= (float)W + 1.0f) || !(y0 <= (float)H + 1.0f)) return 0;
  box[0] = iclamp(f2i(floorf(fmaxf_(x0, -2.0f))) - 1, 0, (int32_t)W - 1);
  box[1] = iclamp(f2i(floorf(fminf_(x1, (float)W + 2.0f))) + 1, 0, (int32_t)W - 1);
  box[2] = iclamp(f2i(floorf(fmaxf_(y0, -2.0f))) - 1, 0, (int32_t)H - 1);
  box[3] = iclamp(f2i(floorf(fminf_(y1, (float)H + 2.0f))) + 1, 0, (int32_t)H - 1);
  return 1;
}

int orc_raster_gbuffer(const orc_scene *s, const float *F, uint32_t W, uint32_t H, float *depth_out, float *normal_out,
                       uint32_t *tri_out) {
  size_t npx = (size_t)W * H;
  uint64_t *key = (uint64_t *)calloc(npx, sizeof(uint64_t));
  v3 *dirs = (v3 *)malloc(npx * sizeof(v3));
  if (!key || !dirs) { free(key); free(dirs); return -1; }
  v3 eye = fromf(F + F_EYE), fwd = fromf(F + F_FWD);
  float near = F[F_EYE + 3];
  for (uint32_t y = 0; y < H; y++)
    for (uint32_t x = 0; x < W; x++) dirs[(size_t)y * W + x] = sub(world_at(F, (int32_t)x, (int32_t)y, 1.0f), eye);
  const uint32_t nd = s->ndraw ? s->ndraw : s->ntris, ni = s->draw_inst ? s->draw_ninst : 1u;
  for (uint32_t t = 0; t < nd * ni; t++) {
    const uint32_t *i = s->tri + 4u * (t % nd);
    v3 p[3] = {fromf(s->pos + 3u * i[0]), fromf(s->pos + 3u * i[1]), fromf(s->pos + 3u * i[2])};
    if (s->draw_inst) {
      v3 o = fromf(s->draw_inst + 4u * (t / nd));
      p[0] = add(p[0], o); p[1] = add(p[1], o); p[2] = add(p[2], o);
    }
    int32_t box[4];
    if (!screen_box(F, W, H, p, box)) continue;
    for (int32_t y = box[2]; y <= box[3]; y++)
      for (int32_t x = box[0]; x <= box[1]; x++) {
        size_t q = (size_t)y * W + (size_t)x;
        float tt, uu, vv;
        if (!ray_tri(eye, dirs[q], p[0], p[1], p[2], &tt, &uu, &vv)) continue;
        float w = tt * dot(dirs[q], fwd);
        if (!(w >= near)) continue;
        float depth = near / w;
        uint64_t k = ((uint64_t)ubits(depth) << 32) | (uint64_t)(0xffffffffu - t);
        if (k > key[q] && orc_raster_alpha_ok(s, i, (1.0f - uu) - vv, uu, vv)) key[q] = k;   /* masked: discard */
      }
  }
  for (size_t q = 0; q < npx; q++) {
    float *n = normal_out + 4 * q;
    if (key[q] == 0) {
      depth_out[q] = 0.0f; n[0] = n[1] = n[2] = n[3] = 0.0f;
      if (tri_out) tri_out[q] = 0xffffffffu;
      continue;
    }
    uint32_t t = 0xffffffffu - (uint32_t)(key[q] & 0xffffffffu);
    depth_out[q] = fbits((uint32_t)(key[q] >> 32));
    if (tri_out) tri_out[q] = t;
    const uint32_t *i = s->tri + 4u * (t % nd);
    v3 a = fromf(s->pos + 3u * i[0]), b = fromf(s->pos + 3u * i[1]), c = fromf(s->pos + 3u * i[2]);
    if (s->draw_inst) {
      v3 o = fromf(s->draw_inst + 4u * (t / nd));
      a = add(a, o); b = add(b, o); c = add(c, o);
    }
    float tt = 0, uu = 0, vv = 0;
    ray_tri(eye, dirs[q], a, b, c, &tt, &uu, &vv);
    v3 n0 = fromf(s->nrm + 3u * i[0]), n1 = fromf(s->nrm + 3u * i[1]), n2 = fromf(s->nrm + 3u * i[2]);
    v3 nn = add(add(muls(n0, 1.0f - uu - vv), muls(n1, uu)), muls(n2, vv));
    float flip = dot(cross(sub(b, a), sub(c, a)), sub(eye, a)) > 0.0f ? 1.0f : -1.0f;
    nn = muls(normalize3(nn), flip);
    n[0] = orc_f16_to_f32(orc_f32_to_f16(nn.x));
    n[1] = orc_f16_to_f32(orc_f32_to_f16(nn.y));
    n[2] = orc_f16_to_f32(orc_f32_to_f16(nn.z));
    n[3] = 0.0f;
  }
  free(key); free(dirs);
  return 0;
}
