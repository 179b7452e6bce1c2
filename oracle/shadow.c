/*
 * Sun shadow map and voxel sun visibility -- part of the CPU oracle (test infrastructure only; see gi_oracle.h).
 *
 * Restates:
 *   - the reference's shadow pass (src/core/lighting.ts:133-140, 175-189: depth32float, cleared to 1, compare 'less',
 *     depthBias 2, depthBiasSlopeScale 2, cull none, alpha-masked fragments discarded) as a per-texel-centre raster of
 *     the light's orthographic clip space.  The reference draws it with a graphics pipeline; the rules fixed here
 *     (inclusive edge functions at texel centres, depth interpolated with the edge weights, the Vulkan depth-bias terms
 *     r = 2^(e - 23) of the largest |z| and the larger window-space slope) are this build's definition, shared with
 *     the CUDA kernels.  The stored depth is the smallest biased depth, so the result does not depend on the order in
 *     which triangles are drawn.  Alpha-masked materials: untextured, every fragment kept or none (the factor's alpha
 *     against the cutoff); textured, each texel by the texture at level 0 at its barycentric weights times the factor.
 *   - shadowCoord / shadowTap (src/core/frame.ts:35-52): layer 0 (lightViewProj, bias shadow.y) where x projects inside
 *     it, else layer 1 (lightViewProjFar, bias shadow.z) when the frame has two layers (shadow.x >= 1.5; the
 *     camera-following layers of instanced worlds, lighting.ts:93-125), else lit; textureSampleCompareLevel with a
 *     'less-equal' comparison sampler, linear filtering and clamp-to-edge within the layer, its four comparisons
 *     weighted bilinearly in f32.
 *   - voxSun (src/core/voxel.ts:633-671): the mean of four taps on the representative's plane.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "gi_oracle.h"
#include "orc_math.h"

enum { F_LVP = 64, F_SUN_DIR = 88, F_LVPF = 140, F_SHADOW = 156 };

static v3 light_clip(const float *m, v3 p) {
  return V(m[0] * p.x + m[4] * p.y + m[8] * p.z + m[12] * 1.0f, m[1] * p.x + m[5] * p.y + m[9] * p.z + m[13] * 1.0f,
           m[2] * p.x + m[6] * p.y + m[10] * p.z + m[14] * 1.0f);
}

/* 2^(e - 23) for the exponent e of |z| (the Vulkan depth-bias unit of a float depth buffer); zero and subnormals
 * take the smallest normal exponent. */
static float bias_unit(float zmax) {
  int eb = (int)((ubits(zmax) >> 23) & 0xffu);
  if (eb < 1) eb = 1;
  return ldexpf(1.0f, eb - 127 - 23);
}

/* Number of shadow-map layers the frame asks for (shadow.x: 1, or 2 for the camera-following layers of a world). */
uint32_t orc_shadow_layers(const float *frame) { return frame[F_SHADOW] >= 1.5f ? 2u : 1u; }

static void render_layer(const orc_scene *s, const float *m, uint32_t S, float *map);

/* Every layer the frame asks for: layer l at map + l S^2, drawn with lightViewProj (l = 0) or lightViewProjFar. */
int orc_shadow_render(const orc_scene *s, const float *frame, uint32_t S, float *map) {
  for (uint32_t l = 0; l < orc_shadow_layers(frame); l++)
    render_layer(s, frame + (l ? F_LVPF : F_LVP), S, map + (size_t)l * S * S);
  return 0;
}

static void render_layer(const orc_scene *s, const float *m, uint32_t S, float *map) {
  for (size_t i = 0; i < (size_t)S * S; i++) map[i] = 1.0f;
  const float inv = 1.0f / (float)S, fS = (float)S;
  const uint32_t nd = s->ndraw ? s->ndraw : s->ntris, ni = s->draw_inst ? s->draw_ninst : 1u;
  for (uint32_t t = 0; t < nd * ni; t++) {
    const uint32_t *idx = &s->tri[4u * (t % nd)];
    const orc_material *mt = &s->mats[idx[3]];
    /* alpha-masked: untextured, every fragment discarded or none; textured, each texel tested */
    int per_texel = (mt->flags & 1u) != 0u && orc_tex_layer_of(s, mt) != 0u;
    if (!per_texel && (mt->flags & 1u) != 0u && mt->base_color[3] < mt->alpha_cutoff) continue;
    v3 o = s->draw_inst ? fromf(s->draw_inst + 4u * (t / nd)) : V(0.0f, 0.0f, 0.0f);
    v3 pa = fromf(&s->pos[3u * idx[0]]), pb = fromf(&s->pos[3u * idx[1]]), pc = fromf(&s->pos[3u * idx[2]]);
    if (s->draw_inst) { pa = add(pa, o); pb = add(pb, o); pc = add(pc, o); }
    v3 c0 = light_clip(m, pa);
    v3 c1 = light_clip(m, pb);
    v3 c2 = light_clip(m, pc);
    float det = (c1.x - c0.x) * (c2.y - c0.y) - (c2.x - c0.x) * (c1.y - c0.y);
    if (!(det != 0.0f)) continue;
    float dzx = ((c1.z - c0.z) * (c2.y - c0.y) - (c2.z - c0.z) * (c1.y - c0.y)) / det;
    float dzy = ((c2.z - c0.z) * (c1.x - c0.x) - (c1.z - c0.z) * (c2.x - c0.x)) / det;
    float slope = fmaxf_(fabsf(dzx), fabsf(dzy)) * (2.0f * inv);   /* per texel: NDC spans 2 over S texels */
    float zmax = fmaxf_(fmaxf_(fabsf(c0.z), fabsf(c1.z)), fabsf(c2.z));
    float bias = 2.0f * bias_unit(zmax) + 2.0f * slope;
    /* window box with one texel of margin */
    float xw[3] = {(c0.x + 1.0f) * 0.5f * fS, (c1.x + 1.0f) * 0.5f * fS, (c2.x + 1.0f) * 0.5f * fS};
    float yw[3] = {(1.0f - c0.y) * 0.5f * fS, (1.0f - c1.y) * 0.5f * fS, (1.0f - c2.y) * 0.5f * fS};
    float x0 = fminf_(fminf_(xw[0], xw[1]), xw[2]), x1 = fmaxf_(fmaxf_(xw[0], xw[1]), xw[2]);
    float y0 = fminf_(fminf_(yw[0], yw[1]), yw[2]), y1 = fmaxf_(fmaxf_(yw[0], yw[1]), yw[2]);
    if (!(x1 >= -1.0f) || !(y1 >= -1.0f) || !(x0 <= fS + 1.0f) || !(y0 <= fS + 1.0f)) continue;
    int32_t i0 = iclamp(f2i(floorf(fmaxf_(x0, -2.0f))) - 1, 0, (int32_t)S - 1);
    int32_t i1 = iclamp(f2i(floorf(fminf_(x1, fS + 2.0f))) + 1, 0, (int32_t)S - 1);
    int32_t j0 = iclamp(f2i(floorf(fmaxf_(y0, -2.0f))) - 1, 0, (int32_t)S - 1);
    int32_t j1 = iclamp(f2i(floorf(fminf_(y1, fS + 2.0f))) + 1, 0, (int32_t)S - 1);
    for (int32_t j = j0; j <= j1; j++) {
      float y = 1.0f - ((float)j + 0.5f) * inv * 2.0f;
      for (int32_t i = i0; i <= i1; i++) {
        float x = ((float)i + 0.5f) * inv * 2.0f - 1.0f;
        float w0 = (c2.x - c1.x) * (y - c1.y) - (c2.y - c1.y) * (x - c1.x);
        float w1 = (c0.x - c2.x) * (y - c2.y) - (c0.y - c2.y) * (x - c2.x);
        float w2 = (c1.x - c0.x) * (y - c0.y) - (c1.y - c0.y) * (x - c0.x);
        int in = (w0 >= 0.0f && w1 >= 0.0f && w2 >= 0.0f) || (w0 <= 0.0f && w1 <= 0.0f && w2 <= 0.0f);
        if (!in) continue;
        float sum = (w0 + w1) + w2;
        if (!(sum != 0.0f)) continue;
        float z = ((w0 * c0.z + w1 * c1.z) + w2 * c2.z) / sum;
        if (!(z >= 0.0f && z <= 1.0f)) continue;   /* depth clipping */
        if (per_texel && !orc_raster_alpha_ok(s, idx, w0 / sum, w1 / sum, w2 / sum)) continue;
        float zb = z + bias;
        float *d = &map[(size_t)j * S + (size_t)i];
        if (zb < *d) *d = zb;
      }
    }
  }
}

static float compare4(const float *map, uint32_t S, float u, float v, float ref);

float orc_sun_tap(const float *frame, const float *map, uint32_t S, const float x3[3]) {
  v3 c = light_clip(frame + F_LVP, fromf(x3));
  float u = c.x * 0.5f + 0.5f, v = c.y * -0.5f + 0.5f;
  if (u >= 0.0f && v >= 0.0f && u <= 1.0f && v <= 1.0f) return compare4(map, S, u, v, c.z - frame[F_SHADOW + 1]);
  if (frame[F_SHADOW] < 1.5f) return 1.0f;   /* one layer, x outside it: lit */
  v3 c1 = light_clip(frame + F_LVPF, fromf(x3));
  float u1 = c1.x * 0.5f + 0.5f, v1 = c1.y * -0.5f + 0.5f;
  if (u1 >= 0.0f && v1 >= 0.0f && u1 <= 1.0f && v1 <= 1.0f)
    return compare4(map + (size_t)S * S, S, u1, v1, c1.z - frame[F_SHADOW + 2]);
  return 1.0f;                                /* outside both layers: lit */
}

/* textureSampleCompareLevel of one layer: 'less-equal', linear, clamp-to-edge */
static float compare4(const float *map, uint32_t S, float u, float v, float ref) {
  float tx = u * (float)S - 0.5f, ty = v * (float)S - 0.5f;
  float fx = floorf(tx), fy = floorf(ty);
  float ax = tx - fx, ay = ty - fy;
  int32_t i0 = f2i(fx), j0 = f2i(fy), n = (int32_t)S - 1;
  int32_t ia = iclamp(i0, 0, n), ib = iclamp(i0 + 1, 0, n), ja = iclamp(j0, 0, n), jb = iclamp(j0 + 1, 0, n);
  float c00 = ref <= map[(size_t)ja * S + ia] ? 1.0f : 0.0f, c10 = ref <= map[(size_t)ja * S + ib] ? 1.0f : 0.0f;
  float c01 = ref <= map[(size_t)jb * S + ia] ? 1.0f : 0.0f, c11 = ref <= map[(size_t)jb * S + ib] ? 1.0f : 0.0f;
  return (c00 * (1.0f - ax) + c10 * ax) * (1.0f - ay) + (c01 * (1.0f - ax) + c11 * ax) * ay;
}

static float tap(const float *frame, const float *map, uint32_t S, v3 x) {
  float p[3] = {x.x, x.y, x.z};
  return orc_sun_tap(frame, map, S, p);
}

/* voxSun (voxel.ts:643-671) for every occupied voxel of the built world. */
int orc_vox_sun(orc_vox *vx, const float *frame, const float *map, uint32_t S) {
  uint32_t nb = vx->hdr[0] < vx->max_bricks ? vx->hdr[0] : vx->max_bricks;
  v3 sd = fromf(&frame[F_SUN_DIR]);
  for (uint32_t ptr = 0; ptr < nb; ptr++) {
    uint32_t first = vx->base[ptr];
    if (first >= ORC_MARK) continue;
    uint32_t code = vx->code[ptr];
    uint32_t L = code >> 27;
    i3 b = I((int32_t)((code >> 18) & 511u), (int32_t)((code >> 9) & 511u), (int32_t)(code & 511u));
    float vs = ldexpf(vx->v0, (int)L);
    uint32_t r = 0;
    for (uint32_t bit = 0; bit < 512u; bit++) {
      if ((vx->occ[ptr * 16u + (bit >> 5)] & (1u << (bit & 31u))) == 0u) continue;
      uint32_t ai = first + r++;
      if (ai >= vx->max_voxels) continue;
      i3 c = I(b.x * 8 + (int32_t)(bit & 7u), b.y * 8 + (int32_t)((bit >> 3) & 7u), b.z * 8 + (int32_t)(bit >> 6));
      i3 o = I(vx->origin[L][0], vx->origin[L][1], vx->origin[L][2]);
      v3 pc = add(muls(muls(vi2f(o), vs), 8.0f), muls(adds(vi2f(c), 0.5f), vs));
      uint32_t e = vx->attr[ai * 4u + 1u];
      /* unpack2x16snorm: max(k / 32767, -1) */
      float ex = fmaxf_((float)(int16_t)(e & 0xffffu) / 32767.0f, -1.0f);
      float ey = fmaxf_((float)(int16_t)(e >> 16) / 32767.0f, -1.0f);
      v3 n = V(ex, ey, 1.0f - fabsf(ex) - fabsf(ey));
      float q0 = fmaxf_(-n.z, 0.0f);
      n.x += n.x >= 0.0f ? -q0 : q0;
      n.y += n.y >= 0.0f ? -q0 : q0;
      v3 q = pc;
      if (dot(n, n) > 1e-4f) { n = normalize3(n); q = add(pc, muls(n, vx->plane[ai])); }
      else n = V(0.0f, 1.0f, 0.0f);
      v3 ns = dot(n, sd) < 0.0f ? neg(n) : n;
      v3 t1 = normalize3(cross(ns, fabsf(ns.y) > 0.9f ? V(1.0f, 0.0f, 0.0f) : V(0.0f, 1.0f, 0.0f)));
      v3 t2 = cross(ns, t1);
      float h = 0.25f * vs;
      v3 oo = add(q, muls(ns, 0.25f * vs + 0.03f));
      v3 sp = add(t1, t2), sm = sub(t1, t2);
      float vis = 0.25f * (((tap(frame, map, S, add(oo, muls(sp, h))) + tap(frame, map, S, add(oo, muls(sm, h))))
                            + tap(frame, map, S, sub(oo, muls(sp, h)))) + tap(frame, map, S, sub(oo, muls(sm, h))));
      vx->sunvis[ai] = vis;
    }
  }
  return 0;
}
