/* Sequential restatement of the screen-probe radiance cascades over the voxel tracer (src/core/rc.ts, method
 * 'screen', world tracer 'voxel', depthCascades 0: the config token 'voxel').  Test infrastructure only.
 *
 * Follows rc.ts:95-141 (shading), :210-245 (traceWorld), :291-311 (octahedral maps, packing), :572-590
 * (setupScreen), :600-622 (trace), :681-743 (upperAvg, mergeScreen), :745-774 (shBasis, projectSH),
 * :819-829 (evalSH), :929-954 (gatherScreen), and voxel.ts:81-202 (voxRank, voxAt, voxLevelFor, traceVox).
 * Multi-bounce (bounce.ts) is restated too: the volume's frame (orc_bounce_frame) and the cascades' read of the
 * irradiance it injects into the voxels (when orc_vox.bn_inj is set), and the cascades' read of the dynamic layer
 * (dyn.c) when orc_vox.dyn is set.  The triangle comparator is off.  The hit radiance adds the voxel's emissive radiance (the reference has no emission). */
#include <stdlib.h>
#include "gi_oracle.h"
#include "orc_math.h"
#include "orc_par.h"
#include "orc_rc.h"

/* worldAt (frame.ts:22-26); mat4 * vec4 summed in column order. */
v3 world_at(const float *F, int32_t px, int32_t py, float d) {
  float nx = ((float)px + 0.5f) * F[F_SIZE + 2] * 2.0f - 1.0f;
  float ny = 1.0f - ((float)py + 0.5f) * F[F_SIZE + 3] * 2.0f;
  const float *m = F + F_IVP;
  float h[4];
  for (int i = 0; i < 4; i++) h[i] = m[i] * nx + m[4 + i] * ny + m[8 + i] * d + m[12 + i] * 1.0f;
  return V(h[0] / h[3], h[1] / h[3], h[2] / h[3]);
}
float view_z(const float *F, v3 p) { return dot(sub(p, fromf(F + F_EYE)), fromf(F + F_FWD)); }

/* octDecode / dirOf (rc.ts:291-308) */
static v3 oct_decode(float u, float v) {
  float fx = u * 2.0f - 1.0f, fy = v * 2.0f - 1.0f;
  v3 n = V(fx, fy, 1.0f - fabsf(fx) - fabsf(fy));
  float t = fmaxf_(-n.z, 0.0f);
  n.x += n.x >= 0.0f ? -t : t;
  n.y += n.y >= 0.0f ? -t : t;
  return normalize3(n);
}
v3 dir_of(uint32_t di, uint32_t res) {
  return oct_decode(((float)(di % res) + 0.5f) / (float)res, ((float)(di / res) + 0.5f) / (float)res);
}

float round_store(float x, uint32_t atlas) {
  if (atlas == 1) return orc_f16_to_f32(orc_f32_to_f16(x));
  if (atlas == 2) return orc_bf16_to_f32(orc_f32_to_bf16(x));
  return x;
}

/* voxRank (voxel.ts:81-87) */
uint32_t vox_rank(const orc_vox *vx, uint32_t brick, uint32_t bit) {
  uint32_t w = bit >> 5;
  uint32_t r = popc(vx->occ[brick * 16u + w] & ((1u << (bit & 31u)) - 1u));
  for (uint32_t i = 0; i < w; i++) r += popc(vx->occ[brick * 16u + i]);
  return vx->base[brick] + r;
}
/* voxAt (voxel.ts:90-107): (brick, bit, level) or brick ORC_EMPTY */
void vox_at(const orc_vox *vx, uint32_t L, i3 c, uint32_t out[3]) {
  uint32_t l = L;
  i3 cc = c;
  int32_t n8 = (int32_t)vx->G * 8;
  for (;;) {
    uint32_t ptr = vx->ptr[ptr_index(vx, l, I(cc.x >> 3, cc.y >> 3, cc.z >> 3))];
    if (ptr != ORC_DROP) {
      if (ptr >= ORC_MARK) { out[0] = ORC_EMPTY; out[1] = 0; out[2] = l; return; }
      uint32_t bit = (uint32_t)((cc.x & 7) + 8 * (cc.y & 7) + 64 * (cc.z & 7));
      if ((vx->occ[ptr * 16u + (bit >> 5)] & (1u << (bit & 31u))) == 0u) { out[0] = ORC_EMPTY; out[1] = 0; out[2] = l; return; }
      out[0] = ptr; out[1] = bit; out[2] = l;
      return;
    }
    if (l + 1u >= vx->levels) { out[0] = ORC_EMPTY; out[1] = 0; out[2] = l; return; }
    i3 o = org(vx, l);
    i3 w = I((o.x * 8 + cc.x) >> 1, (o.y * 8 + cc.y) >> 1, (o.z * 8 + cc.z) >> 1);
    l++;
    i3 o1 = org(vx, l);
    cc = I(w.x - o1.x * 8, w.y - o1.y * 8, w.z - o1.z * 8);
    if (cc.x < 0 || cc.y < 0 || cc.z < 0 || cc.x >= n8 || cc.y >= n8 || cc.z >= n8) { out[0] = ORC_EMPTY; out[1] = 0; out[2] = l; return; }
  }
}
/* voxInside / voxLevelFor (voxel.ts:108-119) */
static int vox_inside(const orc_vox *vx, uint32_t L, v3 p) {
  float bs = vox_size(vx, L) * 8.0f;
  v3 lo = muls(vi2f(org(vx, L)), bs);
  float ext = (float)vx->G * bs;
  v3 hi = adds(lo, ext);
  return p.x > lo.x && p.y > lo.y && p.z > lo.z && p.x < hi.x && p.y < hi.y && p.z < hi.z;
}
uint32_t vox_level_for(const orc_vox *vx, uint32_t L, v3 e) {
  uint32_t l = L;
  while (l + 1u < vx->levels && !vox_inside(vx, l, e)) l++;
  return l;
}

/* style.ts:18-25 */
static v3 toon_albedo(v3 a) {
  float l = dot(a, V(0.2126f, 0.7152f, 0.0722f));
  v3 r = add(V(l, l, l), muls(sub(a, V(l, l, l)), 1.6f));
  return V(fclampf(r.x, 0.0f, 1.0f), fclampf(r.y, 0.0f, 1.0f), fclampf(r.z, 0.0f, 1.0f));
}
static float toon_ramp(float x) { return x > 0.3f ? 1.0f : (x > 0.05f ? 0.5f : 0.0f); }

/* shadeHitV (rc.ts:108-116) with e = 0 (no multi-bounce) */
static v3 shade_hit_v(const float *F, v3 n0, const float alb[4], v3 d, v3 e, float vis) {
  v3 n = dot(n0, n0) > 0.01f ? n0 : neg(d);
  if (dot(n, d) > 0.0f) n = neg(n);
  v3 a = V(alb[0], alb[1], alb[2]);
  v3 b = mul(divs(a, PI_F), e);
  float ndl = fmaxf_(dot(n, fromf(F + F_SUN)), 0.0f);
  if (ndl <= 0.0f) return b;
  v3 sunE = fromf(F + F_SUNE);
  if (alb[3] > 0.5f && F[F_STYLE] > 0.5f) {
    v3 ts = muls(mul(divs(toon_albedo(a), 3.14159265f), sunE), toon_ramp(ndl * vis));
    return add(b, ts);
  }
  return add(b, muls(muls(mul(divs(a, PI_F), sunE), ndl), vis));
}


/* ---- multi-bounce reads (bounce.ts:44-75, 90-93; rc.ts:198-202) ---- */
static float bn_get(const orc_bounce *b, const float *vol, int32_t x, int32_t y, int32_t z, int k) {
  return vol[(((size_t)z * b->dy + (size_t)y) * b->dx + (size_t)x) * 4u + (size_t)k];
}
static float bn_axis_a(const orc_bounce *b, const float *vol, i3 c, int a) { return bn_get(b, vol, c.x, c.y, a * (int32_t)b->dz + c.z, 3); }
static v3 bn_axis_rgb(const orc_bounce *b, const float *vol, i3 c, int a) {
  int32_t z = a * (int32_t)b->dz + c.z;
  return V(bn_get(b, vol, c.x, c.y, z, 0), bn_get(b, vol, c.x, c.y, z, 1), bn_get(b, vol, c.x, c.y, z, 2));
}
static i3 bn_origin(const orc_bounce *b, const float *vol) {
  int32_t z = 6 * (int32_t)b->dz;
  return I(f2i(bn_get(b, vol, 0, 0, z, 0)), f2i(bn_get(b, vol, 0, 0, z, 1)), f2i(bn_get(b, vol, 0, 0, z, 2)));
}
/* WGSL smoothstep */
static float smoothstep_(float e0, float e1, float x) {
  float t = fclampf((x - e0) / (e1 - e0), 0.0f, 1.0f);
  return t * t * (3.0f - 2.0f * t);
}
/* bnRead (bounce.ts:49-74) */
static v3 bn_read(const orc_bounce *b, const float *vol, v3 q, v3 p, v3 n) {
  i3 org0 = bn_origin(b, vol);
  v3 g = sub(V(q.x / b->cell, q.y / b->cell, q.z / b->cell), vi2f(org0));
  i3 bb = vf2i(vfloor(g));
  v3 fr = sub(g, vi2f(bb)), n2 = mul(n, n);
  float tol = 0.5f * b->v0;
  v3 e = V(0.0f, 0.0f, 0.0f);
  float ws = 0.0f;
  for (int k = 0; k < 8; k++) {
    i3 off = I(k & 1, (k >> 1) & 1, (k >> 2) & 1);
    i3 cc = I(bb.x + off.x, bb.y + off.y, bb.z + off.z);
    if (cc.x < 0 || cc.y < 0 || cc.z < 0 || cc.x >= (int32_t)b->dx || cc.y >= (int32_t)b->dy || cc.z >= (int32_t)b->dz) continue;
    v3 pp = muls(vi2f(I(org0.x + cc.x, org0.y + cc.y, org0.z + cc.z)), b->cell);
    v3 u = sub(q, pp);
    if (bn_axis_a(b, vol, cc, 0) <= 0.0f) continue;
    if (fabsf(u.x) > bn_axis_a(b, vol, cc, u.x >= 0.0f ? 0 : 1) + tol || fabsf(u.y) > bn_axis_a(b, vol, cc, u.y >= 0.0f ? 2 : 3) + tol
        || fabsf(u.z) > bn_axis_a(b, vol, cc, u.z >= 0.0f ? 4 : 5) + tol) continue;
    v3 t3 = V(off.x == 1 ? fr.x : 1.0f - fr.x, off.y == 1 ? fr.y : 1.0f - fr.y, off.z == 1 ? fr.z : 1.0f - fr.z);
    float w = t3.x * t3.y * t3.z * smoothstep_(-0.05f, 0.25f, dot(sub(pp, p), n) / b->cell);
    if (w <= 0.0f) continue;
    v3 s = add(add(muls(bn_axis_rgb(b, vol, cc, n.x >= 0.0f ? 0 : 1), n2.x), muls(bn_axis_rgb(b, vol, cc, n.y >= 0.0f ? 2 : 3), n2.y)),
               muls(bn_axis_rgb(b, vol, cc, n.z >= 0.0f ? 4 : 5), n2.z));
    e = add(e, muls(s, w));
    ws += w;
  }
  return ws > 1e-6f ? divs(e, ws) : V(0.0f, 0.0f, 0.0f);
}
/* voxSide (rc.ts:120-124) */
static float vox_side(v3 p, v3 n, v3 d, v3 pc, float v) {
  float s = dot(sub(p, pc), n);
  if (fabsf(s) > 0.05f * v) return s > 0.0f ? 1.0f : -1.0f;
  return dot(n, d) > 0.0f ? -1.0f : 1.0f;
}

/* The hit: attributes of voxel (brick, bit), shaded (voxShade, rc.ts:136-140) plus the emissive radiance.  entry: where
 * the ray enters the voxel; pc, vsz: its centre and size (the multi-bounce term's side and shading point). */
static void shade_voxel(const ctx_t *cx, uint32_t brick, uint32_t bit, v3 d, v3 entry, v3 pc, float vsz, trace_t *out) {
  const orc_vox *vx = cx->vx;
  uint32_t w[4] = {0, 0, 0, 0};
  float vis = 0.0f;
  uint32_t ai = 0;
  int has = vx->base[brick] != ORC_EMPTY;
  if (has) {
    ai = vox_rank(vx, brick, bit);
    for (int k = 0; k < 4; k++) w[k] = vx->attr[ai * 4u + k];
    vis = vx->sunvis[ai];
  }
  float alb[4];
  for (int k = 0; k < 4; k++) alb[k] = (float)((w[0] >> (8 * k)) & 0xffu) / 255.0f;
  float nx = fmaxf_((float)(int16_t)(w[1] & 0xffffu) / 32767.0f, -1.0f);
  float ny = fmaxf_((float)(int16_t)(w[1] >> 16) / 32767.0f, -1.0f);
  v3 n = V(nx, ny, 1.0f - fabsf(nx) - fabsf(ny));
  float q = fmaxf_(-n.z, 0.0f);
  n.x += n.x >= 0.0f ? -q : q;
  n.y += n.y >= 0.0f ? -q : q;
  /* voxBounce: the irradiance e at the shading point p = entry - d vsz / 4 */
  v3 e = V(0.0f, 0.0f, 0.0f);
  v3 p = sub(entry, muls(d, 0.25f * vsz));
  if (has && cx->bn) {
    if (dot(n, n) <= 0.01f) e = bn_read(cx->bn, cx->bn_prev, p, p, neg(d));
    else e = bn_read(cx->bn, cx->bn_prev, p, p, muls(n, vox_side(p, n, d, pc, vsz)));
  } else if (has && vx->bn_inj) {
    const float *q = vx->bn_inj + (size_t)ai * 6u + (vox_side(p, n, d, pc, vsz) < 0.0f ? 3u : 0u);
    e = V(q[0], q[1], q[2]);
  }
  v3 r = shade_hit_v(cx->F, n, alb, d, e, vis);
  v3 em = V(orc_f16_to_f32((uint16_t)(w[2] & 0xffffu)), orc_f16_to_f32((uint16_t)(w[2] >> 16)), orc_f16_to_f32((uint16_t)(w[3] & 0xffffu)));
  r = add(r, em);
  out->r = r.x; out->g = r.y; out->b = r.z; out->T = 0.0f;
}

/* traceVox (voxel.ts:121-202) with a configurable step cap. */
void trace_vox(const ctx_t *cx, v3 o, v3 d, float t0, float t1, float tskip, uint32_t L, uint32_t cap, trace_t *out) {
  const orc_vox *vx = cx->vx;
  out->r = out->g = out->b = 0.0f; out->T = 1.0f; out->lvl = ORC_EMPTY; out->ptr = ORC_EMPTY; out->bit = 0; out->tin = 0;
  out->steps = 0;
  float v = vox_size(vx, L);
  int32_t G = (int32_t)vx->G;
  v3 lo = muls(muls(vi2f(org(vx, L)), v), 8.0f);
  v3 hi = adds(lo, (float)G * v * 8.0f);
  v3 dd = V(fabsf(d.x) < 1e-9f ? 1e-9f : d.x, fabsf(d.y) < 1e-9f ? 1e-9f : d.y, fabsf(d.z) < 1e-9f ? 1e-9f : d.z);
  v3 inv = V(1.0f / dd.x, 1.0f / dd.y, 1.0f / dd.z);
  v3 ta = mul(sub(lo, o), inv), tb = mul(sub(hi, o), inv);
  v3 tn = vmin(ta, tb), tf = vmax(ta, tb);
  float t = fmaxf_(fmaxf_(fmaxf_(tn.x, tn.y), tn.z), t0);
  float tEnd = fminf_(fminf_(fminf_(tf.x, tf.y), tf.z), t1);
  if (t >= tEnd) return;
  i3 st = I(dd.x > 0.0f ? 1 : -1, dd.y > 0.0f ? 1 : -1, dd.z > 0.0f ? 1 : -1);
  v3 sp = V(st.x > 0 ? 1.0f : 0.0f, st.y > 0 ? 1.0f : 0.0f, st.z > 0 ? 1.0f : 0.0f);
  int32_t nVox = G * 8;
  i3 c = iclamp3(vf2i(vfloor(divs(sub(add(o, muls(d, t)), lo), v))), I(0, 0, 0), I(nVox - 1, nVox - 1, nVox - 1));
  v3 tMax = mul(sub(add(muls(add(vi2f(c), sp), v), lo), o), inv);
  v3 tDelta = vabs(muls(inv, v));
  float tIn = t;
  for (uint32_t it = 0; it < cap; it++) {
    out->steps++;
    i3 b = I(c.x >> 3, c.y >> 3, c.z >> 3);
    uint32_t ptr = vx->ptr[ptr_index(vx, L, b)];
    if (ptr == ORC_DROP) {
      uint32_t r[3];
      vox_at(vx, L, c, r);
      if (r[0] != ORC_EMPTY && tIn >= tskip) {
        float vl = vox_size(vx, r[2]);
        v3 pcl = add(lo, muls(adds(vi2f(c), 0.5f), v));
        v3 pc = muls(adds(vfloor(divs(pcl, vl)), 0.5f), vl);
        shade_voxel(cx, r[0], r[1], d, add(o, muls(d, tIn)), pc, vl, out);
        out->lvl = r[2]; out->ptr = r[0]; out->bit = r[1]; out->tin = ubits(tIn);
        return;
      }
      float tx = fminf_(fminf_(tMax.x, tMax.y), tMax.z);
      if (tx >= tEnd) break;
      tIn = tx;
      if (tMax.x <= tMax.y && tMax.x <= tMax.z) { c.x += st.x; tMax.x += tDelta.x; }
      else if (tMax.y <= tMax.z) { c.y += st.y; tMax.y += tDelta.y; }
      else { c.z += st.z; tMax.z += tDelta.z; }
      if (c.x < 0 || c.y < 0 || c.z < 0 || c.x >= nVox || c.y >= nVox || c.z >= nVox) break;
      continue;
    }
    if (ptr >= ORC_MARK) {
      v3 bt = mul(sub(add(muls(add(vi2f(I(b.x * 8, b.y * 8, b.z * 8)), muls(sp, 8.0f)), v), lo), o), inv);
      float te = fminf_(fminf_(bt.x, bt.y), bt.z);
      if (te >= tEnd) break;
      i3 nb = b;
      if (bt.x <= bt.y && bt.x <= bt.z) nb.x += st.x; else if (bt.y <= bt.z) nb.y += st.y; else nb.z += st.z;
      if (nb.x < 0 || nb.y < 0 || nb.z < 0 || nb.x >= G || nb.y >= G || nb.z >= G) break;
      t = te; tIn = te;
      c = iclamp3(vf2i(vfloor(divs(sub(add(o, muls(d, t)), lo), v))), I(nb.x * 8, nb.y * 8, nb.z * 8),
                  I(nb.x * 8 + 7, nb.y * 8 + 7, nb.z * 8 + 7));
      tMax = mul(sub(add(muls(add(vi2f(c), sp), v), lo), o), inv);
      continue;
    }
    uint32_t bit = (uint32_t)((c.x & 7) + 8 * (c.y & 7) + 64 * (c.z & 7));
    uint32_t occ = vx->occ[ptr * 16u + (bit >> 5)];
    float tExit = fminf_(fminf_(tMax.x, tMax.y), tMax.z);
    if ((occ & (1u << (bit & 31u))) != 0u && tIn >= tskip) {
      shade_voxel(cx, ptr, bit, d, add(o, muls(d, tIn)), add(lo, muls(adds(vi2f(c), 0.5f), v)), v, out);
      out->lvl = L; out->ptr = ptr; out->bit = bit; out->tin = ubits(tIn);
      return;
    }
    if (tExit >= tEnd) break;
    tIn = tExit;
    if (tMax.x <= tMax.y && tMax.x <= tMax.z) { c.x += st.x; tMax.x += tDelta.x; }
    else if (tMax.y <= tMax.z) { c.y += st.y; tMax.y += tDelta.y; }
    else { c.z += st.z; tMax.z += tDelta.z; }
    if (c.x < 0 || c.y < 0 || c.z < 0 || c.x >= nVox || c.y >= nVox || c.z >= nVox) break;
  }
}

/* voxLevel (rc.ts:210-213): round(log2(v / v0)) taken exactly, clamped to the levels. */
uint32_t vox_level(const orc_vox *vx, const orc_layout *ly, float s0, uint32_t c) {
  float v = ly->vox_scale * s0 * exp2_(ly->level_map * (float)c);
  int32_t r = (int32_t)orc_round_log2(v / vx->v0);
  int32_t top = (int32_t)vx->levels - 1;
  return (uint32_t)(r < 0 ? 0 : (r > top ? top : r));
}

typedef struct {
  const ctx_t *cx; const orc_layout *ly; orc_rc_out *o; uint32_t c;
  uint32_t n_traces, n_steps, n_cap;
} trace_job;

static void trace_range(void *p, uint64_t b, uint64_t e) {
  trace_job *j = (trace_job *)p;
  const orc_vox *vx = j->cx->vx;
  const orc_layout *ly = j->ly;
  orc_rc_out *o = j->o;
  const orc_casc *L = &ly->c[j->c];
  uint32_t dirs = L->res * L->res;
  uint32_t n_traces = 0, n_steps = 0, n_cap = 0;
  for (uint32_t t = (uint32_t)b; t < (uint32_t)e; t++) {
    uint32_t pi = t / dirs, di = t % dirs;
    const orc_probe *pr = &o->probes[L->probe_off + pi];
    trace_t tr;
    memset(&tr, 0, sizeof tr);
    tr.T = 1.0f; tr.lvl = ORC_EMPTY; tr.ptr = ORC_EMPTY;
    if (pr->pos[3] > 0.0f) {
      v3 dir = dir_of(di, L->res);
      float s0 = pr->pos[3];
      float t0 = L->b0 * s0, t1 = L->b1 * s0;
      v3 po = V(pr->pos[0], pr->pos[1], pr->pos[2]);
      v3 pn = V(pr->nrm[0], pr->nrm[1], pr->nrm[2]);
      uint32_t Lv = vox_level_for(vx, vox_level(vx, ly, s0, j->c), add(po, muls(dir, t1)));
      float v = vox_size(vx, Lv);
      v3 ooff = add(po, muls(pn, ly->vox_offset * v));
      trace_vox(j->cx, ooff, dir, t0, t1, ly->vox_skip * v, Lv, ly->dda_cap, &tr);
      dyn_compose(vx, po, dir, t0, t1, ooff, 3.5449077f / (float)L->res, &tr);
      n_traces += 1;
      n_steps += tr.steps;
      n_cap += tr.steps >= ly->dda_cap ? 1u : 0u;
    }
    float *r = o->rad + 4u * ((size_t)L->rad_off + t);
    r[0] = round_store(tr.r, ly->atlas); r[1] = round_store(tr.g, ly->atlas);
    r[2] = round_store(tr.b, ly->atlas); r[3] = round_store(tr.T, ly->atlas);
    if (o->hit) {
      uint32_t *h = o->hit + 4u * ((size_t)L->rad_off + t);
      h[0] = tr.lvl; h[1] = tr.ptr; h[2] = tr.bit; h[3] = tr.tin;
    }
  }
  __atomic_fetch_add(&j->n_traces, n_traces, __ATOMIC_RELAXED);
  __atomic_fetch_add(&j->n_steps, n_steps, __ATOMIC_RELAXED);
  __atomic_fetch_add(&j->n_cap, n_cap, __ATOMIC_RELAXED);
}

int orc_rc_trace(const orc_vox *vx, const orc_layout *ly, const orc_gbuf *g, orc_rc_out *o) {
  ctx_t cx = {vx, g->frame, {g->frame[F_SKY], g->frame[F_SKY + 1], g->frame[F_SKY + 2]}, NULL, NULL};
  const float *F = g->frame;
  int32_t W = (int32_t)g->width, H = (int32_t)g->height;
  memset(o->counts, 0, 80 * 4);
  /* setupScreen (rc.ts:572-590) */
  for (uint32_t c = 0; c < ly->cascades; c++) {
    const orc_casc *L = &ly->c[c];
    uint32_t n = L->tiles_x * L->tiles_y;
    o->counts[c] = n;
    for (uint32_t t = 0; t < n; t++) {
      uint32_t tx = t % L->tiles_x, ty = t / L->tiles_x;
      int32_t px = imin((int32_t)(tx * L->tile_size + L->tile_size / 2u), W - 1);
      int32_t py = imin((int32_t)(ty * L->tile_size + L->tile_size / 2u), H - 1);
      float d = g->depth[(size_t)py * (size_t)W + (size_t)px];
      orc_probe pr;
      memset(&pr, 0, sizeof pr);
      pr.grid[0] = (int32_t)tx; pr.grid[1] = (int32_t)ty;
      if (d > 0.0f) {
        v3 x = world_at(F, px, py, d);
        const float *nn = g->normal + 4u * ((size_t)py * (size_t)W + (size_t)px);
        v3 nrm = V(nn[0], nn[1], nn[2]);
        float s0 = length3(sub(x, fromf(F + F_EYE))) * F[F_RC + 1] * F[F_RC + 2];
        float e2 = exp2_((float)c);
        v3 p = add(x, muls(muls(muls(nrm, F[F_RC2]), s0), e2));
        pr.pos[0] = p.x; pr.pos[1] = p.y; pr.pos[2] = p.z; pr.pos[3] = s0;
        pr.nrm[0] = nrm.x; pr.nrm[1] = nrm.y; pr.nrm[2] = nrm.z; pr.nrm[3] = view_z(F, x);
      }
      o->probes[L->probe_off + t] = pr;
    }
  }
  /* trace (rc.ts:600-622) -> traceWorld (:216-245) -> traceVox */
  for (uint32_t c = 0; c < ly->cascades; c++) {
    const orc_casc *L = &ly->c[c];
    uint32_t dirs = L->res * L->res, np = L->tiles_x * L->tiles_y;
    trace_job j = {&cx, ly, o, c, 0, 0, 0};
    orc_parallel((uint64_t)np * dirs, 512, trace_range, &j);
    if (ly->stats > 0) { o->counts[24 + c] = j.n_traces; o->counts[32 + c] = j.n_steps; o->counts[64 + c] = j.n_cap; }
  }
  return 0;
}

/* upperAvg (rc.ts:681-686) */
v3 upper_avg(const orc_layout *ly, const float *rad, uint32_t cu, uint32_t q, uint32_t u, uint32_t v, uint32_t lr) {
  const orc_casc *U = &ly->c[cu];
  if (U->res == lr) {
    const float *p = rad + 4u * ((size_t)U->rad_off + q * U->res * U->res + v * U->res + u);
    return V(p[0], p[1], p[2]);
  }
  size_t base = (size_t)U->rad_off + q * U->res * U->res + v * 2u * U->res + u * 2u;
  const float *a = rad + 4u * base, *b = rad + 4u * (base + 1u), *c = rad + 4u * (base + U->res), *d = rad + 4u * (base + U->res + 1u);
  return muls(add(add(add(V(a[0], a[1], a[2]), V(b[0], b[1], b[2])), V(c[0], c[1], c[2])), V(d[0], d[1], d[2])), 0.25f);
}

void sh_basis(v3 n, float y[9]) {
  y[0] = 0.282095f; y[1] = 0.488603f * n.y; y[2] = 0.488603f * n.z; y[3] = 0.488603f * n.x;
  y[4] = 1.092548f * n.x * n.y; y[5] = 1.092548f * n.y * n.z; y[6] = 0.315392f * (3.0f * n.z * n.z - 1.0f);
  y[7] = 1.092548f * n.x * n.z; y[8] = 0.546274f * (n.x * n.x - n.y * n.y);
}

typedef struct { const orc_layout *ly; const orc_gbuf *g; orc_rc_out *o; uint32_t c; } mg_job;

/* mergeScreen (rc.ts:710-743), cascade j->c, in place */
static void merge_range(void *p, uint64_t b, uint64_t e) {
  mg_job *j = (mg_job *)p;
  const orc_layout *ly = j->ly;
  orc_rc_out *o = j->o;
  const float *F = j->g->frame;
  uint32_t c = j->c, N = ly->cascades;
  const orc_casc *L = &ly->c[c];
  uint32_t dirs = L->res * L->res;
  v3 sky = fromf(F + F_SKY);
  for (uint32_t t = (uint32_t)b; t < (uint32_t)e; t++) {
    uint32_t pi = t / dirs, di = t % dirs;
    float *rv = o->rad + 4u * ((size_t)L->rad_off + t);
    v3 up = sky;
    if (c + 1u < N && rv[3] > 0.0f) {
      up = V(0.0f, 0.0f, 0.0f);
      const orc_probe *pr = &o->probes[L->probe_off + pi];
      if (pr->pos[3] > 0.0f) {
        const orc_casc *U = &ly->c[c + 1u];
        float cx = ((float)(pi % L->tiles_x) + 0.5f) * (float)L->tile_size;
        float cy = ((float)(pi / L->tiles_x) + 0.5f) * (float)L->tile_size;
        float ux = cx / (float)U->tile_size - 0.5f, uy = cy / (float)U->tile_size - 0.5f;
        int32_t bx = f2i(floorf(ux)), by = f2i(floorf(uy));
        float fx = ux - (float)bx, fy = uy - (float)by;
        uint32_t u0 = di % L->res, v0 = di / L->res;
        v3 acc = V(0.0f, 0.0f, 0.0f);
        float ws = 0.0f;
        for (uint32_t k = 0; k < 4; k++) {
          int32_t ox = (int32_t)(k & 1u), oy = (int32_t)(k >> 1);
          int32_t qx = iclamp(bx + ox, 0, (int32_t)U->tiles_x - 1), qy = iclamp(by + oy, 0, (int32_t)U->tiles_y - 1);
          uint32_t qi = (uint32_t)qy * U->tiles_x + (uint32_t)qx;
          const orc_probe *qp = &o->probes[U->probe_off + qi];
          if (qp->pos[3] <= 0.0f) continue;
          float fwx = ox == 1 ? fx : 1.0f - fx, fwy = oy == 1 ? fy : 1.0f - fy;
          float rel = fabsf(qp->nrm[3] - pr->nrm[3]) / pr->nrm[3];
          float w = (fwx * fwy + 1e-4f) * (gi_exp(-20.0f * rel) + 1e-4f);
          acc = fmas(upper_avg(ly, o->rad, c + 1u, qi, u0, v0, L->res), w, acc);
          ws += w;
        }
        if (ws > 0.0f) up = divs(acc, ws);
      }
    }
    v3 m = fmas(up, rv[3], V(rv[0], rv[1], rv[2]));
    rv[0] = round_store(m.x, ly->atlas); rv[1] = round_store(m.y, ly->atlas); rv[2] = round_store(m.z, ly->atlas);
    rv[3] = round_store(1.0f, ly->atlas);
  }
}

/* projectSH (rc.ts:752-774) */
static void sh_range(void *p, uint64_t b, uint64_t e) {
  mg_job *j = (mg_job *)p;
  const orc_layout *ly = j->ly;
  orc_rc_out *o = j->o;
  const float *F = j->g->frame;
  const orc_casc *L0 = &ly->c[0];
  float a_k[3] = {PI_F, 2.0f * PI_F / 3.0f, PI_F / 4.0f};
  for (uint32_t pi = (uint32_t)b; pi < (uint32_t)e; pi++) {
    v3 cf[9];
    for (int k = 0; k < 9; k++) cf[k] = V(0.0f, 0.0f, 0.0f);
    for (uint32_t d = 0; d < 16; d++) {
      const float *rp = o->rad + 4u * ((size_t)L0->rad_off + pi * 16u + d);
      v3 r = muls(V(rp[0], rp[1], rp[2]), F[F_OMEGA + d]);
      float y[9];
      sh_basis(dir_of(d, 4u), y);
      for (int k = 0; k < 9; k++) cf[k] = fmas(r, y[k], cf[k]);
    }
    float *sh = o->sh + 32u * pi;
    for (int k = 0; k < 32; k++) sh[k] = 0.0f;
    for (int k = 0; k < 9; k++) {
      float a = k == 0 ? a_k[0] : (k < 4 ? a_k[1] : a_k[2]);
      sh[k * 3 + 0] = round_store(cf[k].x * a, ly->f32_out ? 0u : ly->atlas);
      sh[k * 3 + 1] = round_store(cf[k].y * a, ly->f32_out ? 0u : ly->atlas);
      sh[k * 3 + 2] = round_store(cf[k].z * a, ly->f32_out ? 0u : ly->atlas);
    }
  }
}

/* gatherScreen (rc.ts:929-954), rows [b, e) */
static void gather_range(void *p, uint64_t b, uint64_t e) {
  mg_job *j = (mg_job *)p;
  const orc_layout *ly = j->ly;
  const orc_gbuf *g = j->g;
  orc_rc_out *o = j->o;
  const float *F = g->frame;
  const orc_casc *L0 = &ly->c[0];
  int32_t W = (int32_t)g->width;
  uint32_t out_fmt = ((ly->atlas == 0 || ly->f32_out) && !ly->irr_f16) ? 0u : 1u;
  for (int32_t py = (int32_t)b; py < (int32_t)e; py++)
    for (int32_t px = 0; px < W; px++) {
      size_t q = (size_t)py * (size_t)W + (size_t)px;
      float *out = o->irr + 4u * q;
      float d = g->depth[q];
      if (!(d > 0.0f)) { out[0] = out[1] = out[2] = out[3] = 0.0f; continue; }
      v3 x = world_at(F, px, py, d);
      v3 n = V(g->normal[4 * q], g->normal[4 * q + 1], g->normal[4 * q + 2]);
      float z = view_z(F, x);
      float ux = ((float)px + 0.5f) / (float)L0->tile_size - 0.5f, uy = ((float)py + 0.5f) / (float)L0->tile_size - 0.5f;
      int32_t bx = f2i(floorf(ux)), by = f2i(floorf(uy));
      float fx = ux - (float)bx, fy = uy - (float)by;
      v3 acc = V(0.0f, 0.0f, 0.0f);
      float ws = 0.0f;
      float y[9];
      sh_basis(n, y);
      for (uint32_t k = 0; k < 4; k++) {
        int32_t ox = (int32_t)(k & 1u), oy = (int32_t)(k >> 1);
        int32_t qx = iclamp(bx + ox, 0, (int32_t)L0->tiles_x - 1), qy = iclamp(by + oy, 0, (int32_t)L0->tiles_y - 1);
        uint32_t qi = (uint32_t)qy * L0->tiles_x + (uint32_t)qx;
        const orc_probe *pr = &o->probes[L0->probe_off + qi];
        if (pr->pos[3] <= 0.0f) continue;
        float fwx = ox == 1 ? fx : 1.0f - fx, fwy = oy == 1 ? fy : 1.0f - fy;
        float rel = fabsf(pr->nrm[3] - z) / z;
        float nd = fmaxf_(dot(n, V(pr->nrm[0], pr->nrm[1], pr->nrm[2])), 0.0f);
        float w = (fwx * fwy + 1e-4f) * (gi_exp(-20.0f * rel) + 1e-4f) * (nd * nd * nd * nd + 1e-3f);
        /* evalSH (rc.ts:819-829) */
        const float *sh = o->sh + 32u * qi;
        v3 es = V(0.0f, 0.0f, 0.0f);
        for (int k2 = 0; k2 < 9; k2++) es = fmas(V(sh[3 * k2], sh[3 * k2 + 1], sh[3 * k2 + 2]), y[k2], es);
        es = vmax(es, V(0.0f, 0.0f, 0.0f));
        acc = fmas(es, w, acc);
        ws += w;
      }
      v3 r = ws > 0.0f ? divs(acc, ws) : V(0.0f, 0.0f, 0.0f);
      out[0] = out_fmt ? round_store(r.x, 1) : r.x;
      out[1] = out_fmt ? round_store(r.y, 1) : r.y;
      out[2] = out_fmt ? round_store(r.z, 1) : r.z;
      out[3] = 1.0f;
    }
}

int orc_rc_merge_gather(const orc_layout *ly, const orc_gbuf *g, orc_rc_out *o) {
  mg_job j = {ly, g, o, 0};
  for (int32_t ci = (int32_t)ly->cascades - 1; ci >= 0; ci--) {
    j.c = (uint32_t)ci;
    const orc_casc *L = &ly->c[j.c];
    orc_parallel((uint64_t)L->tiles_x * L->tiles_y * L->res * L->res, 4096, merge_range, &j);
  }
  orc_parallel((uint64_t)ly->c[0].tiles_x * ly->c[0].tiles_y, 256, sh_range, &j);
  orc_parallel(g->height, 4, gather_range, &j);
  return 0;
}

/* ---- the multi-bounce volume's frame (bounce.ts:96-246, Bounce.encode :356-368) ---- */
#define BN_DDA_CAP 1024u   /* traceVox's step cap (voxel.ts:142) for the volume's rays */

static float f16r(float x) { return orc_f16_to_f32(orc_f32_to_f16(x)); }
static void bn_put(const orc_bounce *b, float *vol, i3 c, int a, float x, float y, float z, float w) {
  float *t = vol + (((size_t)(a * (int32_t)b->dz + c.z) * b->dy + (size_t)c.y) * b->dx + (size_t)c.x) * 4u;
  t[0] = f16r(x); t[1] = f16r(y); t[2] = f16r(z); t[3] = f16r(w);
}
/* occAt (bounce.ts:99-104) */
static int bn_occ_at(const orc_vox *vx, uint32_t L, v3 p) {
  float vs = vox_size(vx, L);
  i3 c = vf2i(vfloor(divs(sub(p, muls(muls(vi2f(org(vx, L)), vs), 8.0f)), vs)));
  int32_t n = (int32_t)vx->G * 8;
  if (c.x < 0 || c.y < 0 || c.z < 0 || c.x >= n || c.y >= n || c.z >= n) return 0;
  uint32_t r[3];
  vox_at(vx, L, c, r);
  return r[0] != ORC_EMPTY;
}
/* bnTrace (bounce.ts:156-167) */
static void bn_trace(const ctx_t *cx, const orc_bounce *b, v3 o, v3 d, float tmax, float out[4]) {
  const orc_vox *vx = cx->vx;
  float b0 = 0.0f;
  for (uint32_t k = 0; k < vx->levels && b0 * b->cell < tmax; k++) {
    float b1 = b0 * 4.0f + 1.0f;
    uint32_t L = vox_level_for(vx, k, add(o, muls(muls(d, b1), b->cell)));
    trace_t r;
    trace_vox(cx, o, d, b0 * b->cell, fminf_(b1 * b->cell, tmax), 0.0f, L, BN_DDA_CAP, &r);
    if (r.T < 0.5f) {
      v3 entry = add(o, muls(d, fbits(r.tin)));
      out[0] = r.r; out[1] = r.g; out[2] = r.b; out[3] = dot(sub(entry, o), d);
      return;
    }
    b0 = b1;
  }
  out[0] = cx->sky[0]; out[1] = cx->sky[1]; out[2] = cx->sky[2]; out[3] = 1e9f;
}
static v3 bn_axis_vec(uint32_t a) {
  float s = (a & 1u) == 1u ? -1.0f : 1.0f;
  return a / 2u == 0u ? V(s, 0.0f, 0.0f) : (a / 2u == 1u ? V(0.0f, s, 0.0f) : V(0.0f, 0.0f, s));
}

/* dynE of the bounce volume (bounce.ts:267-296): the irradiance at p of a dynamic voxel with projected areas P over
 * its six axis faces, E = sum_a P_a E_a / sum_a P_a, E_a trilinear over the 8 probes around p with bnRead's rules
 * (active, reach, side of the face) */
static v3 dyn_e(const orc_bounce *b, const float *vol, v3 p, const float P[6]) {
  i3 org0 = bn_origin(b, vol);
  v3 g = sub(V(p.x / b->cell, p.y / b->cell, p.z / b->cell), vi2f(org0));
  i3 bb = vf2i(vfloor(g));
  v3 fr = sub(g, vi2f(bb));
  float tol = 0.5f * b->v0;
  v3 e[6];
  float ws[6];
  for (int a = 0; a < 6; a++) { e[a] = V(0.0f, 0.0f, 0.0f); ws[a] = 0.0f; }
  for (int k = 0; k < 8; k++) {
    i3 off = I(k & 1, (k >> 1) & 1, (k >> 2) & 1);
    i3 cc = I(bb.x + off.x, bb.y + off.y, bb.z + off.z);
    if (cc.x < 0 || cc.y < 0 || cc.z < 0 || cc.x >= (int32_t)b->dx || cc.y >= (int32_t)b->dy || cc.z >= (int32_t)b->dz) continue;
    v3 pp = muls(vi2f(I(org0.x + cc.x, org0.y + cc.y, org0.z + cc.z)), b->cell);
    v3 u = sub(p, pp);
    if (bn_axis_a(b, vol, cc, 0) <= 0.0f) continue;
    if (fabsf(u.x) > bn_axis_a(b, vol, cc, u.x >= 0.0f ? 0 : 1) + tol || fabsf(u.y) > bn_axis_a(b, vol, cc, u.y >= 0.0f ? 2 : 3) + tol
        || fabsf(u.z) > bn_axis_a(b, vol, cc, u.z >= 0.0f ? 4 : 5) + tol) continue;
    v3 t3 = V(off.x == 1 ? fr.x : 1.0f - fr.x, off.y == 1 ? fr.y : 1.0f - fr.y, off.z == 1 ? fr.z : 1.0f - fr.z);
    float wt = t3.x * t3.y * t3.z;
    for (int a = 0; a < 6; a++) {
      if (P[a] <= 0.0f) continue;
      float w = wt * smoothstep_(-0.05f, 0.25f, dot(sub(pp, p), bn_axis_vec((uint32_t)a)) / b->cell);
      if (w <= 0.0f) continue;
      e[a] = add(e[a], muls(bn_axis_rgb(b, vol, cc, a), w));
      ws[a] += w;
    }
  }
  v3 sum = V(0.0f, 0.0f, 0.0f);
  float ps = 0.0f;
  for (int a = 0; a < 6; a++) {
    if (ws[a] > 1e-6f) sum = add(sum, divs(muls(e[a], P[a]), ws[a]));
    ps += P[a];
  }
  return divs(sum, fmaxf_(ps, 1e-9f));
}

/* dynInject (dynlayer.ts:173-191), phase 31: every voxel of the layer's allocated bricks with area adds albedo / pi
 * times dynE of the previous frame's volume to its radiance (the layer as this frame's build left it) */
static void dyn_inject_bounce(const orc_bounce *b, const orc_vox *vx, orc_dyn *dl, const float *prev) {
  const uint32_t G = vx->G, G3 = G * G * G;
  const uint32_t slots = dl->hdr[8] < dl->nb ? dl->hdr[8] : dl->nb;
  for (uint32_t slot = 0; slot < slots; slot++) {
    const uint32_t pi = dl->meta[slot], L = pi / G3, r = pi % G3;
    for (uint32_t bit = 0; bit < 512u; bit++) {
      const uint32_t base = (slot * 512u + bit) * 13u;
      if (dyn_word_at(dl, base, 6u, L) <= 0.0f) continue;
      float P[6];
      for (uint32_t k = 0; k < 6u; k++) P[k] = dyn_word_at(dl, base, k, L);
      i3 c = I((int32_t)(r % G) * 8 + (int32_t)(bit & 7u), (int32_t)((r / G) % G) * 8 + (int32_t)((bit >> 3) & 7u),
               (int32_t)(r / (G * G)) * 8 + (int32_t)(bit >> 6));
      float v = vox_size(vx, L);
      v3 p = add(muls(muls(vi2f(org(vx, L)), v), 8.0f), muls(adds(vi2f(c), 0.5f), v));
      v3 E = dyn_e(b, prev, p, P);
      v3 alb = V(dyn_word_at(dl, base, 10u, L), dyn_word_at(dl, base, 11u, L), dyn_word_at(dl, base, 12u, L));
      v3 a = mul(divs(alb, PI_F), E);
      float add3[3] = {a.x, a.y, a.z};
      dyn_add_radiance(dl, base, L, add3);
    }
  }
}

int orc_bounce_frame(orc_bounce *b, const orc_vox *vx, const float *F, float *inj_out) {
  /* phase 31: the layer receives the previous frame's volume (the last one written) before it is swapped */
  const int objects = b->objects && vx->dyn;
  if (objects) dyn_inject_bounce(b, vx, (orc_dyn *)vx->dyn, b->vol[b->list[2]]);
  /* bnClear */
  b->list[0] = 0u; b->list[1] += 1u; b->list[2] ^= 1u;
  float *cur = b->vol[b->list[2]];
  const float *prev = b->vol[b->list[2] ^ 1u];
  const uint32_t n = b->dx * b->dy * b->dz;
  const i3 o = I(f2i(floorf(F[F_EYE] / b->cell)) - (int32_t)(b->dx / 2u), f2i(floorf(F[F_EYE + 1] / b->cell)) - (int32_t)(b->dy / 2u),
                 f2i(floorf(F[F_EYE + 2] / b->cell)) - (int32_t)(b->dz / 2u));
  /* bnClassify (bounce.ts:112-138) */
  bn_put(b, cur, I(0, 0, 0), 6, (float)o.x, (float)o.y, (float)o.z, 0.0f);
  int32_t lr = (int32_t)orc_round_log2(fmaxf_(b->cell, 1e-4f) / b->v0);
  uint32_t L = (uint32_t)(lr < 0 ? 0 : (lr > (int32_t)vx->levels - 1 ? (int32_t)vx->levels - 1 : lr));
  for (uint32_t i = 0; i < n; i++) {
    i3 c = I((int32_t)(i % b->dx), (int32_t)((i / b->dx) % b->dy), (int32_t)(i / (b->dx * b->dy)));
    v3 p = muls(vi2f(I(o.x + c.x, o.y + c.y, o.z + c.z)), b->cell);
    int near = 0;
    for (uint32_t k = 0; k < 8u && !near; k++)
      near = bn_occ_at(vx, L, add(p, muls(adds(V((float)(k & 1u), (float)((k >> 1) & 1u), (float)(k >> 2)), -0.5f), b->cell)));
    if (near && !bn_occ_at(vx, 0u, p)) {
      i3 w = I(o.x + c.x, o.y + c.y, o.z + c.z);
      if (b->div > 1u && ((uint32_t)(w.x + w.y + w.z + 1048576) + b->list[1]) % b->div != 0u) {
        i3 po = bn_origin(b, prev);
        i3 pc = I(w.x - po.x, w.y - po.y, w.z - po.z);
        if (pc.x >= 0 && pc.y >= 0 && pc.z >= 0 && pc.x < (int32_t)b->dx && pc.y < (int32_t)b->dy && pc.z < (int32_t)b->dz
            && bn_axis_a(b, prev, pc, 0) > 0.0f) {
          for (int a = 0; a < 6; a++) {
            v3 t = bn_axis_rgb(b, prev, pc, a);
            bn_put(b, cur, c, a, t.x, t.y, t.z, bn_axis_a(b, prev, pc, a));
          }
          continue;
        }
      }
      b->list[4u + b->list[0]++] = i;
    } else {
      for (int a = 0; a < 6; a++) bn_put(b, cur, c, a, 0.0f, 0.0f, 0.0f, 0.0f);
    }
  }
  /* bnUpdate (bounce.ts:172-208) */
  ctx_t cx = {vx, F, {F[F_SKY], F[F_SKY + 1], F[F_SKY + 2]}, b, prev};
  float rad[64][4];
  float reach[6];
  for (uint32_t slot = 0; slot < b->list[0]; slot++) {
    uint32_t i = b->list[4u + slot];
    i3 c = I((int32_t)(i % b->dx), (int32_t)((i / b->dx) % b->dy), (int32_t)(i / (b->dx * b->dy)));
    v3 p = muls(vi2f(I(o.x + c.x, o.y + c.y, o.z + c.z)), b->cell);
    for (uint32_t r = 0; r < b->rays; r++) {
      bn_trace(&cx, b, p, fromf(b->dirs + 4u * r), 1e9f, rad[r]);
      if (objects) {   /* bnTraceDyn (bounce.ts:169-174): the layer in front of the static result, one ray's cone */
        float oo[3] = {p.x, p.y, p.z}, dd[3] = {b->dirs[4u * r], b->dirs[4u * r + 1u], b->dirs[4u * r + 2u]}, dl[4];
        orc_trace_dyn(vx, oo, dd, 0.0f, fminf_(rad[r][3], 1e4f), sqrtf((4.0f * PI_F) / (float)b->rays), dl);
        for (int k = 0; k < 3; k++) rad[r][k] = dl[k] + (1.0f - dl[3]) * rad[r][k];
      }
    }
    for (uint32_t a = 0; a < 6u; a++) {
      float t[4];
      bn_trace(&cx, b, p, bn_axis_vec(a), 1.5f * b->cell, t);
      reach[a] = fmaxf_(fminf_(t[3], 1.5f * b->cell), 1e-3f);
    }
    for (uint32_t a = 0; a < 6u; a++) {
      v3 axis = bn_axis_vec(a), e = V(0.0f, 0.0f, 0.0f);
      float ws = 0.0f;
      for (uint32_t r = 0; r < b->rays; r++) {
        float w = fmaxf_(dot(axis, fromf(b->dirs + 4u * r)), 0.0f);
        e = add(e, muls(V(rad[r][0], rad[r][1], rad[r][2]), w));
        ws += w;
      }
      v3 irr = divs(muls(e, PI_F), fmaxf_(ws, 1e-6f));
      bn_put(b, cur, c, (int)a, irr.x, irr.y, irr.z, reach[a]);
    }
  }
  /* bnInject (bounce.ts:213-246) */
  uint32_t nb = vx->hdr[0] < vx->max_bricks ? vx->hdr[0] : vx->max_bricks;
  for (uint32_t ptr = 0; ptr < nb; ptr++) {
    uint32_t first = vx->base[ptr];
    if (first >= ORC_MARK) continue;
    uint32_t code = vx->code[ptr], Lv = code >> 27;
    i3 bc = I((int32_t)((code >> 18) & 511u), (int32_t)((code >> 9) & 511u), (int32_t)(code & 511u));
    float vs = vox_size(vx, Lv);
    v3 lo = muls(muls(vi2f(org(vx, Lv)), vs), 8.0f);
    uint32_t r = 0;
    for (uint32_t bit = 0; bit < 512u; bit++) {
      if ((vx->occ[ptr * 16u + (bit >> 5)] & (1u << (bit & 31u))) == 0u) continue;
      uint32_t ai = first + r++;
      i3 cc = I(bc.x * 8 + (int32_t)(bit & 7u), bc.y * 8 + (int32_t)((bit >> 3) & 7u), bc.z * 8 + (int32_t)(bit >> 6));
      v3 p = add(lo, muls(adds(vi2f(cc), 0.5f), vs));
      uint32_t e = vx->attr[ai * 4u + 1u];
      float ex = fmaxf_((float)(int16_t)(e & 0xffffu) / 32767.0f, -1.0f);
      float ey = fmaxf_((float)(int16_t)(e >> 16) / 32767.0f, -1.0f);
      v3 nn = V(ex, ey, 1.0f - fabsf(ex) - fabsf(ey));
      float q0 = fmaxf_(-nn.z, 0.0f);
      nn.x += nn.x >= 0.0f ? -q0 : q0;
      nn.y += nn.y >= 0.0f ? -q0 : q0;
      v3 nf = dot(nn, nn) > 0.01f ? normalize3(nn) : V(0.0f, 1.0f, 0.0f);
      float off = Lv == 0u ? 0.0f : 0.5f * vs;
      v3 ef = bn_read(b, cur, add(p, muls(nf, off)), p, nf);
      v3 eb = bn_read(b, cur, add(p, muls(neg(nf), off)), p, neg(nf));
      float *q = inj_out + (size_t)ai * 6u;
      q[0] = f16r(ef.x); q[1] = f16r(ef.y); q[2] = f16r(ef.z); q[3] = f16r(eb.x); q[4] = f16r(eb.y); q[5] = f16r(eb.z);
    }
  }
  return 0;
}
