// Screen-probe radiance cascades traced in the voxel clipmap, on sm_100a (src/core/rc.ts, method 'screen', world
// tracer 'voxel': setupScreen :572, trace :600 -> traceWorld :216 -> traceVox voxel.ts:121, mergeScreen :710,
// projectSH :752, gatherScreen :929).
//
// Form changes from the reference's dispatches, results unchanged:
//  * setupScreen and trace each run once over all cascades (the reference dispatches them per cascade); the texel
//    directions are tabulated once per Rc and each probe's voxel level once per solve (same functions, same bits);
//  * the trace kernel is persistent: each warp takes 32 rays at a time from a global ray counter;
//  * indirect dispatches become launches sized from the host-known probe counts (screen probes: tiles).
#include <cuda_runtime.h>

#include "gi_dev.cuh"
#include "gi_internal.h"
#include "gi_scan.cuh"

namespace gi {

// voxRank (voxel.ts:81-87)
// (the brick's 16 words in four 128-bit loads; words past the bit's word masked out)
__device__ __forceinline__ uint32_t vox_rank(const VoxDev &v, uint32_t brick, uint32_t bit) {
  uint32_t w = bit >> 5, part = (1u << (bit & 31u)) - 1u;
  const uint4 *o = reinterpret_cast<const uint4 *>(v.occ + brick * 16u);
  uint32_t r = 0;
#pragma unroll
  for (uint32_t q = 0; q < 4; q++) {
    uint4 x = __ldg(&o[q]);
    uint32_t wd[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
    for (uint32_t k = 0; k < 4; k++) {
      uint32_t i = 4u * q + k;
      r += __popc(wd[k] & (i < w ? 0xffffffffu : (i == w ? part : 0u)));
    }
  }
  return v.base[brick] + r;
}

// voxAt (voxel.ts:90-107): brick, bit, level (brick GI_EMPTY when empty)
__device__ __forceinline__ uint3 vox_at(const VoxDev &v, uint32_t L, i3 c) {
  uint32_t l = L;
  i3 cc = c;
  int n8 = (int)v.G * 8;
  for (;;) {
    uint32_t ptr = v.ptr[ptr_index(v, l, mki(cc.x >> 3, cc.y >> 3, cc.z >> 3))];
    if (ptr != GI_DROP) {
      if (ptr >= GI_MARK) return make_uint3(GI_EMPTY, 0u, l);
      uint32_t bit = (uint32_t)((cc.x & 7) + 8 * (cc.y & 7) + 64 * (cc.z & 7));
      if ((v.occ[ptr * 16u + (bit >> 5)] & (1u << (bit & 31u))) == 0u) return make_uint3(GI_EMPTY, 0u, l);
      return make_uint3(ptr, bit, l);
    }
    if (l + 1u >= v.levels) return make_uint3(GI_EMPTY, 0u, l);
    i3 o = org(v, l);
    i3 w = mki((o.x * 8 + cc.x) >> 1, (o.y * 8 + cc.y) >> 1, (o.z * 8 + cc.z) >> 1);
    l++;
    i3 o1 = org(v, l);
    cc = mki(w.x - o1.x * 8, w.y - o1.y * 8, w.z - o1.z * 8);
    if (cc.x < 0 || cc.y < 0 || cc.z < 0 || cc.x >= n8 || cc.y >= n8 || cc.z >= n8) return make_uint3(GI_EMPTY, 0u, l);
  }
}

// voxInside / voxLevelFor (voxel.ts:108-119)
__device__ __forceinline__ bool vox_inside(const VoxDev &v, uint32_t L, f3 p) {
  const f3 lo = mk(v.box_lo[L][0], v.box_lo[L][1], v.box_lo[L][2]), hi = mk(v.box_hi[L][0], v.box_hi[L][1], v.box_hi[L][2]);
  return p.x > lo.x && p.y > lo.y && p.z > lo.z && p.x < hi.x && p.y < hi.y && p.z < hi.z;
}
__device__ __forceinline__ uint32_t vox_level_for(const VoxDev &v, uint32_t L, f3 e) {
  uint32_t l = L;
  while (l + 1u < v.levels && !vox_inside(v, l, e)) l++;
  return l;
}

// style.ts:18-25
__device__ __forceinline__ f3 toon_albedo(f3 a) {
  float l = dot(a, mk(0.2126f, 0.7152f, 0.0722f));
  f3 r = mk(l, l, l) + (a - mk(l, l, l)) * 1.6f;
  return mk(fclampf(r.x, 0.0f, 1.0f), fclampf(r.y, 0.0f, 1.0f), fclampf(r.z, 0.0f, 1.0f));
}
__device__ __forceinline__ float toon_ramp(float x) { return x > 0.3f ? 1.0f : (x > 0.05f ? 0.5f : 0.0f); }

// ---- multi-bounce reads (bounce.ts:44-75, 90-93; rc.ts:198-202) ---------------------------------------------------
__device__ __forceinline__ float4 bn_texel(const BounceDev &b, const uint2 *vol, int x, int y, int z) {
  uint2 u = vol[((size_t)z * b.dy + (size_t)y) * b.dx + (size_t)x];
  return make_float4(h2f(u.x & 0xffffu), h2f(u.x >> 16), h2f(u.y & 0xffffu), h2f(u.y >> 16));
}
__device__ __forceinline__ float4 bn_axis(const BounceDev &b, const uint2 *vol, i3 c, int a) {
  return bn_texel(b, vol, c.x, c.y, a * (int)b.dz + c.z);
}
__device__ __forceinline__ i3 bn_origin(const BounceDev &b, const uint2 *vol) {   // bnOrigin
  float4 o = bn_texel(b, vol, 0, 0, 6 * (int)b.dz);
  return mki(f2i(o.x), f2i(o.y), f2i(o.z));
}
// WGSL smoothstep: t = clamp((x - e0) / (e1 - e0), 0, 1), t t (3 - 2 t)
__device__ __forceinline__ float smoothstep_(float e0, float e1, float x) {
  float t = fclampf((x - e0) / (e1 - e0), 0.0f, 1.0f);
  return t * t * (3.0f - 2.0f * t);
}
// bnRead (bounce.ts:49-74): the irradiance on the side n of a surface at p, read at q, trilinear over the 8 probes
// around q that are active, on that side and whose reach along their axes covers q
__device__ f3 bn_read(const BounceDev &b, const uint2 *vol, f3 q, f3 p, f3 n) {
  const i3 org = bn_origin(b, vol);
  const f3 g = mk(q.x / b.cell, q.y / b.cell, q.z / b.cell) - vi2f(org);
  const i3 bb = vfloori(g);
  const f3 fr = g - vi2f(bb), n2 = n * n;
  const float tol = 0.5f * b.v0;
  f3 e = mk(0.0f, 0.0f, 0.0f);
  float ws = 0.0f;
  for (int k = 0; k < 8; k++) {
    const i3 off = mki(k & 1, (k >> 1) & 1, (k >> 2) & 1);
    const i3 cc = mki(bb.x + off.x, bb.y + off.y, bb.z + off.z);
    if (cc.x < 0 || cc.y < 0 || cc.z < 0 || cc.x >= (int)b.dx || cc.y >= (int)b.dy || cc.z >= (int)b.dz) continue;
    const f3 pp = vi2f(mki(org.x + cc.x, org.y + cc.y, org.z + cc.z)) * b.cell;
    const f3 u = q - pp;
    if (bn_axis(b, vol, cc, 0).w <= 0.0f) continue;
    if (fabsf(u.x) > bn_axis(b, vol, cc, u.x >= 0.0f ? 0 : 1).w + tol || fabsf(u.y) > bn_axis(b, vol, cc, u.y >= 0.0f ? 2 : 3).w + tol
        || fabsf(u.z) > bn_axis(b, vol, cc, u.z >= 0.0f ? 4 : 5).w + tol) continue;
    const f3 t3 = mk(off.x == 1 ? fr.x : 1.0f - fr.x, off.y == 1 ? fr.y : 1.0f - fr.y, off.z == 1 ? fr.z : 1.0f - fr.z);
    const float w = t3.x * t3.y * t3.z * smoothstep_(-0.05f, 0.25f, dot(pp - p, n) / b.cell);
    if (w <= 0.0f) continue;
    const float4 ax = bn_axis(b, vol, cc, n.x >= 0.0f ? 0 : 1), ay = bn_axis(b, vol, cc, n.y >= 0.0f ? 2 : 3);
    const float4 az = bn_axis(b, vol, cc, n.z >= 0.0f ? 4 : 5);
    e = e + ((mk(ax.x, ax.y, ax.z) * n2.x + mk(ay.x, ay.y, ay.z) * n2.y) + mk(az.x, az.y, az.z) * n2.z) * w;
    ws += w;
  }
  return ws > 1e-6f ? e / ws : mk(0.0f, 0.0f, 0.0f);
}
// voxSide (rc.ts:120-124): the side of the voxel the ray comes from
__device__ __forceinline__ float vox_side(f3 p, f3 n, f3 d, f3 pc, float v) {
  float s = dot(p - pc, n);
  if (fabsf(s) > 0.05f * v) return s > 0.0f ? 1.0f : -1.0f;
  return dot(n, d) > 0.0f ? -1.0f : 1.0f;
}
// The cascades' voxBounce (rc.ts:198-202): the irradiance bnInject stored for the side the ray comes from; 0 with
// multi-bounce off
struct InjectedBounce {
  const uint4 *inj;
  __device__ __forceinline__ f3 operator()(uint32_t ai, bool has, f3 p, f3 n, f3 d, f3 pc, float v) const {
    if (!inj || !has) return mk(0.0f, 0.0f, 0.0f);
    const uint4 w = inj[ai];
    const bool back = vox_side(p, n, d, pc, v) < 0.0f;
    const uint32_t a = back ? w.z : w.x, c = back ? w.w : w.y;
    return mk(h2f(a & 0xffffu), h2f(a >> 16), h2f(c & 0xffffu));
  }
};
// The bounce volume's own rays (bounce.ts:90-93): the previous frame's volume, read at the hit
struct VolumeBounce {
  const BounceDev *b;
  const uint2 *prev;
  __device__ __forceinline__ f3 operator()(uint32_t, bool has, f3 p, f3 n, f3 d, f3 pc, float v) const {
    if (!has) return mk(0.0f, 0.0f, 0.0f);   // no attributes: the albedo is 0 and so is the reflected term
    if (dot(n, n) <= 0.01f) return bn_read(*b, prev, p, p, -d);
    return bn_read(*b, prev, p, p, n * vox_side(p, n, d, pc, v));
  }
};

// voxShade (rc.ts:136-140) -> shadeHitV (rc.ts:108-116), plus the voxel's emissive radiance.  entry: where the ray
// enters the voxel; pc, vsz: the voxel's centre and size; bs: the irradiance e of the multi-bounce term at the shading
// point p = entry - d vsz / 4.
template <class BS>
__device__ __forceinline__ f3 shade_voxel(const VoxDev &v, const float *__restrict__ F, const float *__restrict__ r_unorm8,
                                          uint32_t brick, uint32_t bit, f3 d, f3 entry, f3 pc, float vsz, const BS &bs) {
  uint4 w = make_uint4(0, 0, 0, 0);
  float vis = 0.0f;
  uint32_t ai = 0;
  const bool has = v.base[brick] != GI_EMPTY;
  if (has) {
    ai = vox_rank(v, brick, bit);
    w = v.attr[ai];
    vis = v.sunvis[ai];
  }
  // k / 255 for a byte k: the quotients, tabulated (the same IEEE quotients as dividing)
  float alb0 = __ldg(&r_unorm8[w.x & 0xffu]), alb1 = __ldg(&r_unorm8[(w.x >> 8) & 0xffu]);
  float alb2 = __ldg(&r_unorm8[(w.x >> 16) & 0xffu]), alb3 = __ldg(&r_unorm8[w.x >> 24]);
  // unpack2x16snorm: the IEEE quotients k / 32767 without a division (snorm16)
  float nx = snorm16(w.y & 0xffffu), ny = snorm16(w.y >> 16);
  f3 n0 = mk(nx, ny, 1.0f - fabsf(nx) - fabsf(ny));
  float q = mx(-n0.z, 0.0f);
  n0.x += n0.x >= 0.0f ? -q : q;
  n0.y += n0.y >= 0.0f ? -q : q;
  // shadeHitV
  f3 n = dot(n0, n0) > 0.01f ? n0 : -d;
  if (dot(n, d) > 0.0f) n = -n;
  f3 a = mk(alb0, alb1, alb2);
  // a / pi for the 256 albedo values a = k / 255: the f32 quotients, tabulated after the k / 255 table
  const f3 api = mk(__ldg(&r_unorm8[256u + (w.x & 0xffu)]), __ldg(&r_unorm8[256u + ((w.x >> 8) & 0xffu)]),
                    __ldg(&r_unorm8[256u + ((w.x >> 16) & 0xffu)]));
  // the multi-bounce term b = a / pi * e (+0 with e = 0)
  f3 r = api * bs(ai, has, entry - d * (0.25f * vsz), n0, d, pc, vsz);
  float ndl = mx(dot(n, mk(F[F_SUN], F[F_SUN + 1], F[F_SUN + 2])), 0.0f);
  if (ndl > 0.0f) {
    f3 sunE = mk(F[F_SUNE], F[F_SUNE + 1], F[F_SUNE + 2]);
    if (alb3 > 0.5f && F[F_STYLE] > 0.5f) r = r + ((toon_albedo(a) / 3.14159265f) * sunE) * toon_ramp(ndl * vis);
    else r = r + ((api * sunE) * ndl) * vis;
  }
  return r + mk(h2f(w.z & 0xffffu), h2f(w.z >> 16), h2f(w.w & 0xffffu));
}

struct TraceOut { f3 rad; float T; uint32_t lvl, ptr, bit, tin, steps; };

// traceVox (voxel.ts:121-202) as its set-up and one iteration of its loop; the f32 operations and their order are the
// reference's.  The box of each level and 1 / d come from tables (VoxDev.box_lo/box_hi, RcDev.idirs) holding the
// same numbers.
struct Dda {
  f3 o, d, inv, lo, tMax, tDelta, sp;
  i3 c, st;
  float vs, tEnd, tskip, tIn;
  uint32_t L, steps;
};
enum { DDA_WALK = 0, DDA_MISS = 1, DDA_HIT = 2, DDA_HIT_DROP = 3 };

// what the walk needs besides its position: the level's voxel size and box, the step signs and the cell increments
__device__ __forceinline__ void dda_derived(const VoxDev &v, Dda &s) {
  s.vs = vox_size(v, s.L);
  s.lo = mk(v.box_lo[s.L][0], v.box_lo[s.L][1], v.box_lo[s.L][2]);
  const f3 dd = mk(fabsf(s.d.x) < 1e-9f ? 1e-9f : s.d.x, fabsf(s.d.y) < 1e-9f ? 1e-9f : s.d.y,
                   fabsf(s.d.z) < 1e-9f ? 1e-9f : s.d.z);
  s.st = mki(dd.x > 0.0f ? 1 : -1, dd.y > 0.0f ? 1 : -1, dd.z > 0.0f ? 1 : -1);
  s.sp = mk(s.st.x > 0 ? 1.0f : 0.0f, s.st.y > 0 ? 1.0f : 0.0f, s.st.z > 0 ? 1.0f : 0.0f);
  s.tDelta = vabs(s.inv * s.vs);
}

// traceVox's set-up (voxel.ts:122-138): false when the interval misses the level's box (T = 1, no step taken).
// inv_pre: the direction's 1 / d with tiny components clamped, tabulated with the directions (the same IEEE
// quotients), or null to divide here.
__device__ __forceinline__ bool dda_begin(const VoxDev &v, f3 o, f3 d, float t0, float t1, float tskip, uint32_t L,
                                          const float4 *inv_pre, Dda &s) {
  s.o = o; s.d = d; s.L = L; s.steps = 0; s.tskip = tskip;
  if (inv_pre) {
    const float4 q = __ldg(inv_pre);
    s.inv = mk(q.x, q.y, q.z);
  } else {
    const f3 dd = mk(fabsf(d.x) < 1e-9f ? 1e-9f : d.x, fabsf(d.y) < 1e-9f ? 1e-9f : d.y, fabsf(d.z) < 1e-9f ? 1e-9f : d.z);
    s.inv = mk(1.0f / dd.x, 1.0f / dd.y, 1.0f / dd.z);
  }
  dda_derived(v, s);
  const f3 hi = mk(v.box_hi[L][0], v.box_hi[L][1], v.box_hi[L][2]);
  const f3 ta = (s.lo - o) * s.inv, tb = (hi - o) * s.inv;
  const f3 tn = vmin(ta, tb), tf = vmax(ta, tb);
  const float t = mx(mx(mx(tn.x, tn.y), tn.z), t0);
  s.tEnd = mn(mn(mn(tf.x, tf.y), tf.z), t1);
  if (t >= s.tEnd) return false;
  const int nVox = (int)v.G * 8;
  s.c = iclamp3(vfloori(((o + d * t) - s.lo) / s.vs), mki(0, 0, 0), mki(nVox - 1, nVox - 1, nVox - 1));
  s.tMax = (((vi2f(s.c) + s.sp) * s.vs + s.lo) - o) * s.inv;
  s.tIn = t;
  return true;
}

// One iteration of traceVox's loop (voxel.ts:142-200) under a step cap: DDA_WALK to go on, DDA_MISS when the walk
// ends empty, DDA_HIT (h = brick, bit, level L) or DDA_HIT_DROP (h = voxAt's brick, bit and coarser level) on the
// first occupied voxel entered at tIn >= tSkip.  `steps` counts the iterations taken (rc.ts:232-235).
__device__ __forceinline__ int dda_step(const VoxDev &v, Dda &s, uint32_t cap, uint3 &h) {
  if (s.steps >= cap) return DDA_MISS;
  s.steps++;
  const int G = (int)v.G, nVox = G * 8;
  const i3 b = mki(s.c.x >> 3, s.c.y >> 3, s.c.z >> 3);
  const uint32_t ptr = __ldg(&v.ptr[s.L * (uint32_t)(G * G * G) + ((uint32_t)b.z * (uint32_t)G + (uint32_t)b.y) * (uint32_t)G
                                    + (uint32_t)b.x]);
  if (ptr == GI_DROP) {
    // dropped brick: voxel by voxel, each read at the coarser level that holds it
    const uint3 r = vox_at(v, s.L, s.c);
    if (r.x != GI_EMPTY && s.tIn >= s.tskip) { h = r; return DDA_HIT_DROP; }
    const float tx = mn(mn(s.tMax.x, s.tMax.y), s.tMax.z);
    if (tx >= s.tEnd) return DDA_MISS;
    s.tIn = tx;
  } else if (ptr >= GI_MARK) {
    // empty brick: jump to its exit
    const f3 bt = (((vi2f(mki(b.x * 8, b.y * 8, b.z * 8)) + s.sp * 8.0f) * s.vs + s.lo) - s.o) * s.inv;
    const float te = mn(mn(bt.x, bt.y), bt.z);
    if (te >= s.tEnd) return DDA_MISS;
    i3 nb = b;
    if (bt.x <= bt.y && bt.x <= bt.z) nb.x += s.st.x; else if (bt.y <= bt.z) nb.y += s.st.y; else nb.z += s.st.z;
    if (nb.x < 0 || nb.y < 0 || nb.z < 0 || nb.x >= G || nb.y >= G || nb.z >= G) return DDA_MISS;
    s.tIn = te;
    s.c = iclamp3(vfloori(((s.o + s.d * te) - s.lo) / s.vs), mki(nb.x * 8, nb.y * 8, nb.z * 8),
                  mki(nb.x * 8 + 7, nb.y * 8 + 7, nb.z * 8 + 7));
    s.tMax = (((vi2f(s.c) + s.sp) * s.vs + s.lo) - s.o) * s.inv;
    return DDA_WALK;
  } else {
    const uint32_t bit = (uint32_t)((s.c.x & 7) + 8 * (s.c.y & 7) + 64 * (s.c.z & 7));
    const uint32_t occ = __ldg(&v.occ[ptr * 16u + (bit >> 5)]);
    const float tExit = mn(mn(s.tMax.x, s.tMax.y), s.tMax.z);
    if ((occ & (1u << (bit & 31u))) != 0u && s.tIn >= s.tskip) { h = make_uint3(ptr, bit, s.L); return DDA_HIT; }
    if (tExit >= s.tEnd) return DDA_MISS;
    s.tIn = tExit;
  }
  if (s.tMax.x <= s.tMax.y && s.tMax.x <= s.tMax.z) { s.c.x += s.st.x; s.tMax.x += s.tDelta.x; }
  else if (s.tMax.y <= s.tMax.z) { s.c.y += s.st.y; s.tMax.y += s.tDelta.y; }
  else { s.c.z += s.st.z; s.tMax.z += s.tDelta.z; }
  if (s.c.x < 0 || s.c.y < 0 || s.c.z < 0 || s.c.x >= nVox || s.c.y >= nVox || s.c.z >= nVox) return DDA_MISS;
  return DDA_WALK;
}

// The shading point of a hit: the voxel's centre and size (for a dropped brick, the coarser voxel that holds the cell)
__device__ __forceinline__ void dda_hit_voxel(const VoxDev &v, const Dda &s, int kind, uint32_t hl, f3 &pc, float &vsz) {
  if (kind == DDA_HIT) {
    pc = s.lo + adds(vi2f(s.c), 0.5f) * s.vs;
    vsz = s.vs;
  } else {
    vsz = vox_size(v, hl);
    const f3 pcl = s.lo + adds(vi2f(s.c), 0.5f) * s.vs;
    pc = adds(vfloor(pcl / vsz), 0.5f) * vsz;
  }
}

// traceVox (voxel.ts:121-202) with a configurable step cap: the walk, then the hit's voxShade
template <class BS>
__device__ __forceinline__ void trace_vox(const VoxDev &v, const float *__restrict__ F, const float *__restrict__ unorm8,
                                          f3 o, f3 d, float t0, float t1,
                                          float tskip, uint32_t L, uint32_t cap, TraceOut &out, const BS &bs,
                                          const float4 *inv_pre = nullptr) {
  out.rad = mk(0.0f, 0.0f, 0.0f); out.T = 1.0f; out.lvl = GI_EMPTY; out.ptr = GI_EMPTY; out.bit = 0; out.tin = 0;
  out.steps = 0;
  Dda s;
  if (!dda_begin(v, o, d, t0, t1, tskip, L, inv_pre, s)) return;
  uint3 h = make_uint3(0u, 0u, 0u);
  int k;
  while ((k = dda_step(v, s, cap, h)) == DDA_WALK) {}
  out.steps = s.steps;
  if (k == DDA_MISS) return;
  f3 pc;
  float vsz;
  dda_hit_voxel(v, s, k, h.z, pc, vsz);
  out.rad = shade_voxel(v, F, unorm8, h.x, h.y, s.d, s.o + s.d * s.tIn, pc, vsz, bs); out.T = 0.0f;
  out.lvl = h.z; out.ptr = h.x; out.bit = h.y; out.tin = __float_as_uint(s.tIn);
}

// ---- the dynamic layer's read (dynlayer.ts:71-162) ------------------------------------------------------------------
// dynFind: the data base of the voxel at p of level L, or of the first coarser level whose brick was not dropped;
// 0xffffffff when empty.  lvl: the level read.
__device__ __forceinline__ uint32_t dyn_find(const RcDev &r, const VoxDev &v, uint32_t L, f3 p, uint32_t &lvl) {
  const int G = (int)v.G;
  const uint32_t ug = v.G, nl = v.levels;
  uint32_t l = L;
  for (;;) {
    const float vs = vox_size(v, l);
    const i3 c = vfloori((p - mk(v.box_lo[l][0], v.box_lo[l][1], v.box_lo[l][2])) / vs);
    lvl = l;
    if (c.x < 0 || c.y < 0 || c.z < 0 || c.x >= G * 8 || c.y >= G * 8 || c.z >= G * 8) return 0xffffffffu;
    const uint32_t ptr = __ldg(&r.dyn_ptr[l * ug * ug * ug + ((uint32_t)(c.z >> 3) * ug + (uint32_t)(c.y >> 3)) * ug
                                           + (uint32_t)(c.x >> 3)]);
    if (ptr == DYN_DROPPED && l + 1u < nl) { l++; continue; }
    if (ptr >= r.dyn_nb) return 0xffffffffu;
    return (ptr * 512u + (uint32_t)((c.x & 7) + 8 * (c.y & 7) + 64 * (c.z & 7))) * DYN_W;
  }
}
// dynWord: level 0 in fixed point, the levels above as resolved f32
__device__ __forceinline__ float dyn_word(const RcDev &r, uint32_t base, uint32_t k, uint32_t L) {
  const uint32_t u = __ldg(&r.dyn_data[base + k]);
  return L == 0u ? (float)u / 65536.0f : __uint_as_float(u);
}
// dynRead: mean radiance and coverage per voxel length for direction d (the three faces against d)
__device__ __forceinline__ float4 dyn_read(const RcDev &r, uint32_t base, uint32_t L, f3 d) {
  if (base == 0xffffffffu) return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  const float a = dyn_word(r, base, 6u, L);
  if (a <= 0.0f) return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  const f3 ad = vabs(d);
  const uint32_t sx = d.x > 0.0f ? 1u : 0u, sy = d.y > 0.0f ? 1u : 0u, sz = d.z > 0.0f ? 1u : 0u;
  const float front = ad.x * dyn_word(r, base, sx, L) + ad.y * dyn_word(r, base, 2u + sy, L) + ad.z * dyn_word(r, base, 4u + sz, L);
  return make_float4(dyn_word(r, base, 7u, L) / a, dyn_word(r, base, 8u, L) / a, dyn_word(r, base, 9u, L) / a, mn(front, 1.0f));
}
// traceDyn: covered radiance and coverage of [t0, t1] along d from o for a cone of width k t, read at the two levels
// around the cone width and interpolated between them
__device__ __forceinline__ float4 trace_dyn(const RcDev &r, const VoxDev &v, f3 o, f3 d, float t0, float t1, float k) {
  const uint32_t *h = r.dyn_hdr;
  if (h[0] == 0u || t1 <= t0) return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  const f3 bmin = adds(mk((float)h[2], (float)h[3], (float)h[4]), -1073741824.0f) * 0.01f;
  const f3 bmax = adds(mk((float)h[5], (float)h[6], (float)h[7]), -1073741824.0f) * 0.01f;
  const f3 dd = mk(fabsf(d.x) < 1e-9f ? 1e-9f : d.x, fabsf(d.y) < 1e-9f ? 1e-9f : d.y, fabsf(d.z) < 1e-9f ? 1e-9f : d.z);
  const f3 qa = bmin - o, qb = bmax - o;
  const f3 ta = mk(qa.x / dd.x, qa.y / dd.y, qa.z / dd.z), tb = mk(qb.x / dd.x, qb.y / dd.y, qb.z / dd.z);
  const f3 tn = vmin(ta, tb), tf = vmax(ta, tb);
  const float ba = mx(mx(mx(tn.x, tn.y), tn.z), t0);
  const float bb = mn(mn(mn(tf.x, tf.y), tf.z), t1);
  if (ba >= bb) return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  const float v0 = v.v0;
  const uint32_t nl = v.levels;
  f3 rad = mk(0.0f, 0.0f, 0.0f);
  float cov = 0.0f, t = t0;
  for (uint32_t i = 0; i < 128u; i++) {
    if (t >= bb || cov >= 1.0f) break;
    const float w = mx(k * t, v0);
    const float te = mn(t + 0.5f * w, t1);
    if (te > ba) {
      const float len = te - t;
      const f3 p = o + d * (0.5f * (t + te));
      const float lf = fclampf(gi_log2(w / v0), 0.0f, (float)(nl - 1u));
      uint32_t L0 = (uint32_t)floorf(lf);
      float f = lf - (float)L0;
      const uint32_t Lw = vox_level_for(v, L0, p);
      if (Lw != L0) { L0 = Lw; f = 0.0f; }
      uint32_t la, lb;
      const float4 sa = dyn_read(r, dyn_find(r, v, L0, p, la), la, d);
      float aa = sa.w * len / vox_size(v, la);
      f3 ra = mk(sa.x, sa.y, sa.z) * aa;
      if (f > 0.0f && L0 + 1u < nl) {
        const float4 sb = dyn_read(r, dyn_find(r, v, L0 + 1u, p, lb), lb, d);
        const float ab = sb.w * len / vox_size(v, lb);
        const f3 rb = mk(sb.x, sb.y, sb.z) * ab;
        ra = ra * (1.0f - f) + rb * f;   // mix(ra, rb, f)
        aa = aa * (1.0f - f) + ab * f;
      }
      if (aa > 0.0f) {
        const float a = mn(aa, 1.0f - cov);
        rad = rad + ra * (a / aa);
        cov += a;
      }
    }
    t = te;
  }
  return make_float4(rad.x, rad.y, rad.z, cov);
}
// traceWorld's read of the dynamic layer (rc.ts:223-231): in front of the static hit (or to t1 on a miss), from at
// least one level-0 voxel out, composited over the voxel trace's result.  o: the probe; ooff: the trace's start (o moved
// along the probe normal); k: the cone width per unit distance (3.5449077 / res).
__device__ __forceinline__ void dyn_compose(const RcDev &r, const VoxDev &v, f3 o, f3 d, float t0, float t1, f3 ooff, float k,
                                            TraceOut &out) {
  if (!r.dyn_hdr || __ldg(&r.dyn_hdr[0]) == 0u) return;
  float tS = t1;
  if (out.T < 0.5f) tS = dot((ooff + d * __uint_as_float(out.tin)) - o, d);
  const float4 dl = trace_dyn(r, v, o, d, mx(t0, v.v0), mn(t1, tS), k);
  if (dl.w > 0.0f) {
    const float s = 1.0f - dl.w;
    out.rad = mk(dl.x + s * out.rad.x, dl.y + s * out.rad.y, dl.z + s * out.rad.z);
    out.T = s * out.T;
  }
}

// voxLevel (rc.ts:210-213), round(log2) taken exactly
__device__ __forceinline__ uint32_t vox_level(const VoxDev &v, const RcDev &r, float s0, uint32_t c) {
  float vv = r.vox_scale * s0 * exp2_(r.level_map * (float)c);
  int k = round_log2(vv / v.v0);
  int top = (int)v.levels - 1;
  return (uint32_t)(k < 0 ? 0 : (k > top ? top : k));
}

__device__ __forceinline__ uint32_t casc_of_ray(const RcDev &r, uint32_t i) {
  uint32_t c = 0;
#pragma unroll
  for (uint32_t k = 1; k < 8; k++) if (k < r.cascades && i >= r.c[k].ray_off) c = k;
  return c;
}

// setupScreen (rc.ts:572-590) of probe i (all cascades numbered together)
__device__ __forceinline__ void setup_probe(const RcDev &r, const VoxDev &v, uint32_t i) {
  uint32_t c = 0;
  for (uint32_t k = 1; k < r.cascades; k++) if (i >= r.c[k].probe_off) c = k;
  const CascDev &L = r.c[c];
  uint32_t t = i - L.probe_off;
  if (t == 0) r.counts[c] = L.tiles_x * L.tiles_y;
  const float *F = r.frame;
  uint32_t tx = t % L.tiles_x, ty = t / L.tiles_x;
  int px = min((int)(tx * L.tile_size + L.tile_size / 2u), (int)r.width - 1);
  int py = min((int)(ty * L.tile_size + L.tile_size / 2u), (int)r.height - 1);
  size_t q = (size_t)py * r.width + (size_t)px;
  float d = r.depth[q];
  ProbeDev pr;
  pr.pos = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  pr.nrm = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  pr.grid = make_int4((int)tx, (int)ty, 0, 0);
  if (d > 0.0f) {
    f3 x = world_at(F, px, py, d);
    uint2 nn = r.normal[q];
    f3 nrm = mk(h2f(nn.x & 0xffffu), h2f(nn.x >> 16), h2f(nn.y & 0xffffu));
    float s0 = length3(x - mk(F[F_EYE], F[F_EYE + 1], F[F_EYE + 2])) * F[F_RC + 1] * F[F_RC + 2];
    f3 p = x + ((nrm * F[F_RC2]) * s0) * exp2_((float)c);
    pr.pos = make_float4(p.x, p.y, p.z, s0);
    pr.nrm = make_float4(nrm.x, nrm.y, nrm.z, view_z(F, x));
  }
  r.probes[i] = pr;
  r.plevel[i] = pr.pos.w > 0.0f ? vox_level(v, r, pr.pos.w, c) : 0u;
}

constexpr uint32_t RS_KEYS = 128, RS_PER_BLOCK = 1024;   // walk-length order: keys, rays per scatter block

// every cascade in one launch
__global__ void k_setup_screen(RcDev r, VoxDev v) {
  grid_dep_wait();
  // the 80 counter words and the trace's ray counter start at zero (words below `cascades` are set by the probes);
  // the walk-length order's key counts and cursors too
  if (blockIdx.x == 0 && threadIdx.x < 81u && threadIdx.x >= r.cascades) r.counts[threadIdx.x] = 0u;
  if (blockIdx.x == 0 && r.rhist && threadIdx.x < 2u * RS_KEYS) r.rhist[threadIdx.x] = 0u;
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < r.probes_total) setup_probe(r, v, i);
}

// The direction a probe's k-th ray takes in the probe-major orders: 32 consecutive rays (a warp) take an 8 x 4 tile of
// the probe's direction map, tiles row by row (res >= 16; a smaller map is one or two warps as it is).  Neighbouring
// directions walk alike, so a warp's lanes idle less than on 32 directions of a row.  A bijection of [0, res^2).
__device__ __forceinline__ uint32_t dir_tile(const CascDev &L, uint32_t k) {
  if (L.res < 16u) return k;
  const uint32_t w = k & 31u, tt = k >> 5, tl = L.dirs_log2 / 2u - 3u;   // res / 8 = 2^tl tiles per row
  return (((tt >> tl) << 2) + (w >> 3)) * L.res + ((tt & ((1u << tl) - 1u)) << 3) + (w & 7u);
}

// trace (rc.ts:600-622) -> traceWorld (rc.ts:216-245) of the ray at position j of the trace order (cascade c): writes
// its atlas element (and the debug copies); true when its probe is valid and the ray was marched.
template <int A, bool DYN = false>
__device__ __forceinline__ bool trace_ray(const RcDev &r, const VoxDev &v, uint32_t j, uint32_t c, TraceOut &out,
                                          bool probe_major) {
  typedef typename Atlas<A>::T T;
  T *rad = reinterpret_cast<T *>(r.rad);
  const float *F = r.frame;
  out.rad = mk(0.0f, 0.0f, 0.0f); out.T = 1.0f; out.lvl = GI_EMPTY; out.ptr = GI_EMPTY; out.bit = 0; out.tin = 0;
  out.steps = 0;
  bool traced = false;
  const CascDev &L = r.c[c];
  uint32_t t = j - L.ray_off, pi, di;
  if (probe_major) {                  // probe-major: a probe's rays together; a warp's on neighbouring directions
    pi = t >> L.dirs_log2;
    di = t & ((1u << L.dirs_log2) - 1u);
    di = dir_tile(L, di);
  } else {                            // direction-major: one direction over consecutive probes
    di = t / L.np;
    pi = t - di * L.np;
  }
  uint32_t i = L.ray_off + (pi << L.dirs_log2) + di;   // the ray's atlas element
  ProbeDev pr = r.probes[L.probe_off + pi];
  if (pr.pos.w > 0.0f) {
    float4 dv = r.dirs[L.dir_off + di];   // dirOf(di, res), tabulated
    f3 dir = mk(dv.x, dv.y, dv.z);
    float s0 = pr.pos.w;
    float t0 = L.b0 * s0, t1 = L.b1 * s0;
    f3 po = ld3(pr.pos), pn = ld3(pr.nrm);
    uint32_t Lv = vox_level_for(v, r.plevel[L.probe_off + pi], po + dir * t1);
    float vs = vox_size(v, Lv);
    const f3 ooff = po + pn * (r.vox_offset * vs);
    trace_vox(v, F, r.unorm8, ooff, dir, t0, t1, r.vox_skip * vs, Lv, r.dda_cap, out, InjectedBounce{r.bn_inj},
              r.idirs + L.dir_off + di);
    if (DYN) dyn_compose(r, v, po, dir, t0, t1, ooff, 3.5449077f / (float)L.res, out);
    traced = true;
  }
  Atlas<A>::store(rad, i, make_float4(out.rad.x, out.rad.y, out.rad.z, out.T));
  if (r.hits) r.hits[i] = make_uint4(out.lvl, out.ptr, out.bit, out.tin);
  if (r.rad_traced) Atlas<A>::store(reinterpret_cast<T *>(r.rad_traced), i, make_float4(out.rad.x, out.rad.y, out.rad.z, out.T));
  return traced;
}

// Walk-length order (trace_order 2, screen probes): the rays are handed out by the previous solve's DDA step count and
// hit, longest walks first, so a warp's lanes walk about as long as each other and the persistent queue ends on short
// rays.  Each ray's result does not depend on which lane traces it or when.  A ray's key: its step count (exact below
// 48, then in 16-step groups up to 63) x 2 + hit; k_trace stores it per atlas element, the next solve counts the keys
// (k_rsort_hist) and scatters the atlas indices by key (k_rsort_scatter) before its trace.
__device__ __forceinline__ uint32_t rsort_key(uint32_t steps, bool hit) {
  const uint32_t s = steps < 48u ? steps : min(48u + ((steps - 48u) >> 4), 63u);
  return s * 2u + (hit ? 1u : 0u);
}

// per-key ray counts of the stored keys (rhist[0 .. 127], zeroed by the setup with the cursors after them)
__global__ void __launch_bounds__(256) k_rsort_hist(RcDev r) {
  grid_dep_wait();
  __shared__ uint32_t h[RS_KEYS];
  if (threadIdx.x < RS_KEYS) h[threadIdx.x] = 0u;
  __syncthreads();
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < r.rays_total; i += gridDim.x * blockDim.x)
    atomicAdd(&h[r.rsteps[i]], 1u);
  __syncthreads();
  if (threadIdx.x < RS_KEYS && h[threadIdx.x]) atomicAdd(&r.rhist[threadIdx.x], h[threadIdx.x]);
}

// the trace order: atlas indices by descending key; a block ranks its 1024 rays per key in shared memory and reserves
// each key's range with one atomic (the order inside a key is whatever the blocks' reservations give)
__global__ void __launch_bounds__(256) k_rsort_scatter(RcDev r) {
  grid_dep_wait();
  __shared__ uint32_t cnt[RS_KEYS], start[RS_KEYS], base[RS_KEYS];
  if (threadIdx.x < RS_KEYS) { cnt[threadIdx.x] = 0u; start[threadIdx.x] = r.rhist[threadIdx.x]; }
  __syncthreads();
  if (threadIdx.x == 0) {   // rays with larger keys come first
    uint32_t a = 0;
    for (int k = (int)RS_KEYS - 1; k >= 0; k--) { const uint32_t n = start[k]; start[k] = a; a += n; }
  }
  const uint32_t b0 = blockIdx.x * RS_PER_BLOCK;
  uint32_t key[4], rank[4];
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const uint32_t i = b0 + (uint32_t)k * 256u + threadIdx.x;
    key[k] = i < r.rays_total ? (uint32_t)r.rsteps[i] : RS_KEYS;
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < 4; k++) rank[k] = key[k] < RS_KEYS ? atomicAdd(&cnt[key[k]], 1u) : 0u;
  __syncthreads();
  if (threadIdx.x < RS_KEYS && cnt[threadIdx.x])
    base[threadIdx.x] = start[threadIdx.x] + atomicAdd(&r.rhist[RS_KEYS + threadIdx.x], cnt[threadIdx.x]);
  __syncthreads();
#pragma unroll
  for (int k = 0; k < 4; k++) {
    if (key[k] >= RS_KEYS) continue;
    const uint32_t pos = base[key[k]] + rank[k];
    if (pos < r.rays_total) r.rperm[pos] = b0 + (uint32_t)k * 256u + threadIdx.x;
  }
}

// Persistent: every warp takes rays from a global counter, 32 x trace_rays at a time, the top cascade's first (its
// walks are the longest; a queue that ended on them left SMs idle behind its last warps: 0.197 -> 0.170 ms on the
// colonnade).  SORT: positions go through the walk-length order (rperm) and each ray's key is stored for the next
// solve.
template <int A, bool DYN, bool SORT>
__global__ void __launch_bounds__(256) k_trace(RcDev r, VoxDev v, uint32_t *ray_counter) {
  grid_dep_wait();
  uint32_t lane = threadIdx.x & 31u;
  uint32_t steps_acc = 0, traces_acc = 0, cap_acc = 0;
  uint32_t cur_c = 0xffffffffu;
  const uint32_t per = 32u * r.trace_rays;
  for (;;) {
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(ray_counter, per);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= r.rays_total) break;
   for (uint32_t k = 0; k < r.trace_rays; k++) {
    uint32_t j = base + k * 32u + lane;   // position in the trace order
    bool live = j < r.rays_total;
    if (SORT && live) j = r.rperm[j];     // the atlas element at that position
    else if (live) j = r.rays_total - 1u - j;   // the top cascade first: the queue ends on the shortest walks
    uint32_t c = live ? casc_of_ray(r, j) : 0u;
    TraceOut out;
    out.steps = 0;
    bool traced = live && trace_ray<A, DYN>(r, v, j, c, out, SORT || r.trace_order == 0u);
    if (SORT && live) r.rsteps[j] = (uint8_t)rsort_key(traced ? out.steps : 0u, traced && out.T < 0.5f);
    if (r.stats) {
      // per-cascade counters (rc.ts:232-235); flush when the lane's cascade changes
      if (live && traced) {
        if (c != cur_c && cur_c != 0xffffffffu) {
          atomicAdd(&r.counts[24 + cur_c], traces_acc); atomicAdd(&r.counts[32 + cur_c], steps_acc);
          atomicAdd(&r.counts[64 + cur_c], cap_acc);
          traces_acc = steps_acc = cap_acc = 0;
        }
        cur_c = c;
        traces_acc++; steps_acc += out.steps; cap_acc += out.steps >= r.dda_cap ? 1u : 0u;
      }
    }
   }
  }
  if (r.stats) {   // the warp leaves the loop together: one atomic per cascade the warp's lanes hold
    const unsigned grp = __match_any_sync(0xffffffffu, cur_c);
    const uint32_t tr = __reduce_add_sync(grp, traces_acc), sp = __reduce_add_sync(grp, steps_acc);
    const uint32_t cp = __reduce_add_sync(grp, cap_acc);
    if (cur_c != 0xffffffffu && (uint32_t)(__ffs(grp) - 1) == lane) {
      atomicAdd(&r.counts[24 + cur_c], tr); atomicAdd(&r.counts[32 + cur_c], sp); atomicAdd(&r.counts[64 + cur_c], cp);
    }
  }
}

__device__ __forceinline__ void sh_basis(f3 n, float y[9]) {
  y[0] = 0.282095f; y[1] = 0.488603f * n.y; y[2] = 0.488603f * n.z; y[3] = 0.488603f * n.x;
  y[4] = 1.092548f * n.x * n.y; y[5] = 1.092548f * n.y * n.z; y[6] = 0.315392f * (3.0f * n.z * n.z - 1.0f);
  y[7] = 1.092548f * n.x * n.z; y[8] = 0.546274f * (n.x * n.x - n.y * n.y);
}

// projectSH (rc.ts:752-774) of cascade-0 probe pi, fused into its merge: the probe's 16 directions (res 4) are held by
// its four quad threads, four consecutive lanes, 4 merged radiances each (as stored).  Every lane of the group collects
// the 16 with shuffles and sums the 27 coefficients over the directions in order 0..15, with fused multiply-adds; lane
// i of the group stores the probe's coefficient groups 2i and 2i+1.
template <int A>
__device__ __forceinline__ void project_sh_quads(const RcDev &r, uint32_t pi, const f3 mr[4]) {
  const uint32_t lane = threadIdx.x & 31u, gbase = lane & ~3u;
  const unsigned gmask = 0xFu << gbase;
  const float *F = r.frame;
  f3 cf[9];
#pragma unroll
  for (int k = 0; k < 9; k++) cf[k] = mk(0.0f, 0.0f, 0.0f);
#pragma unroll
  for (uint32_t d = 0; d < 16u; d++) {
    const uint32_t u = d & 3u, vr = d >> 2, j = (vr & 1u) * 2u + (u & 1u);
    const int src = (int)(gbase + (vr >> 1) * 2u + (u >> 1));
    f3 rd = mk(__shfl_sync(gmask, mr[j].x, src), __shfl_sync(gmask, mr[j].y, src), __shfl_sync(gmask, mr[j].z, src));
    f3 rr = rd * F[F_OMEGA + d];
    float4 dv = r.dirs[r.c[0].dir_off + d];   // dirOf(d, 4), tabulated
    float y[9];
    sh_basis(mk(dv.x, dv.y, dv.z), y);
#pragma unroll
    for (int k = 0; k < 9; k++) cf[k] = fma3(rr, y[k], cf[k]);
  }
  float vals[32];
#pragma unroll
  for (int k = 0; k < 32; k++) vals[k] = 0.0f;
  const float a0 = GI_PI, a1 = 2.0f * GI_PI / 3.0f, a2 = GI_PI / 4.0f;
#pragma unroll
  for (int k = 0; k < 9; k++) {
    float a = k == 0 ? a0 : (k < 4 ? a1 : a2);
    vals[k * 3 + 0] = cf[k].x * a; vals[k * 3 + 1] = cf[k].y * a; vals[k * 3 + 2] = cf[k].z * a;
  }
  typedef typename Atlas<A>::T T;
#pragma unroll
  for (uint32_t q = 0; q < 8u; q++) {
    if ((q >> 1) != (lane & 3u)) continue;
    float4 val = make_float4(vals[4 * q], vals[4 * q + 1], vals[4 * q + 2], vals[4 * q + 3]);
    if (r.f32_out) reinterpret_cast<float4 *>(r.sh)[(size_t)pi * 8u + q] = val;
    else Atlas<A>::store(reinterpret_cast<T *>(r.sh), (size_t)pi * 8u + q, val);
  }
}

// mergeScreen (rc.ts:710-743) for cascade c, in place, one 2x2 quad of directions (four rays) per thread.  The four
// upper probes and their weights depend only on the probe, so a thread computes them once for its four rays.
// upperAvg (rc.ts:681-686) of the upper cascade comes from up_avg, the quad averages the upper cascade's merge wrote
// from its stored (rounded) texels: the same four values summed in the same order, so the same bits.  When this
// cascade's resolution is twice the lower one's, the thread writes its own quad's average for the merge below.
template <int A>
__device__ __forceinline__ void merge_quad(const RcDev &r, uint32_t c, uint32_t t, const float4 *__restrict__ up_avg,
                                           float4 *__restrict__ my_avg) {
  typedef typename Atlas<A>::T T;
  T *rad = reinterpret_cast<T *>(r.rad);
  const CascDev &L = r.c[c];
  uint32_t hr = L.res >> 1, hq_log2 = L.dirs_log2 - 2u;   // quads per row, log2 quads per probe
  if (t >= (L.np << hq_log2)) return;
  uint32_t pi = t >> hq_log2, qd = t & ((1u << hq_log2) - 1u);
  uint32_t u0 = (qd % hr) * 2u, v0 = (qd / hr) * 2u;
  const float *F = r.frame;
  const bool has_up = c + 1u < r.cascades;
  bool pr_ok = false;
  float w[4];
  uint32_t qi[4];
  bool qok[4];
  if (has_up) {
    ProbeDev pr = r.probes[L.probe_off + pi];
    pr_ok = pr.pos.w > 0.0f;
    if (pr_ok) {
      const CascDev &U = r.c[c + 1u];
      float cx = ((float)(pi % L.tiles_x) + 0.5f) * (float)L.tile_size;
      float cy = ((float)(pi / L.tiles_x) + 0.5f) * (float)L.tile_size;
      float ux = div_tile(cx, U) - 0.5f, uy = div_tile(cy, U) - 0.5f;
      int bx = __float2int_rd(ux), by = __float2int_rd(uy);
      float fx = ux - (float)bx, fy = uy - (float)by;
#pragma unroll
      for (uint32_t k = 0; k < 4; k++) {
        int ox = (int)(k & 1u), oy = (int)(k >> 1);
        int qx = iclamp(bx + ox, 0, (int)U.tiles_x - 1), qy = iclamp(by + oy, 0, (int)U.tiles_y - 1);
        qi[k] = (uint32_t)qy * U.tiles_x + (uint32_t)qx;
        ProbeDev qp = r.probes[U.probe_off + qi[k]];
        qok[k] = qp.pos.w > 0.0f;
        float fwx = ox == 1 ? fx : 1.0f - fx, fwy = oy == 1 ? fy : 1.0f - fy;
        float rel = fabsf(qp.nrm.w - pr.nrm.w) / pr.nrm.w;
        w[k] = (fwx * fwy + 1e-4f) * (gi_exp(-20.0f * rel) + 1e-4f);
      }
    }
  }
  f3 qsum = mk(0.0f, 0.0f, 0.0f);
  f3 mr[4];   // the four merged radiances as stored (rounded to the atlas)
#pragma unroll
  for (uint32_t j = 0; j < 4; j++) {   // (0,0) (1,0) (0,1) (1,1): upperAvg's a, b, c, d order
    uint32_t u = u0 + (j & 1u), v = v0 + (j >> 1);
    size_t idx = (size_t)L.rad_off + ((size_t)pi << L.dirs_log2) + v * L.res + u;
    float4 vv = Atlas<A>::load(rad, idx);
    f3 up = mk(F[F_SKY], F[F_SKY + 1], F[F_SKY + 2]);
    if (has_up && vv.w > 0.0f) {
      up = mk(0.0f, 0.0f, 0.0f);
      if (pr_ok) {
        const CascDev &U = r.c[c + 1u];
        f3 acc = mk(0.0f, 0.0f, 0.0f);
        float ws = 0.0f;
#pragma unroll
        for (uint32_t k = 0; k < 4; k++) {
          if (!qok[k]) continue;
          f3 ua;
          if (U.res == L.res) {
            float4 p = Atlas<A>::load(rad, (size_t)U.rad_off + ((size_t)qi[k] << U.dirs_log2) + v * U.res + u);
            ua = mk(p.x, p.y, p.z);
          } else {
            float4 p = up_avg[((size_t)qi[k] << L.dirs_log2) + v * L.res + u];
            ua = mk(p.x, p.y, p.z);
          }
          acc = fma3(ua, w[k], acc);
          ws += w[k];
        }
        if (ws > 0.0f) up = acc / ws;
      }
    }
    f3 m = fma3(up, vv.w, mk(vv.x, vv.y, vv.z));
    Atlas<A>::store(rad, idx, make_float4(m.x, m.y, m.z, 1.0f));
    mr[j] = mk(Atlas<A>::round(m.x), Atlas<A>::round(m.y), Atlas<A>::round(m.z));
    if (my_avg) qsum = qsum + mr[j];
  }
  if (my_avg) {
    f3 a = qsum * 0.25f;
    my_avg[((size_t)pi << hq_log2) + (v0 >> 1) * hr + (u0 >> 1)] = make_float4(a.x, a.y, a.z, 0.0f);
  }
  if (c == 0u) project_sh_quads<A>(r, pi, mr);
}

template <int A>
__global__ void __launch_bounds__(512) k_merge(RcDev r, uint32_t c, const float4 *__restrict__ up_avg,
                                               float4 *__restrict__ my_avg) {
  grid_dep_wait();
  merge_quad<A>(r, c, blockIdx.x * blockDim.x + threadIdx.x, up_avg, my_avg);
}


// SH element i as f32: stored as f32 with f32_out, else in the atlas format
template <int A>
__device__ __forceinline__ float4 sh_load(const RcDev &r, size_t i) {
  if (r.f32_out) return reinterpret_cast<const float4 *>(r.sh)[i];
  return Atlas<A>::load(reinterpret_cast<const typename Atlas<A>::T *>(r.sh), i);
}

// gatherScreen (rc.ts:929-954), evalSH (rc.ts:819-829) for one pixel.  Src supplies the 2x2 cascade-0 probes around
// the pixel: probe(k, qi) and coef(k, qi, j), the j-th 4-component group of its SH as f32.
template <int A, class Src>
__device__ __forceinline__ void gather_pixel(const RcDev &r, uint32_t px, uint32_t py, const Src &src) {
  size_t q = (size_t)py * r.width + px;
  const float *F = r.frame;
  float d = r.depth[q];
  f3 res = mk(0.0f, 0.0f, 0.0f);
  float alpha = 0.0f;
  if (d > 0.0f) {
    alpha = 1.0f;
    const CascDev &L = r.c[0];
    f3 x = world_at(F, (int)px, (int)py, d);
    uint2 nn = r.normal[q];
    f3 n = mk(h2f(nn.x & 0xffffu), h2f(nn.x >> 16), h2f(nn.y & 0xffffu));
    float z = view_z(F, x);
    float ux = div_tile((float)px + 0.5f, L) - 0.5f, uy = div_tile((float)py + 0.5f, L) - 0.5f;
    int bx = __float2int_rd(ux), by = __float2int_rd(uy);
    float fx = ux - (float)bx, fy = uy - (float)by;
    float y[9];
    sh_basis(n, y);
    f3 e = mk(0.0f, 0.0f, 0.0f);
    float ws = 0.0f;
#pragma unroll
    for (uint32_t k = 0; k < 4; k++) {
      int ox = (int)(k & 1u), oy = (int)(k >> 1);
      int qx = iclamp(bx + ox, 0, (int)L.tiles_x - 1), qy = iclamp(by + oy, 0, (int)L.tiles_y - 1);
      uint32_t qi = (uint32_t)qy * L.tiles_x + (uint32_t)qx;
      ProbeDev pr = src.probe(k, qi);
      if (pr.pos.w <= 0.0f) continue;
      float fwx = ox == 1 ? fx : 1.0f - fx, fwy = oy == 1 ? fy : 1.0f - fy;
      float rel = fabsf(pr.nrm.w - z) / z;
      float nd = mx(dot(n, ld3(pr.nrm)), 0.0f);
      float w = (fwx * fwy + 1e-4f) * (gi_exp(-20.0f * rel) + 1e-4f) * (nd * nd * nd * nd + 1e-3f);
      float v[32];
#pragma unroll
      for (int j = 0; j < 8; j++) {
        float4 sc = src.coef(k, qi, j);
        v[4 * j] = sc.x; v[4 * j + 1] = sc.y; v[4 * j + 2] = sc.z; v[4 * j + 3] = sc.w;
      }
      f3 es = mk(0.0f, 0.0f, 0.0f);
#pragma unroll
      for (int k2 = 0; k2 < 9; k2++) es = fma3(mk(v[3 * k2], v[3 * k2 + 1], v[3 * k2 + 2]), y[k2], es);
      es = vmax(es, mk(0.0f, 0.0f, 0.0f));
      e = fma3(es, w, e);
      ws += w;
    }
    if (ws > 0.0f) res = e / ws;
  }
  if ((A == GI_ATLAS_F32 || r.f32_out) && !r.irr_f16) reinterpret_cast<float4 *>(r.irr)[q] = make_float4(res.x, res.y, res.z, alpha);
  else reinterpret_cast<uint2 *>(r.irr)[q] = make_uint2((uint32_t)f2h(res.x) | ((uint32_t)f2h(res.y) << 16),
                                                       (uint32_t)f2h(res.z) | ((uint32_t)f2h(alpha) << 16));
}

template <int A>
struct GlobalProbes {   // each lane reads its own probes
  const RcDev &r;
  __device__ __forceinline__ ProbeDev probe(uint32_t, uint32_t qi) const { return r.probes[r.c[0].probe_off + qi]; }
  __device__ __forceinline__ float4 coef(uint32_t, uint32_t qi, int j) const { return sh_load<A>(r, (size_t)qi * 8u + j); }
};

struct SharedProbes {   // the warp's four probes, staged in shared memory (k = the 2x2 corner)
  const float4 *pn;      // [2k] pos, [2k + 1] nrm
  const float4 *coefs;   // [8k + j]
  __device__ __forceinline__ ProbeDev probe(uint32_t k, uint32_t) const {
    ProbeDev p;
    p.pos = pn[2u * k];
    p.nrm = pn[2u * k + 1u];
    p.grid = make_int4(0, 0, 0, 0);
    return p;
  }
  __device__ __forceinline__ float4 coef(uint32_t k, uint32_t, int j) const { return coefs[8u * k + (uint32_t)j]; }
};

// One thread per pixel, BX x (256 / BX) pixels per block
template <int A, uint32_t BX>
__global__ void __launch_bounds__(256) k_gather(RcDev r) {
  grid_dep_wait();
  uint32_t px = blockIdx.x * BX + threadIdx.x % BX, py = blockIdx.y * (256u / BX) + threadIdx.x / BX;
  if (px >= r.width || py >= r.height) return;
  gather_pixel<A>(r, px, py, GlobalProbes<A>{r});
}

// Warp tiles of P x (32 / P) pixels aligned to the cascade-0 probe cells (P = the tile size): every pixel of a tile
// interpolates the same four probes, so the warp loads their records and SH once into shared memory (one 128-bit load
// per lane) and the pixels read them as broadcasts.  A warp whose pixels turn out not to share their probes (they
// always do for these P; the check keeps it exact regardless) reads them per lane.  Blocks of 2 x 4 warp tiles.
template <int A, uint32_t P>
__device__ __forceinline__ void gather_tiles(const RcDev &r, uint32_t blk_x, uint32_t blk_y) {
  constexpr uint32_t TH = 32u / P;
  __shared__ float4 s_coef[8][32];
  __shared__ float4 s_pn[8][8];
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  const int tx = (int)(blk_x * 2u + (warp & 1u)), ty = (int)(blk_y * 4u + (warp >> 1));
  const int px = tx * (int)P - (int)(P / 2u) + (int)(lane % P), py = ty * (int)TH - (int)(P / 2u) + (int)(lane / P);
  const bool on = px >= 0 && py >= 0 && px < (int)r.width && py < (int)r.height;
  const unsigned on_mask = __ballot_sync(0xffffffffu, on);
  if (on_mask == 0u) return;   // whole warp off the screen
  const CascDev &L = r.c[0];
  int bx = __float2int_rd(div_tile((float)px + 0.5f, L) - 0.5f), by = __float2int_rd(div_tile((float)py + 0.5f, L) - 0.5f);
  const int src_lane = __ffs(on_mask) - 1;
  const int bx0 = __shfl_sync(0xffffffffu, bx, src_lane), by0 = __shfl_sync(0xffffffffu, by, src_lane);
  if (!__all_sync(0xffffffffu, !on || (bx == bx0 && by == by0))) {
    if (on) gather_pixel<A>(r, (uint32_t)px, (uint32_t)py, GlobalProbes<A>{r});
    return;
  }
  {
    uint32_t k = lane >> 3, j = lane & 7u;
    int qx = iclamp(bx0 + (int)(k & 1u), 0, (int)L.tiles_x - 1), qy = iclamp(by0 + (int)(k >> 1), 0, (int)L.tiles_y - 1);
    uint32_t qi = (uint32_t)qy * L.tiles_x + (uint32_t)qx;
    s_coef[warp][lane] = sh_load<A>(r, (size_t)qi * 8u + j);
    if (lane < 8u) {
      uint32_t kk = lane >> 1;
      int qx2 = iclamp(bx0 + (int)(kk & 1u), 0, (int)L.tiles_x - 1), qy2 = iclamp(by0 + (int)(kk >> 1), 0, (int)L.tiles_y - 1);
      const ProbeDev &pr = r.probes[L.probe_off + (uint32_t)qy2 * L.tiles_x + (uint32_t)qx2];
      s_pn[warp][lane] = (lane & 1u) ? pr.nrm : pr.pos;
    }
  }
  __syncwarp();
  if (on) gather_pixel<A>(r, (uint32_t)px, (uint32_t)py, SharedProbes{s_pn[warp], s_coef[warp]});
}

template <int A, uint32_t P>
__global__ void __launch_bounds__(256) k_gather_tiled(RcDev r) {
  grid_dep_wait();
  gather_tiles<A, P>(r, blockIdx.x, blockIdx.y);
}

// ---- the multi-bounce volume (bounce.ts): clear, classify, update, inject ------------------------------------------
constexpr uint32_t BN_DDA_CAP = 1024;   // traceVox's step cap (voxel.ts:142) for the volume's rays

__device__ __forceinline__ uint2 bn_pack(float4 x) {
  return make_uint2((uint32_t)f2h(x.x) | ((uint32_t)f2h(x.y) << 16), (uint32_t)f2h(x.z) | ((uint32_t)f2h(x.w) << 16));
}
__device__ __forceinline__ size_t bn_index(const BounceDev &b, i3 c, int a) {
  return ((size_t)(a * (int)b.dz + c.z) * b.dy + (size_t)c.y) * b.dx + (size_t)c.x;
}
// bnOriginNow (bounce.ts:98): the probe coordinates of this frame's probe 0
__device__ __forceinline__ i3 bn_origin_now(const BounceDev &b, const float *__restrict__ F) {
  return mki(__float2int_rd(F[F_EYE] / b.cell) - (int)(b.dx / 2u), __float2int_rd(F[F_EYE + 1] / b.cell) - (int)(b.dy / 2u),
             __float2int_rd(F[F_EYE + 2] / b.cell) - (int)(b.dz / 2u));
}
// occAt (bounce.ts:99-104)
__device__ __forceinline__ bool bn_occ_at(const VoxDev &v, uint32_t L, f3 p) {
  const float vs = vox_size(v, L);
  const i3 c = vfloori((p - (vi2f(org(v, L)) * vs) * 8.0f) / vs);
  const int n = (int)v.G * 8;
  if (c.x < 0 || c.y < 0 || c.z < 0 || c.x >= n || c.y >= n || c.z >= n) return false;
  return vox_at(v, L, c).x != GI_EMPTY;
}

// bnClear (bounce.ts:107): the list empty, the frame counter on, the volumes swapped
__global__ void k_bn_clear(BounceDev b) {
  grid_dep_wait();
  if (threadIdx.x == 0) { b.list[0] = 0u; b.list[1] += 1u; b.list[2] ^= 1u; }
}

// bnClassify (bounce.ts:112-138): one thread per probe (and one for the origin texel)
__global__ void __launch_bounds__(256) k_bn_classify(BounceDev b, VoxDev v, const float *__restrict__ F) {
  grid_dep_wait();
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t cur = b.list[2];
  uint2 *out = b.vol[cur];
  const uint2 *prev = b.vol[cur ^ 1u];
  const i3 o = bn_origin_now(b, F);
  if (i == b.n) out[bn_index(b, mki(0, 0, 0), 6)] = bn_pack(make_float4((float)o.x, (float)o.y, (float)o.z, 0.0f));
  if (i >= b.n) return;
  const i3 c = mki((int)(i % b.dx), (int)((i / b.dx) % b.dy), (int)(i / (b.dx * b.dy)));
  const f3 p = vi2f(mki(o.x + c.x, o.y + c.y, o.z + c.z)) * b.cell;
  // levelOf(BN_CELL): round(log2(max(size, 1e-4) / v0)) clamped to the levels
  int lr = round_log2(mx(b.cell, 1e-4f) / b.v0);
  const uint32_t L = (uint32_t)(lr < 0 ? 0 : (lr > (int)v.levels - 1 ? (int)v.levels - 1 : lr));
  bool near = false;
  for (uint32_t k = 0; k < 8u && !near; k++)
    near = bn_occ_at(v, L, p + adds(mk((float)(k & 1u), (float)((k >> 1) & 1u), (float)(k >> 2)), -0.5f) * b.cell);
  if (near && !bn_occ_at(v, 0u, p)) {
    // staggered: a probe is traced every div frames (by its world position), kept from the previous volume between
    const i3 w = mki(o.x + c.x, o.y + c.y, o.z + c.z);
    if (b.div > 1u && ((uint32_t)(w.x + w.y + w.z + 1048576) + b.list[1]) % b.div != 0u) {
      const i3 po = bn_origin(b, prev);
      const i3 pc = mki(w.x - po.x, w.y - po.y, w.z - po.z);
      if (pc.x >= 0 && pc.y >= 0 && pc.z >= 0 && pc.x < (int)b.dx && pc.y < (int)b.dy && pc.z < (int)b.dz
          && bn_axis(b, prev, pc, 0).w > 0.0f) {
        for (int a = 0; a < 6; a++) out[bn_index(b, c, a)] = prev[bn_index(b, pc, a)];
        return;
      }
    }
    const uint32_t s = atomicAdd(&b.list[0], 1u);
    b.list[4u + s] = i;
  } else {
    for (int a = 0; a < 6; a++) out[bn_index(b, c, a)] = make_uint2(0u, 0u);
  }
}

// bnTrace (bounce.ts:156-167): the ray in segments [b_k, b_k+1] cells (b_k = (4^k - 1) / 3) on level k's voxels;
// rgb and the distance to the hit (sky and 1e9 past the last level)
__device__ float4 bn_trace(const VoxDev &v, const float *__restrict__ F, const float *__restrict__ unorm8,
                           const BounceDev &b, const uint2 *prev, f3 o, f3 d, float tmax) {
  float b0 = 0.0f;
  for (uint32_t k = 0; k < v.levels && b0 * b.cell < tmax; k++) {
    const float b1 = b0 * 4.0f + 1.0f;
    const uint32_t L = vox_level_for(v, k, o + (d * b1) * b.cell);
    TraceOut r;
    trace_vox(v, F, unorm8, o, d, b0 * b.cell, mn(b1 * b.cell, tmax), 0.0f, L, BN_DDA_CAP, r, VolumeBounce{&b, prev});
    if (r.T < 0.5f) {
      const f3 entry = o + d * __uint_as_float(r.tin);
      return make_float4(r.rad.x, r.rad.y, r.rad.z, dot(entry - o, d));
    }
    b0 = b1;
  }
  return make_float4(F[F_SKY], F[F_SKY + 1], F[F_SKY + 2], 1e9f);
}

// bnUpdate (bounce.ts:172-208) in two launches.  k_bn_rays: one thread per ray of a listed probe, the probe's rays
// [0, rays) the irradiance rays and [rays, rays + 6) the axis rays (reach up to the first occupied voxel, at most 1.5
// cells), results kept per (probe, ray).  k_bn_sum: one thread per (probe, axis) sums the ambient cube over the rays
// in order.  The same operations as the reference's one workgroup per probe, with every lane tracing a ray.
__device__ __forceinline__ f3 bn_axis_vec(uint32_t a) {
  const float sg = (a & 1u) == 1u ? -1.0f : 1.0f;
  return a / 2u == 0u ? mk(sg, 0.0f, 0.0f) : (a / 2u == 1u ? mk(0.0f, sg, 0.0f) : mk(0.0f, 0.0f, sg));
}
// DYN (objects on, a layer bound): the irradiance rays read the dynamic layer in front of the static result at the
// width of one ray's cone (bnTraceDyn, bounce.ts:169-174)
template <bool DYN>
__global__ void __launch_bounds__(256) k_bn_rays(BounceDev b, VoxDev v, RcDev r) {
  grid_dep_wait();
  const float *__restrict__ F = r.frame;
  const float *__restrict__ unorm8 = r.unorm8;
  const uint32_t per = b.rays + 6u, total = b.list[0] * per;
  const uint2 *prev = b.vol[b.list[2] ^ 1u];
  const i3 o = bn_origin_now(b, F);
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    const uint32_t slot = t / per, k = t - slot * per;
    const uint32_t i = b.list[4u + slot];
    const i3 c = mki((int)(i % b.dx), (int)((i / b.dx) % b.dy), (int)(i / (b.dx * b.dy)));
    const f3 p = vi2f(mki(o.x + c.x, o.y + c.y, o.z + c.z)) * b.cell;
    float4 res;
    if (k < b.rays) {
      const float4 dv = b.dirs[k];
      res = bn_trace(v, F, unorm8, b, prev, p, mk(dv.x, dv.y, dv.z), 1e9f);
      if (DYN) {
        const float4 dl = trace_dyn(r, v, p, mk(dv.x, dv.y, dv.z), 0.0f, mn(res.w, 1e4f),
                                    sqrtf((4.0f * GI_PI) / (float)b.rays));
        const float s = 1.0f - dl.w;
        res = make_float4(dl.x + s * res.x, dl.y + s * res.y, dl.z + s * res.z, res.w);
      }
    } else {
      res = make_float4(0.0f, 0.0f, 0.0f,
                        mx(mn(bn_trace(v, F, unorm8, b, prev, p, bn_axis_vec(k - b.rays), 1.5f * b.cell).w, 1.5f * b.cell), 1e-3f));
    }
    b.ray_out[t] = res;
  }
}
__global__ void __launch_bounds__(256) k_bn_sum(BounceDev b) {
  grid_dep_wait();
  const uint32_t per = b.rays + 6u, total = b.list[0] * 6u;
  uint2 *out = b.vol[b.list[2]];
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    const uint32_t slot = t / 6u, a = t - slot * 6u;
    const uint32_t i = b.list[4u + slot];
    const i3 c = mki((int)(i % b.dx), (int)((i / b.dx) % b.dy), (int)(i / (b.dx * b.dy)));
    const float4 *rr = b.ray_out + (size_t)slot * per;
    const f3 axis = bn_axis_vec(a);
    f3 e = mk(0.0f, 0.0f, 0.0f);
    float ws = 0.0f;
    for (uint32_t r = 0; r < b.rays; r++) {
      const float4 dv = b.dirs[r], x = rr[r];
      const float w = mx(dot(axis, mk(dv.x, dv.y, dv.z)), 0.0f);
      e = e + mk(x.x, x.y, x.z) * w;
      ws += w;
    }
    const f3 irr = (e * GI_PI) / mx(ws, 1e-6f);
    out[bn_index(b, c, (int)a)] = bn_pack(make_float4(irr.x, irr.y, irr.z, rr[b.rays + a].w));
  }
}

// bnInject (bounce.ts:213-246): every occupied voxel stores this frame's volume read on its two sides.  One thread
// per voxel of the attribute pool (its brick by a binary search of the voxel prefix, as resolveAttr).
__global__ void __launch_bounds__(256) k_bn_inject(BounceDev b, VoxDev v) {
  grid_dep_wait();
  const uint2 *cur = b.vol[b.list[2]];
  const uint32_t nb = min(v.hdr[0], v.max_bricks);
  const uint32_t nv = nb ? min(v.vpre[nb], v.max_voxels) : 0u;
  for (uint32_t ai = blockIdx.x * blockDim.x + threadIdx.x; ai < nv; ai += gridDim.x * blockDim.x) {
    uint32_t lo = 0, hi = nb;
    while (hi - lo > 1u) {
      uint32_t m = (lo + hi) >> 1;
      if (v.vpre[m] <= ai) lo = m; else hi = m;
    }
    const uint32_t ptr = lo;
    if (v.base[ptr] == GI_EMPTY) continue;
    uint32_t r = ai - v.vpre[ptr], bit = 0;
    const uint4 *o4 = reinterpret_cast<const uint4 *>(v.occ) + ptr * 4u;
    for (int q = 0; q < 4; q++) {
      const uint4 o = o4[q];
      const uint32_t ws4[4] = {o.x, o.y, o.z, o.w};
      for (int j = 0; j < 4; j++) {
        const uint32_t pc = __popc(ws4[j]);
        if (r < pc && bit == 0u) {
          uint32_t wd = ws4[j];
          bit = (uint32_t)(q * 4 + j) * 32u + nth_set_bit(wd, r) + 1u;
        }
        if (bit == 0u) r -= pc;
      }
    }
    bit -= 1u;
    const uint32_t code = v.code[ptr], L = code >> 27;
    const i3 bc = mki((int)((code >> 18) & 511u), (int)((code >> 9) & 511u), (int)(code & 511u));
    const i3 cc = mki(bc.x * 8 + (int)(bit & 7u), bc.y * 8 + (int)((bit >> 3) & 7u), bc.z * 8 + (int)(bit >> 6));
    const float vs = vox_size(v, L);
    const f3 p = region_lo(v, L) + adds(vi2f(cc), 0.5f) * vs;
    const uint32_t e = v.attr[ai].y;
    const double inv32767 = 1.0 / 32767.0;   // unpack2x16snorm as the exact f64 product
    const float ex = mx(__double2float_rn((double)(int16_t)(e & 0xffffu) * inv32767), -1.0f);
    const float ey = mx(__double2float_rn((double)(int16_t)(e >> 16) * inv32767), -1.0f);
    f3 n = mk(ex, ey, 1.0f - fabsf(ex) - fabsf(ey));
    const float q0 = mx(-n.z, 0.0f);
    n.x += n.x >= 0.0f ? -q0 : q0;
    n.y += n.y >= 0.0f ? -q0 : q0;
    const f3 nf = dot(n, n) > 0.01f ? normalize3(n) : mk(0.0f, 1.0f, 0.0f);
    const float off = L == 0u ? 0.0f : 0.5f * vs;   // bnSide: coarser levels read half a voxel towards the side
    const f3 ef = bn_read(b, cur, p + nf * off, p, nf);
    const f3 eb = bn_read(b, cur, p + (-nf) * off, p, -nf);
    b.inj[ai] = make_uint4((uint32_t)f2h(ef.x) | ((uint32_t)f2h(ef.y) << 16), (uint32_t)f2h(ef.z),
                           (uint32_t)f2h(eb.x) | ((uint32_t)f2h(eb.y) << 16), (uint32_t)f2h(eb.z));
  }
}

// dynE of the bounce volume (bounce.ts:267-296): the irradiance at p of a dynamic voxel with projected areas P over its
// six axis faces, E = sum_a P_a E_a / sum_a P_a, E_a trilinear over the 8 probes around p with bnRead's rules (active,
// reach, side of the face)
__device__ f3 dyn_e(const BounceDev &b, const uint2 *vol, f3 p, const float P[6]) {
  const i3 org0 = bn_origin(b, vol);
  const f3 g = mk(p.x / b.cell, p.y / b.cell, p.z / b.cell) - vi2f(org0);
  const i3 bb = vfloori(g);
  const f3 fr = g - vi2f(bb);
  const float tol = 0.5f * b.v0;
  f3 e[6];
  float ws[6];
#pragma unroll
  for (int a = 0; a < 6; a++) { e[a] = mk(0.0f, 0.0f, 0.0f); ws[a] = 0.0f; }
  for (int k = 0; k < 8; k++) {
    const i3 off = mki(k & 1, (k >> 1) & 1, (k >> 2) & 1);
    const i3 cc = mki(bb.x + off.x, bb.y + off.y, bb.z + off.z);
    if (cc.x < 0 || cc.y < 0 || cc.z < 0 || cc.x >= (int)b.dx || cc.y >= (int)b.dy || cc.z >= (int)b.dz) continue;
    const f3 pp = vi2f(mki(org0.x + cc.x, org0.y + cc.y, org0.z + cc.z)) * b.cell;
    const f3 u = p - pp;
    if (bn_axis(b, vol, cc, 0).w <= 0.0f) continue;
    if (fabsf(u.x) > bn_axis(b, vol, cc, u.x >= 0.0f ? 0 : 1).w + tol || fabsf(u.y) > bn_axis(b, vol, cc, u.y >= 0.0f ? 2 : 3).w + tol
        || fabsf(u.z) > bn_axis(b, vol, cc, u.z >= 0.0f ? 4 : 5).w + tol) continue;
    const f3 t3 = mk(off.x == 1 ? fr.x : 1.0f - fr.x, off.y == 1 ? fr.y : 1.0f - fr.y, off.z == 1 ? fr.z : 1.0f - fr.z);
    const float wt = t3.x * t3.y * t3.z;
#pragma unroll
    for (int a = 0; a < 6; a++) {
      if (P[a] <= 0.0f) continue;
      const float w = wt * smoothstep_(-0.05f, 0.25f, dot(pp - p, bn_axis_vec((uint32_t)a)) / b.cell);
      if (w <= 0.0f) continue;
      const float4 ax = bn_axis(b, vol, cc, a);
      e[a] = e[a] + mk(ax.x, ax.y, ax.z) * w;
      ws[a] += w;
    }
  }
  f3 sum = mk(0.0f, 0.0f, 0.0f);
  float ps = 0.0f;
#pragma unroll
  for (int a = 0; a < 6; a++) {
    if (ws[a] > 1e-6f) sum = sum + (e[a] * P[a]) / ws[a];
    ps += P[a];
  }
  return sum / mx(ps, 1e-9f);
}

// dynInject (dynlayer.ts:173-191), phase 31: before this frame's volume, every voxel of the layer's allocated bricks
// with area adds albedo / pi times dynE of the previous frame's volume to its radiance words (level 0 in fixed point,
// the levels above in f32).  One thread per voxel slot; each thread owns its voxel's words.
__global__ void __launch_bounds__(256) k_dyn_inject(RcDev r, BounceDev b, VoxDev v) {
  grid_dep_wait();
  const uint2 *prev = b.vol[b.list[2]];   // the volume written last (k_bn_clear swaps after this)
  const uint32_t G = v.G, G3 = G * G * G;
  const uint32_t n = min(r.dyn_hdr[8], r.dyn_nb) * 512u;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t slot = i >> 9, bit = i & 511u;
    const uint32_t pi = r.dyn_meta[slot], L = pi / G3, rr = pi % G3;
    const uint32_t base = i * DYN_W;
    if (dyn_word(r, base, 6u, L) <= 0.0f) continue;
    float P[6];
#pragma unroll
    for (uint32_t k = 0; k < 6u; k++) P[k] = dyn_word(r, base, k, L);
    const i3 c = mki((int)(rr % G) * 8 + (int)(bit & 7u), (int)((rr / G) % G) * 8 + (int)((bit >> 3) & 7u),
                     (int)(rr / (G * G)) * 8 + (int)(bit >> 6));
    const float vs = vox_size(v, L);
    const f3 p = region_lo(v, L) + adds(vi2f(c), 0.5f) * vs;
    const f3 E = dyn_e(b, prev, p, P);
    const f3 alb = mk(dyn_word(r, base, 10u, L), dyn_word(r, base, 11u, L), dyn_word(r, base, 12u, L));
    const f3 add = (alb / GI_PI) * E;
    const float a3[3] = {add.x, add.y, add.z};
#pragma unroll
    for (uint32_t k = 0; k < 3u; k++) {
      uint32_t *w = &r.dyn_data[base + 7u + k];
      if (L == 0u) *w += __float2uint_rz(rintf(a3[k] * DYN_FIX));
      else *w = __float_as_uint(__uint_as_float(*w) + a3[k]);
    }
  }
}

// One frame of the bounce volume (Bounce.encode, bounce.ts:356-368), at the start of the trace pass; with objects on
// and a layer bound, dynInject first and the irradiance rays reading the layer
static cudaError_t launch_bounce(const BounceDev &b, const VoxDev &v, const RcDev &r, uint32_t sm_count, cudaStream_t st) {
  const float *frame = r.frame;
  const bool dyn = r.objects && r.dyn_hdr;
  if (dyn) GI_TRY(gi_launch(k_dyn_inject, sm_count * 8u, 256, st, r, b, v));
  GI_TRY(gi_launch(k_bn_clear, 1, 32, st, b));
  GI_TRY(gi_launch(k_bn_classify, (b.n + 1u + 255u) / 256u, 256, st, b, v, frame));
  if (dyn) GI_TRY(gi_launch(k_bn_rays<true>, sm_count * 4u, 256, st, b, v, r));
  else GI_TRY(gi_launch(k_bn_rays<false>, sm_count * 4u, 256, st, b, v, r));
  GI_TRY(gi_launch(k_bn_sum, sm_count, 256, st, b));
  GI_TRY(gi_launch(k_bn_inject, sm_count * 8u, 256, st, b, v));
  return cudaSuccess;
}

// ---- batches of solves, one launch per pass (gi_batch_capture_passes) ----------------------------------------------

// The last solve s with pre[s] <= x (the owner of item x: solves with no items share the next one's start)
__device__ __forceinline__ uint32_t batch_owner(const uint32_t *__restrict__ pre, uint32_t n, uint32_t x) {
  uint32_t lo = 0, hi = n;
  while (hi - lo > 1u) {
    uint32_t m = (lo + hi) >> 1;
    if (__ldg(&pre[m]) <= x) lo = m; else hi = m;
  }
  return lo;
}

__global__ void __launch_bounds__(256) k_setup_batch(BatchDev B) {
  grid_dep_wait();
  const uint32_t s = batch_owner(B.setup_blk, B.n, blockIdx.x), b = blockIdx.x - B.setup_blk[s];
  const RcDev &r = B.rc[s];
  if (b == 0 && threadIdx.x < 81u && threadIdx.x >= r.cascades) r.counts[threadIdx.x] = 0u;
  if (blockIdx.x == 0 && threadIdx.x == 0) B.counter[0] = 0u;
  const uint32_t i = b * 256u + threadIdx.x;
  if (i < r.probes_total) setup_probe(r, B.vox[s], i);
}

// Persistent over the rays of every solve: warps take 32 rays at a time; solves are padded to 32 rays, so a fetch
// belongs to one solve
template <int A>
__global__ void __launch_bounds__(256) k_trace_batch(BatchDev B) {
  grid_dep_wait();
  const uint32_t lane = threadIdx.x & 31u, total = B.ray_pre[B.n];
  for (;;) {
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(B.counter, 32u);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= total) break;
    const uint32_t s = batch_owner(B.ray_pre, B.n, base);
    const RcDev &r = B.rc[s];
    const uint32_t j = base - B.ray_pre[s] + lane;
    if (j < r.rays_total) {
      TraceOut out;
      trace_ray<A>(r, B.vox[s], j, casc_of_ray(r, j), out, r.trace_order != 1u);
    }
  }
}

// Merge step k: every solve merges its cascade C - 1 - k (solves with fewer cascades have no blocks)
template <int A>
__global__ void __launch_bounds__(256) k_merge_batch(BatchDev B, uint32_t k) {
  grid_dep_wait();
  const uint32_t *pre = B.merge_blk + k * (B.n + 1u);
  const uint32_t s = batch_owner(pre, B.n, blockIdx.x);
  const RcDev &r = B.rc[s];
  const uint32_t c = r.cascades - 1u - k;
  float4 *mine = (c > 0u && r.c[c - 1u].res * 2u == r.c[c].res) ? r.mavg[c & 1u] : nullptr;
  merge_quad<A>(r, c, (blockIdx.x - pre[s]) * 256u + threadIdx.x, r.mavg[(c + 1u) & 1u], mine);
}

template <int A, uint32_t P>
__global__ void __launch_bounds__(256) k_gather_batch(BatchDev B) {
  grid_dep_wait();
  const uint32_t s = batch_owner(B.gather_blk, B.n, blockIdx.x), lb = blockIdx.x - B.gather_blk[s];
  const RcDev &r = B.rc[s];
  const uint32_t gx = ((r.width + P / 2u + P - 1u) / P + 1u) / 2u;
  gather_tiles<A, P>(r, lb % gx, lb / gx);
}

template <int A, uint32_t P>
static cudaError_t launch_batch(const BatchDev &b, const BatchSizes &z, uint32_t sm_count, cudaStream_t st) {
  GI_TRY(gi_launch(k_setup_batch, z.setup_blocks, 256, st, b));
  GI_TRY(gi_launch(k_trace_batch<A>, sm_count * 4u, 256, st, b));
  for (uint32_t k = 0; k < b.max_casc; k++)
    if (z.merge_blocks[k]) GI_TRY(gi_launch(k_merge_batch<A>, z.merge_blocks[k], 256, st, b, k));
  GI_TRY(gi_launch(k_gather_batch<A, P>, z.gather_blocks, 256, st, b));
  return cudaGetLastError();
}

template <int A>
static cudaError_t launch_batch_p(const BatchDev &b, const BatchSizes &z, uint32_t sm_count, cudaStream_t st) {
  if (z.P0 == 8u) return launch_batch<A, 8u>(b, z, sm_count, st);
  if (z.P0 == 16u) return launch_batch<A, 16u>(b, z, sm_count, st);
  if (z.P0 == 32u) return launch_batch<A, 32u>(b, z, sm_count, st);
  return cudaErrorInvalidValue;
}

__global__ void k_irr_to_f32(RcDev r, float4 *dst) {
  grid_dep_wait();
  size_t n = (size_t)r.width * r.height;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    if ((r.atlas == GI_ATLAS_F32 || r.f32_out) && !r.irr_f16) dst[i] = reinterpret_cast<const float4 *>(r.irr)[i];
    else {
      uint2 u = reinterpret_cast<const uint2 *>(r.irr)[i];
      dst[i] = make_float4(h2f(u.x & 0xffffu), h2f(u.x >> 16), h2f(u.y & 0xffffu), h2f(u.y >> 16));
    }
  }
}

// dirOf(di, res) (rc.ts:308) of every texel of every cascade, once per Rc
__global__ void k_init_dirs(RcDev r, float4 *dirs, uint32_t ndirs) {
  grid_dep_wait();
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ndirs) return;
  uint32_t c = 0;
  for (uint32_t k = 1; k < r.cascades; k++) if (i >= r.c[k].dir_off) c = k;
  f3 d = dir_of(i - r.c[c].dir_off, r.c[c].res);
  dirs[i] = make_float4(d.x, d.y, d.z, 0.0f);
  // traceVox's 1 / d with tiny components clamped (voxel.ts:127), as trace_vox computes it
  const f3 dd = mk(fabsf(d.x) < 1e-9f ? 1e-9f : d.x, fabsf(d.y) < 1e-9f ? 1e-9f : d.y, fabsf(d.z) < 1e-9f ? 1e-9f : d.z);
  dirs[ndirs + i] = make_float4(1.0f / dd.x, 1.0f / dd.y, 1.0f / dd.z, 0.0f);
}

// rgb16f normals (three halves per pixel) to the rgba16f layout the kernels read, alpha 0
__global__ void k_normal_rgb_to_rgba(const uint16_t *__restrict__ src, uint2 *__restrict__ dst, uint32_t n) {
  grid_dep_wait();
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint16_t *s = src + 3u * (size_t)i;
    dst[i] = make_uint2((uint32_t)s[0] | ((uint32_t)s[1] << 16), (uint32_t)s[2]);
  }
}

__global__ void k_normal_f32_to_f16(const float4 *src, uint2 *dst, uint32_t n) {
  grid_dep_wait();
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float4 s = src[i];
    dst[i] = make_uint2((uint32_t)f2h(s.x) | ((uint32_t)f2h(s.y) << 16), (uint32_t)f2h(s.z) | ((uint32_t)f2h(s.w) << 16));
  }
}

template <int A>
static cudaError_t launch_solve(const RcDev &r, const VoxDev &v, uint32_t sm_count, cudaStream_t st, cudaEvent_t *ev,
                                const RcLaunch *ls, const BounceDev *bn) {
  uint32_t *counter = r.counts + 80;   // the trace's ray counter lives after the 80 counter words
  if (ev) cudaEventRecord(ev[0], st);
  GI_TRY(gi_launch(k_setup_screen, (r.probes_total + 255u) / 256u, 256, st, r, v));
  if (ev) cudaEventRecord(ev[1], st);
  if (bn) GI_TRY(launch_bounce(*bn, v, r, sm_count, st));   // counted in giTrace, as the reference
  RcLaunch d = {8u, 3u, 256u};
  if (ls) d = *ls;
  uint32_t tb = min((r.rays_total + 255u) / 256u, sm_count * d.trace_blocks);
  // the dynamic layer's read is compiled into a kernel of its own: without a layer the trace keeps its registers
  if (r.trace_order == 2u && r.rperm) {   // walk-length order from the previous solve's keys
    GI_TRY(gi_launch(k_rsort_hist, min((r.rays_total + 1023u) / 1024u, sm_count * 8u), 256, st, r));
    GI_TRY(gi_launch(k_rsort_scatter, (r.rays_total + RS_PER_BLOCK - 1u) / RS_PER_BLOCK, 256, st, r));
    if (r.dyn_hdr) GI_TRY(gi_launch(k_trace<A, true, true>, tb, 256, st, r, v, counter));
    else GI_TRY(gi_launch(k_trace<A, false, true>, tb, 256, st, r, v, counter));
  } else if (r.dyn_hdr) {
    GI_TRY(gi_launch(k_trace<A, true, false>, tb, 256, st, r, v, counter));
  } else {
    GI_TRY(gi_launch(k_trace<A, false, false>, tb, 256, st, r, v, counter));
  }
  if (ev) cudaEventRecord(ev[2], st);
  for (int c = (int)r.cascades - 1; c >= 0; c--) {
    const CascDev &L = r.c[c];
    uint32_t n = L.np * (L.res * L.res / 4u);   // quads
    // quad averages: written when the cascade below has half this resolution, read from the cascade above
    float4 *mine = (c > 0 && r.c[c - 1].res * 2u == L.res) ? r.mavg[c & 1] : nullptr;
    const float4 *above = r.mavg[(c + 1) & 1];
    GI_TRY(gi_launch(k_merge<A>, (n + d.merge_threads - 1u) / d.merge_threads, d.merge_threads, st, r, (uint32_t)c, above, mine));
  }
  if (ev) cudaEventRecord(ev[3], st);
  const uint32_t P0 = r.c[0].tile_size;
  if (d.gather_shape == 3 && (P0 == 8u || P0 == 16u || P0 == 32u)) {
    uint32_t th = 32u / P0;   // warp tiles start half a probe cell before the screen
    uint32_t ntx = (r.width + P0 / 2u + P0 - 1u) / P0, nty = (r.height + P0 / 2u + th - 1u) / th;
    dim3 gg((ntx + 1u) / 2u, (nty + 3u) / 4u);
    if (P0 == 8u) GI_TRY(gi_launch(k_gather_tiled<A, 8u>, gg, 256, st, r));
    else if (P0 == 16u) GI_TRY(gi_launch(k_gather_tiled<A, 16u>, gg, 256, st, r));
    else GI_TRY(gi_launch(k_gather_tiled<A, 32u>, gg, 256, st, r));
  } else {
    uint32_t bx = d.gather_shape == 1 ? 32u : (d.gather_shape == 2 ? 8u : 16u), by = 256u / bx;
    dim3 gg((r.width + bx - 1u) / bx, (r.height + by - 1u) / by);
    if (bx == 32u) GI_TRY(gi_launch(k_gather<A, 32u>, gg, 256, st, r));
    else if (bx == 8u) GI_TRY(gi_launch(k_gather<A, 8u>, gg, 256, st, r));
    else GI_TRY(gi_launch(k_gather<A, 16u>, gg, 256, st, r));
  }
  if (ev) cudaEventRecord(ev[4], st);
  return cudaGetLastError();
}

// ---- world probes (method 'world') ----------------------------------------------------------------------------------
#include "world.cuh"

}  // namespace gi

using namespace gi;

cudaError_t gi_world_tables() {
  float t[16 * 16];
  for (int k = 1; k <= 16; k++)
    for (int i = 0; i < 16; i++) {
      volatile float a = (float)i + 0.5f, b = (float)k;
      t[(k - 1) * 16 + i] = i < k ? a / b : 0.0f;
    }
  return cudaMemcpyToSymbol(g_seg_t, t, sizeof t);
}

cudaError_t gi_launch_rc_solve(const RcDev &r, const VoxDev &v, uint32_t sm_count, cudaStream_t st, cudaEvent_t *ev,
                               const RcLaunch *ls, const BounceDev *bn, const WorldDev *w) {
  if (w) {
    switch (r.atlas) {
      case GI_ATLAS_F32: return launch_world<GI_ATLAS_F32>(r, v, *w, sm_count, st, ev, ls, bn);
      case GI_ATLAS_F16: return launch_world<GI_ATLAS_F16>(r, v, *w, sm_count, st, ev, ls, bn);
      case GI_ATLAS_BF16: return launch_world<GI_ATLAS_BF16>(r, v, *w, sm_count, st, ev, ls, bn);
    }
    return cudaErrorInvalidValue;
  }
  switch (r.atlas) {
    case GI_ATLAS_F32: return launch_solve<GI_ATLAS_F32>(r, v, sm_count, st, ev, ls, bn);
    case GI_ATLAS_F16: return launch_solve<GI_ATLAS_F16>(r, v, sm_count, st, ev, ls, bn);
    case GI_ATLAS_BF16: return launch_solve<GI_ATLAS_BF16>(r, v, sm_count, st, ev, ls, bn);
  }
  return cudaErrorInvalidValue;
}

cudaError_t gi_launch_irr_to_f32(const RcDev &r, float4 *dst, cudaStream_t st) {
  k_irr_to_f32<<<256, 256, 0, st>>>(r, dst);
  return cudaGetLastError();
}

cudaError_t gi_launch_init_dirs(const RcDev &r, float4 *dirs, uint32_t ndirs, cudaStream_t st) {
  k_init_dirs<<<(ndirs + 255u) / 256u, 256, 0, st>>>(r, dirs, ndirs);
  return cudaGetLastError();
}

cudaError_t gi_launch_normal_f32_to_f16(const float4 *src, uint2 *dst, uint32_t n, cudaStream_t st) {
  k_normal_f32_to_f16<<<256, 256, 0, st>>>(src, dst, n);
  return cudaGetLastError();
}

__global__ void k_iota(uint32_t *dst, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[i] = i;
}

cudaError_t gi_launch_iota(uint32_t *dst, uint32_t n, cudaStream_t st) {
  k_iota<<<1184, 256, 0, st>>>(dst, n);
  return cudaGetLastError();
}

cudaError_t gi_launch_normal_rgb_to_rgba(const uint16_t *src, uint2 *dst, uint32_t n, cudaStream_t st) {
  k_normal_rgb_to_rgba<<<1184, 256, 0, st>>>(src, dst, n);
  return cudaGetLastError();
}

cudaError_t gi_launch_batch_passes(const BatchDev &b, const BatchSizes &z, uint32_t sm_count, cudaStream_t st) {
  switch (z.atlas) {
    case GI_ATLAS_F32: return launch_batch_p<GI_ATLAS_F32>(b, z, sm_count, st);
    case GI_ATLAS_F16: return launch_batch_p<GI_ATLAS_F16>(b, z, sm_count, st);
    case GI_ATLAS_BF16: return launch_batch_p<GI_ATLAS_BF16>(b, z, sm_count, st);
  }
  return cudaErrorInvalidValue;
}
