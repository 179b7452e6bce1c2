// The dynamic layer on sm_100a (src/core/dynlayer.ts): moving triangles (the scene's tail from DynDev.first) are not
// voxelised into the binary bricks; every frame they are splatted into a separate layer of coverage and mean radiance,
// prefiltered fine to coarse, which the interval tracers read at the width of a direction bin's cone (rc_solve.cu).
//
// Passes (dynlayer.ts:592): mark (thread per dynamic triangle: splat level, wanted bricks, bounds), parents (thread per
// bitset word: every wanted brick wants its ancestors), alloc (the reference's count + alloc as one chained scan over
// the bitset words: slots by rank in bit order, bricks only wanted last frame emptied), finalize (one thread), clear
// (thread per voxel of the allocated bricks), splat (a warp per dynamic triangle, its m^2 samples added in fixed point
// with atomics: exact sums, so the result is the reference's whatever the order), resolve (per level from fine to
// coarse, thread per voxel).  The reference gathers a workgroup's samples in a window of workgroup memory before adding
// them; here every sample is added to the layer, and a voxel is marked non-zero when a sample's weight on it is
// positive (the window marks it only when its summed words are non-zero; no value depends on which).
#include <cuda_runtime.h>

#include "gi_dev.cuh"
#include "gi_internal.h"
#include "gi_scan.cuh"

namespace gi {

constexpr uint32_t DYN_NONE = 0xffffffffu;

__device__ __forceinline__ f3 dyn_lo(const VoxDev &v, uint32_t L) { return mk(v.box_lo[L][0], v.box_lo[L][1], v.box_lo[L][2]); }
__device__ __forceinline__ f3 dyn_hi(const VoxDev &v, uint32_t L) { return mk(v.box_hi[L][0], v.box_hi[L][1], v.box_hi[L][2]); }
__device__ __forceinline__ f3 dyn_pos(const SceneDev &s, uint32_t i) { return ld3(s.pos[i]); }
__device__ __forceinline__ f3 dyn_nrm(const SceneDev &s, uint32_t i) { return ld3(s.nrm[i]); }
__device__ __forceinline__ uint32_t dyn_nw(const VoxDev &v) { return v.levels * v.G * v.G * v.G / 32u; }

// splatLevel (dynlayer.ts:221-229): the finest level whose clipmap holds the box grown by two voxels
__device__ __forceinline__ uint32_t splat_level(const VoxDev &v, f3 mn, f3 mx) {
  for (uint32_t L = 0; L < v.levels; L++) {
    const float vs = vox_size(v, L), v2 = 2.0f * vs;
    const f3 lo = dyn_lo(v, L), hi = dyn_hi(v, L);
    if (mn.x - v2 > lo.x && mn.y - v2 > lo.y && mn.z - v2 > lo.z && mx.x + v2 < hi.x && mx.y + v2 < hi.y && mx.z + v2 < hi.z)
      return L;
  }
  return DYN_NONE;
}

// want (dynlayer.ts:236-243): brick b of level L in this frame's bitset
__device__ __forceinline__ void dyn_want(const DynDev &d, const VoxDev &v, uint32_t L, i3 b) {
  const int G = (int)v.G;
  if (b.x < 0 || b.y < 0 || b.z < 0 || b.x >= G || b.y >= G || b.z >= G) return;
  const uint32_t ug = v.G, g = (v.levels - 1u - L) * ug * ug * ug + ((uint32_t)b.z * ug + (uint32_t)b.y) * ug + (uint32_t)b.x;
  uint32_t *w = d.bits + (d.hdr[10] & 1u) * dyn_nw(v) + (g >> 5);
  const uint32_t m = 1u << (g & 31u);
  if ((*w & m) == 0u) atomicOr(w, m);
}

// mark (dynlayer.ts:246-270).  Block 0 also clears the allocation's scan states.
__global__ void __launch_bounds__(256) k_dyn_mark(DynDev d, VoxDev v, SceneDev s) {
  grid_dep_wait();
  if (blockIdx.x == 0)
    for (uint32_t q = threadIdx.x; q <= d.look_cap; q += blockDim.x) d.look[q] = 0ull;
  const uint32_t t = d.first + blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= d.end) return;
  const uint4 ti = s.tri[t];
  const f3 a = dyn_pos(s, ti.x), b = dyn_pos(s, ti.y), c = dyn_pos(s, ti.z);
  const f3 mn = vmin(vmin(a, b), c), mx = vmax(vmax(a, b), c);
  const uint32_t Ls = splat_level(v, mn, mx);
  if (Ls == DYN_NONE) { atomicAdd(&d.hdr[38], 1u); return; }
  const float vs = vox_size(v, Ls), bs = vs * 8.0f;
  const f3 lo = dyn_lo(v, Ls);
  const i3 g0 = vfloori(((mn - mk(vs, vs, vs)) - lo) / bs), g1 = vfloori(((mx + mk(vs, vs, vs)) - lo) / bs);
  for (int z = g0.z; z <= g1.z; z++)
    for (int y = g0.y; y <= g1.y; y++)
      for (int x = g0.x; x <= g1.x; x++) dyn_want(d, v, Ls, mki(x, y, z));
  // bounds of what a read can see: the box grown by the coarsest voxel (cm, offset by 2^30)
  const float gv = vox_size(v, v.levels - 1u);
  const float mnv[3] = {mn.x, mn.y, mn.z}, mxv[3] = {mx.x, mx.y, mx.z};
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const uint32_t blo = (uint32_t)(__float2int_rz(floorf((mnv[k] - gv) * 100.0f)) + 1073741824);
    const uint32_t bhi = (uint32_t)(__float2int_rz(ceilf((mxv[k] + gv) * 100.0f)) + 1073741824);
    atomicMin(&d.hdr[32 + k], blo);
    atomicMax(&d.hdr[35 + k], bhi);
  }
}

// parents (dynlayer.ts:272-296): thread per bitset word below the coarsest level
__global__ void __launch_bounds__(256) k_dyn_parents(DynDev d, VoxDev v) {
  grid_dep_wait();
  const uint32_t G = v.G, G3 = G * G * G, n = v.levels, nw = dyn_nw(v);
  const uint32_t w = G3 / 32u + blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= nw) return;
  uint32_t m = d.bits[(d.hdr[10] & 1u) * nw + w];
  while (m) {
    const uint32_t bit = __ffs(m) - 1u;
    m &= m - 1u;
    const uint32_t g = w * 32u + bit, lr = g / G3, r = g - lr * G3;
    uint32_t L = n - 1u - lr;
    i3 b = mki((int)(r % G), (int)((r / G) % G), (int)(r / (G * G)));
    while (L + 1u < n) {
      const i3 o = org(v, L), o1 = org(v, L + 1u);
      b = mki(((o.x + b.x) * 8 / 2 - o1.x * 8) >> 3, ((o.y + b.y) * 8 / 2 - o1.y * 8) >> 3, ((o.z + b.z) * 8 / 2 - o1.z * 8) >> 3);
      L++;
      dyn_want(d, v, L, b);
    }
  }
}

// count + alloc (dynlayer.ts:311-362) in one pass: each block takes 256 consecutive bitset words (a word per thread)
// in ticket order; the prefix of the wanted bricks before its words comes from a chained scan.
__global__ void __launch_bounds__(256) k_dyn_alloc(DynDev d, VoxDev v) {
  grid_dep_wait();
  const uint32_t G = v.G, G3 = G * G * G, n = v.levels, nw = dyn_nw(v);
  const uint32_t blk = chain_ticket(d.look);
  const uint32_t w = blk * 256u + threadIdx.x;
  const uint32_t par = d.hdr[10] & 1u;
  uint32_t cur = 0, old = 0;
  if (w < nw) { cur = d.bits[par * nw + w]; old = d.bits[(1u - par) * nw + w]; }
  const uint32_t c = __popc(cur);
  uint32_t tot;
  uint32_t ex = block_scan_256(c, &tot);
  __shared__ uint32_t s_pre;
  if (threadIdx.x == 0) s_pre = chain_prefix(d.look, blk, tot, d.hdr + 6);   // a give-up sets header word 12
  __syncthreads();
  const uint32_t excl = s_pre + ex;
  if (w >= nw) return;
  if ((w * 32u) % G3 == 0u) d.hdr[16u + n - 1u - w * 32u / G3] = excl;
  if (w == nw - 1u) d.hdr[0] = excl + c;
  uint32_t m = cur | old;
  while (m) {
    const uint32_t bit = __ffs(m) - 1u;
    m &= m - 1u;
    const uint32_t g = w * 32u + bit, lr = g / G3, pi = (n - 1u - lr) * G3 + g - lr * G3;
    if ((cur >> bit) & 1u) {
      const uint32_t rank = excl + __popc(cur & ((1u << bit) - 1u));
      if (rank < d.nb) { d.ptr[pi] = rank; d.meta[rank] = pi; }
      else d.ptr[pi] = DYN_DROPPED;
    } else {
      d.ptr[pi] = DYN_EMPTY;
    }
  }
  d.bits[(1u - par) * nw + w] = 0u;
}

// finalize (dynlayer.ts:364-386): slots and counts per level; publishes the bounds and the outside count, flips the
// bitsets
__global__ void k_dyn_finalize(DynDev d, VoxDev v) {
  grid_dep_wait();
  uint32_t *h = d.hdr;
  const uint32_t total = h[0], al = min(total, d.nb);
  h[8] = al; h[1] = total - al;
  for (uint32_t L = 0; L < v.levels; L++) {
    const uint32_t e = L > 0 ? h[16u + L - 1u] : total;
    const uint32_t s0 = min(h[16u + L], d.nb);
    h[16u + L] = s0; h[24u + L] = min(e, d.nb) - s0;
  }
  for (int k = 0; k < 3; k++) {
    h[2 + k] = h[32 + k]; h[32 + k] = 0xffffffffu;
    h[5 + k] = h[35 + k]; h[35 + k] = 0u;
  }
  h[9] = h[38]; h[38] = 0u;
  h[10] += 1u;
}

// clear (dynlayer.ts:387-392): the allocated bricks' words and their bits of non-zero voxels
__global__ void __launch_bounds__(256) k_dyn_clear(DynDev d) {
  grid_dep_wait();
  const uint32_t n = d.hdr[8] * 512u;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
#pragma unroll
    for (uint32_t k = 0; k < DYN_W; k++) d.data[(size_t)i * DYN_W + k] = 0u;
    if (i % 512u < 16u) d.mask[i / 512u * 16u + i % 512u] = 0u;
  }
}

// WGSL u32(round(x)) of a non-negative x: round half to even, saturating
__device__ __forceinline__ uint32_t fix_of(float x) { return __float2uint_rz(rintf(x * DYN_FIX)); }

// shadeSample (dynlayer.ts:445-455): tc the sampled base colour (texture times factor, or the factor untextured); false
// when the alpha test discards the sample
__device__ __forceinline__ bool shade_sample(const gi_material &m, float4 tc, const float *__restrict__ F,
                                             const float *__restrict__ map, uint32_t S, uint32_t layers, f3 p, f3 n,
                                             f3 &rad, f3 &alb) {
  const f3 tex = mk(tc.x, tc.y, tc.z);
  if ((m.flags & 1u) != 0u && tc.w < m.alpha_cutoff) return false;
  alb = tex;
  const float ndl = mx(dot(n, mk(F[F_SUN], F[F_SUN + 1], F[F_SUN + 2])), 0.0f);
  if (ndl <= 0.0f) { rad = mk(0.0f, 0.0f, 0.0f); return true; }
  const float vis = (map && S) ? sun_tap(F, map, S, layers, p + n * 0.03f) : 1.0f;
  const f3 sunE = mk(F[F_SUNE], F[F_SUNE + 1], F[F_SUNE + 2]);
  if ((m.flags & 4u) != 0u && F[F_STYLE] > 0.5f) {   // toonSun (style.ts:18-25)
    const float l = dot(tex, mk(0.2126f, 0.7152f, 0.0722f));
    f3 t = mk(l, l, l) + (tex - mk(l, l, l)) * 1.6f;
    t = mk(fclampf(t.x, 0.0f, 1.0f), fclampf(t.y, 0.0f, 1.0f), fclampf(t.z, 0.0f, 1.0f));
    const float x = ndl * vis, ramp = x > 0.3f ? 1.0f : (x > 0.05f ? 0.5f : 0.0f);
    rad = ((t / GI_PI) * sunE) * ramp;
    return true;
  }
  rad = (((tex / GI_PI) * sunE) * ndl) * vis;
  return true;
}

// splatSample (dynlayer.ts:406-441): the sample's trilinear weights over the 8 nearest voxel centres, added in fixed
// point
__device__ __forceinline__ void splat_sample(const DynDev &d, const VoxDev &v, uint32_t L, f3 p, f3 n, float area, f3 rad,
                                             f3 alb) {
  const float vs = vox_size(v, L);
  const f3 g = adds((p - dyn_lo(v, L)) / vs, -0.5f);
  const i3 c0 = vfloori(g);
  const f3 f = g - vi2f(c0);
  const float s = area / (vs * vs);
  const f3 pn = vmax(n, mk(0.0f, 0.0f, 0.0f)), nn = vmax(-n, mk(0.0f, 0.0f, 0.0f));
  const int G8 = (int)v.G * 8;
  const uint32_t G = v.G;
  const uint32_t nw = d.albedo ? 13u : 10u;
#pragma unroll 1
  for (uint32_t k = 0; k < 8u; k++) {
    const i3 o = mki((int)(k & 1u), (int)((k >> 1) & 1u), (int)(k >> 2));
    const i3 c = mki(c0.x + o.x, c0.y + o.y, c0.z + o.z);
    if (c.x < 0 || c.y < 0 || c.z < 0 || c.x >= G8 || c.y >= G8 || c.z >= G8) continue;
    const f3 tw = mk(o.x == 1 ? f.x : 1.0f - f.x, o.y == 1 ? f.y : 1.0f - f.y, o.z == 1 ? f.z : 1.0f - f.z);
    const float w = ((tw.x * tw.y) * tw.z) * s;
    if (w <= 0.0f) continue;
    const uint32_t ptr = d.ptr[L * G * G * G + ((uint32_t)(c.z >> 3) * G + (uint32_t)(c.y >> 3)) * G + (uint32_t)(c.x >> 3)];
    if (ptr >= d.nb) continue;
    const uint32_t vi = (uint32_t)((c.x & 7) + 8 * (c.y & 7) + 64 * (c.z & 7));
    atomicOr(&d.mask[ptr * 16u + (vi >> 5)], 1u << (vi & 31u));
    uint32_t *q = d.data + ((size_t)ptr * 512u + vi) * DYN_W;
    const float x[13] = {w * pn.x, w * nn.x, w * pn.y, w * nn.y, w * pn.z, w * nn.z, w, w * rad.x, w * rad.y, w * rad.z,
                         w * alb.x, w * alb.y, w * alb.z};
    for (uint32_t j = 0; j < nw; j++) {
      const uint32_t u = fix_of(x[j]);
      if (u) atomicAdd(&q[j], u);
    }
  }
}

// splat (dynlayer.ts:458-526): a warp per dynamic triangle, its m^2 sub-triangles' centroids dealt over the lanes (a
// sample's sums are fixed point, so which lane adds it and when changes nothing).  Sample q of row u: the row's m - u
// upright sub-triangles first, then its m - u - 1 flipped ones.
__global__ void __launch_bounds__(256) k_dyn_splat(DynDev d, VoxDev v, SceneDev s, const float *__restrict__ F,
                                                   const float *__restrict__ map, uint32_t S, uint32_t layers) {
  grid_dep_wait();
  const uint32_t t = d.first + (blockIdx.x * blockDim.x + threadIdx.x) / 32u, lane = threadIdx.x & 31u;
  if (t >= d.end) return;
  const uint4 ti = s.tri[t];
  const f3 a = dyn_pos(s, ti.x), b = dyn_pos(s, ti.y), c = dyn_pos(s, ti.z);
  const uint32_t L = splat_level(v, vmin(vmin(a, b), c), vmax(vmax(a, b), c));
  if (L == DYN_NONE) return;
  const float area = 0.5f * length3(cross(b - a, c - a));
  if (area <= 0.0f) return;
  const float e = mx(mx(length3(b - a), length3(c - b)), length3(a - c));
  const uint32_t m = (uint32_t)fclampf(ceilf(e / vox_size(v, L)), 1.0f, 16.0f);
  const float fm = (float)m, sa = area / (fm * fm);
  const gi_material mat = s.mats[ti.w];
  const uint32_t tex_layer = tex_layer_of(s, mat);
  const f3 n0 = dyn_nrm(s, ti.x), n1 = dyn_nrm(s, ti.y), n2 = dyn_nrm(s, ti.z);
  for (uint32_t q = lane; q < m * m; q += 32u) {
    uint32_t u = 0, r = q;
    while (r >= 2u * (m - u) - 1u) { r -= 2u * (m - u) - 1u; u++; }
    const uint32_t flip = r >= m - u ? 1u : 0u, vv = flip ? r - (m - u) : r;
    const float off = flip == 1u ? 2.0f / 3.0f : 1.0f / 3.0f;
    const float wb = ((float)u + off) / fm, wc = ((float)vv + off) / fm, wa = (1.0f - wb) - wc;
    const f3 p = (a * wa + b * wb) + c * wc;
    f3 nr = (n0 * wa + n1 * wb) + n2 * wc;
    nr = normalize3(dot(nr, nr) > 1e-12f ? nr : cross(b - a, c - a));
    f3 rad, alb;
    float4 tc = make_float4(mat.base_color[0], mat.base_color[1], mat.base_color[2], mat.base_color[3]);
    if (tex_layer) {   // the texture at level 3 + L at the sample's uv, times the factor
      const float2 uv = tri_uv(s, ti, wa, wb, wc);
      const float4 t = tex_sample(s, tex_layer, uv.x, uv.y, 3u + L);
      tc = make_float4(t.x * mat.base_color[0], t.y * mat.base_color[1], t.z * mat.base_color[2], t.w * mat.base_color[3]);
    }
    if (!shade_sample(mat, tc, F, map, S, layers, p, nr, rad, alb)) continue;
    splat_sample(d, v, L, p, nr, sa, rad, alb);
  }
}

// resolve (dynlayer.ts:527-587) of level L >= 1: own splats (fixed point) + a quarter of each non-zero child (fixed
// point on level 0, f32 above), stored as f32
__global__ void __launch_bounds__(256) k_dyn_resolve(DynDev d, VoxDev v, uint32_t L) {
  grid_dep_wait();
  const uint32_t G = v.G, G3 = G * G * G;
  const uint32_t n = d.hdr[24u + L] * 512u, s0 = d.hdr[16u + L];
  const i3 o = org(v, L), o1 = org(v, L - 1u);
  const int G8 = (int)G * 8;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t slot = s0 + i / 512u, bit = i % 512u;
    const uint32_t pi = d.meta[slot], r = pi % G3;
    const i3 c = mki((int)(r % G) * 8 + (int)(bit & 7u), (int)((r / G) % G) * 8 + (int)((bit >> 3) & 7u),
                     (int)(r / (G * G)) * 8 + (int)(bit >> 6));
    const uint32_t own = (d.mask[slot * 16u + (bit >> 5)] >> (bit & 31u)) & 1u;
    const i3 gc = mki((o.x * 8 + c.x) * 2 - o1.x * 8, (o.y * 8 + c.y) * 2 - o1.y * 8, (o.z * 8 + c.z) * 2 - o1.z * 8);
    uint32_t cptr = d.nb;
    if (gc.x >= 0 && gc.y >= 0 && gc.z >= 0 && gc.x < G8 && gc.y < G8 && gc.z < G8)
      cptr = d.ptr[(L - 1u) * G3 + ((uint32_t)(gc.z >> 3) * G + (uint32_t)(gc.y >> 3)) * G + (uint32_t)(gc.x >> 3)];
    uint32_t kids = 0;
    if (cptr < d.nb)
      for (uint32_t q = 0; q < 8u; q++) {
        const uint32_t vq = (uint32_t)(((gc.x & 7) + (int)(q & 1u)) + 8 * ((gc.y & 7) + (int)((q >> 1) & 1u))
                                       + 64 * ((gc.z & 7) + (int)(q >> 2)));
        if ((d.mask[cptr * 16u + (vq >> 5)] >> (vq & 31u)) & 1u) kids |= 1u << q;
      }
    if (own == 0u && kids == 0u) continue;
    uint32_t *q0 = d.data + ((size_t)slot * 512u + bit) * DYN_W;
    float acc[13];
#pragma unroll
    for (uint32_t k = 0; k < DYN_W; k++) acc[k] = (float)q0[k] / DYN_FIX;
    for (uint32_t q = 0; q < 8u; q++) {
      if (((kids >> q) & 1u) == 0u) continue;
      const uint32_t vq = (uint32_t)(((gc.x & 7) + (int)(q & 1u)) + 8 * ((gc.y & 7) + (int)((q >> 1) & 1u))
                                     + 64 * ((gc.z & 7) + (int)(q >> 2)));
      const uint32_t *cb = d.data + ((size_t)cptr * 512u + vq) * DYN_W;
#pragma unroll
      for (uint32_t k = 0; k < DYN_W; k++) {
        const float x = L == 1u ? (float)cb[k] / DYN_FIX : __uint_as_float(cb[k]);
        acc[k] += 0.25f * x;
      }
    }
#pragma unroll
    for (uint32_t k = 0; k < DYN_W; k++) q0[k] = __float_as_uint(acc[k]);
    if (own == 0u) atomicOr(&d.mask[slot * 16u + (bit >> 5)], 1u << (bit & 31u));
  }
}

}  // namespace gi

using namespace gi;

cudaError_t gi_launch_dyn_build(const DynDev &d, const VoxDev &v, const SceneDev &s, const float *frame,
                                const float *shadow, uint32_t S, uint32_t layers, uint32_t sm_count, cudaStream_t st) {
  if (d.end <= d.first) return cudaSuccess;   // no dynamic triangles: the layer keeps its state (DynLayer.encode)
  const uint32_t nt = d.end - d.first, G3 = v.G * v.G * v.G, nw = v.levels * G3 / 32u;
  const uint32_t persist = sm_count * 8u;
  GI_TRY(gi_launch(k_dyn_mark, (nt + 255u) / 256u, 256, st, d, v, s));
  if (v.levels > 1u) GI_TRY(gi_launch(k_dyn_parents, (nw - G3 / 32u + 255u) / 256u, 256, st, d, v));
  GI_TRY(gi_launch(k_dyn_alloc, (nw + 255u) / 256u, 256, st, d, v));
  GI_TRY(gi_launch(k_dyn_finalize, 1, 1, st, d, v));
  GI_TRY(gi_launch(k_dyn_clear, persist, 256, st, d));
  GI_TRY(gi_launch(k_dyn_splat, (nt * 32u + 255u) / 256u, 256, st, d, v, s, frame, shadow, S, layers));
  for (uint32_t L = 1; L < v.levels; L++) GI_TRY(gi_launch(k_dyn_resolve, persist, 256, st, d, v, L));
  return cudaGetLastError();
}
