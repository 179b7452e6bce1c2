// Voxel clipmap rebuild on sm_100a (the reference's VOX_STAGES, src/core/voxel.ts:338-620, as CUDA passes).
//
// Differences of form, not of result, from the reference's dispatch graph:
//  * brick pointers are allocated in one fixed order, coarse levels first then pointer index, whether or not the
//    pool holds them all (the reference uses that order only when it overflows, voxel.ts:405-410, and an atomic
//    counter otherwise); voxel attribute bases are an exclusive scan in brick order.  Both are orders the reference
//    can produce; they make the whole state deterministic, so the GPU state equals the oracle's word for word.
//  * the representative-table clear (clearKeys) zeroes every allocated brick in one full-grid pass;
//  * indirect dispatches (writeArgs) become grid-stride loops that read the device-side counts;
//  * the big-triangle passes run one warp per (triangle, level) (markBricksBig) or per chunk of one (voxBitsBig), taken
//    from a queue, instead of one 64-wide workgroup; resolveAttr runs one thread per voxel;
//  * markParents is folded into markBrick: the thread that marks a brick marks its ancestors;
//  * list appends are warp-aggregated atomics.
#include <cuda_runtime.h>

#include "gi_dev.cuh"
#include "gi_internal.h"
#include "gi_scan.cuh"

namespace gi {

struct Tri { f3 a, b, c; uint4 idx; };

// loadTri (voxel.ts:270-276): the triangle of key = instance * key_stride + row, moved by the instance's offset
__device__ __forceinline__ Tri load_tri(const SceneDev &s, uint32_t key) {
  Tri T;
  if (s.items) {
    const uint32_t inst = key / s.key_stride;
    T.idx = s.tri[key - inst * s.key_stride];
    const float4 o4 = s.inst[inst];
    const f3 o = mk(o4.x, o4.y, o4.z);
    T.a = ld3(s.pos[T.idx.x]) + o;
    T.b = ld3(s.pos[T.idx.y]) + o;
    T.c = ld3(s.pos[T.idx.z]) + o;
    return T;
  }
  T.idx = s.tri[key];
  T.a = ld3(s.pos[T.idx.x]);
  T.b = ld3(s.pos[T.idx.y]);
  T.c = ld3(s.pos[T.idx.z]);
  return T;
}
// workAt (voxel.ts:280-288): thread i of a triangle pass -> its key and its first level
__device__ __forceinline__ uint32_t work_at(const SceneDev &s, uint32_t i, uint32_t &first) {
  first = 0;
  if (!s.items) return i;
  uint32_t lo = 0, hi = s.nitems;
  while (hi - lo > 1u) {
    const uint32_t m = (lo + hi) >> 1;
    if (s.items[m].x <= i) lo = m; else hi = m;
  }
  const uint4 b = s.items[lo];
  const uint32_t j = i - b.x;
  const uint32_t row = (b.y & 0x80000000u) ? (b.y & 0x7fffffffu) + j : s.lists[b.y + j];
  first = b.w;
  return b.z * s.key_stride + row;
}

struct Range { i3 lo, n; };

// voxRange (voxel.ts:293-300)
// `bricks`: the cell is a brick (size * 8), else a voxel
__device__ __forceinline__ Range vox_range(const VoxDev &v, const Tri &T, uint32_t L, bool bricks) {
  float cell = bricks ? vox_size(v, L) * 8.0f : vox_size(v, L);
  f3 lo = region_lo(v, L);
  f3 a_ = vmin(vmin(T.a, T.b), T.c), b_ = vmax(vmax(T.a, T.b), T.c);
  int lim = bricks ? v.lim_brick[L] : v.lim_vox[L];   // f2i(G * size * 8 / cell) (vox_derived)
  i3 a = vfloori((a_ - lo) / cell);
  i3 b = vfloori((b_ - lo) / cell);
  a = iclamp3(a, mki(0, 0, 0), mki(lim, lim, lim));
  b = iclamp3(mki(b.x + 1, b.y + 1, b.z + 1), mki(0, 0, 0), mki(lim, lim, lim));
  Range r;
  r.lo = a;
  r.n = mki(max(b.x - a.x, 0), max(b.y - a.y, 0), max(b.z - a.z, 0));
  return r;
}

// finerHolds (voxel.ts:303-307)
__device__ __forceinline__ i3 finer_cell(const VoxDev &v, uint32_t L, i3 c) {
  i3 o = org(v, L), of = org(v, L - 1);
  return mki((o.x * 8 + c.x) * 2 - of.x * 8, (o.y * 8 + c.y) * 2 - of.y * 8, (o.z * 8 + c.z) * 2 - of.z * 8);
}
__device__ __forceinline__ bool finer_holds(const VoxDev &v, uint32_t L, i3 c) {
  if (L == 0) return false;
  i3 f = finer_cell(v, L, c);
  int n = (int)v.G * 8;
  return f.x >= 0 && f.y >= 0 && f.z >= 0 && f.x < n && f.y < n && f.z < n;
}
__device__ __forceinline__ bool finer_holds_range(const VoxDev &v, uint32_t L, Range r, int s) {
  return finer_holds(v, L, mki(r.lo.x * s, r.lo.y * s, r.lo.z * s))
      && finer_holds(v, L, mki((r.lo.x + r.n.x) * s - 1, (r.lo.y + r.n.y) * s - 1, (r.lo.z + r.n.z) * s - 1));
}
// finerBuilt / finerBuiltRange (voxel.ts:314-320); hdr[2] (brick overflow) is final before the voxel passes run
__device__ __forceinline__ bool finer_built(const VoxDev &v, uint32_t L, i3 c, uint32_t brick_overflow) {
  if (!finer_holds(v, L, c)) return false;
  if (brick_overflow == 0) return true;
  i3 f = finer_cell(v, L, c);
  return v.ptr[ptr_index(v, L - 1, mki(f.x >> 3, f.y >> 3, f.z >> 3))] != GI_DROP;
}

__device__ __forceinline__ i3 range_cell(Range r, int q) {
  return mki(r.lo.x + q % r.n.x, r.lo.y + (q / r.n.x) % r.n.y, r.lo.z + q / (r.n.x * r.n.y));
}

// q / n for q, n <= 8 (n >= 1) without a division: (q * ceil(64 / n)) >> 6, exact while q * (n * ceil(64 / n) - 64)
// < 64, which holds for every such pair.
__device__ __forceinline__ int div_small(int q, int n) {
  int m = (int)((0x080A0B0D10162040ull >> (8u * (uint32_t)(n - 1))) & 0xFFull);
  return (q * m) >> 6;
}
// range_cell of a range of at most 8 cells (q < 8)
__device__ __forceinline__ i3 range_cell_small(Range r, int q) {
  int t = div_small(q, r.n.x);        // q / nx
  int z = div_small(t, r.n.y);        // q / (nx * ny)
  return mki(r.lo.x + q - t * r.n.x, r.lo.y + t - z * r.n.y, r.lo.z + z);
}

// Warp-balanced small work: every lane holds one (triangle, level) item of n <= 8 cells (or bricks); the warp's cells
// are dealt out 32 at a time, so a lane with one cell does not idle while another works through eight.  The owner of
// cell g is the first lane whose inclusive prefix exceeds g (a 5-step search over the prefixes with shuffles); its
// triangle, range and count come over with shuffles.  Each (item, cell) pair is visited once, as in the per-lane loop.
struct SmallItem { Tri T; uint32_t t; Range r; int n; };

__device__ __forceinline__ SmallItem shfl_item(const SmallItem &x, int src) {
  SmallItem y;
  y.T.a = mk(__shfl_sync(0xffffffffu, x.T.a.x, src), __shfl_sync(0xffffffffu, x.T.a.y, src), __shfl_sync(0xffffffffu, x.T.a.z, src));
  y.T.b = mk(__shfl_sync(0xffffffffu, x.T.b.x, src), __shfl_sync(0xffffffffu, x.T.b.y, src), __shfl_sync(0xffffffffu, x.T.b.z, src));
  y.T.c = mk(__shfl_sync(0xffffffffu, x.T.c.x, src), __shfl_sync(0xffffffffu, x.T.c.y, src), __shfl_sync(0xffffffffu, x.T.c.z, src));
  y.T.idx = make_uint4(0u, 0u, 0u, __shfl_sync(0xffffffffu, x.T.idx.w, src));
  y.t = __shfl_sync(0xffffffffu, x.t, src);
  y.r.lo = mki(__shfl_sync(0xffffffffu, x.r.lo.x, src), __shfl_sync(0xffffffffu, x.r.lo.y, src), __shfl_sync(0xffffffffu, x.r.lo.z, src));
  y.r.n = mki(__shfl_sync(0xffffffffu, x.r.n.x, src), __shfl_sync(0xffffffffu, x.r.n.y, src), 0);
  y.n = __shfl_sync(0xffffffffu, x.n, src);
  return y;
}

// Calls f(item, q) for every lane's item and q < item.n (mine = the lane's count, 0 for none); all lanes call it.
template <class F>
__device__ __forceinline__ void warp_deal(const SmallItem &it, uint32_t mine, F f) {
  const uint32_t lane = threadIdx.x & 31u;
  uint32_t incl = mine;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, incl, d);
    if (lane >= (uint32_t)d) incl += y;
  }
  const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
  for (uint32_t base = 0; base < total; base += 32u) {
    uint32_t g = base + lane, o = 0;
#pragma unroll
    for (uint32_t bit = 16; bit >= 1; bit >>= 1) {
      uint32_t val = __shfl_sync(0xffffffffu, incl, (int)(o + bit - 1u));
      if (val <= g) o += bit;
    }
    o = min(o, 31u);
    SmallItem w = shfl_item(it, (int)o);
    uint32_t start = __shfl_sync(0xffffffffu, incl - mine, (int)o);
    if (g < total) f(w, (int)(g - start));
  }
}

// markBrick (voxel.ts:347), read before the atomic, with markParents (voxel.ts:390-403) folded in: the thread whose
// atomic turned brick b of level L from empty to marked walks its parents up the levels, marking each, and stops at
// the first parent outside its level's window or already marked.  An already marked parent was turned by another
// thread, which walks the same chain above it, so the marked set is the closure markParents gives.
__device__ __forceinline__ void mark_brick(const VoxDev &v, uint32_t L, i3 b) {
  uint32_t i = ptr_index(v, L, b);
  if (v.ptr[i] != GI_EMPTY || atomicMin(&v.ptr[i], GI_MARK) != GI_EMPTY) return;
  const int G = (int)v.G;
  const i3 o = org(v, L);
  i3 w = mki(o.x + b.x, o.y + b.y, o.z + b.z);
  for (L++; L < v.levels; L++) {
    w = mki(w.x >> 1, w.y >> 1, w.z >> 1);
    const i3 ol = org(v, L);
    const i3 p = mki(w.x - ol.x, w.y - ol.y, w.z - ol.z);
    if (p.x < 0 || p.y < 0 || p.z < 0 || p.x >= G || p.y >= G || p.z >= G) return;
    i = ptr_index(v, L, p);
    if (v.ptr[i] != GI_EMPTY || atomicMin(&v.ptr[i], GI_MARK) != GI_EMPTY) return;
  }
}

// markRange body for one brick j of the range (voxel.ts:348-358)
__device__ __forceinline__ void mark_one(const VoxDev &v, const Tri &T, uint32_t L, Range r, uint32_t n, uint32_t j) {
  i3 b = n <= 8u ? range_cell_small(r, (int)j) : range_cell(r, (int)j);
  if (finer_holds(v, L, mki(b.x * 8, b.y * 8, b.z * 8)) && finer_holds(v, L, mki(b.x * 8 + 7, b.y * 8 + 7, b.z * 8 + 7))) return;
  float bs = vox_size(v, L) * 8.0f;
  f3 c = region_lo(v, L) + adds(vi2f(b), 0.5f) * bs;
  float hh = 0.5f * bs * 1.0001f;
  if (n == 1u || tri_box(c, mk(hh, hh, hh), T.a, T.b, T.c)) mark_brick(v, L, b);
}

// clear (voxel.ts:338-344)
__global__ void k_clear(VoxDev v) {
  grid_dep_wait();
  uint32_t n = v.levels * v.G * v.G * v.G, nl = v.scan_cap + 1u;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n || i < GI_HDR || i < nl; i += gridDim.x * blockDim.x) {
    if (i < GI_HDR) v.hdr[i] = 0u;
    if (i < 4u) v.work[i] = 0u;
    if (i < n) v.ptr[i] = GI_EMPTY;
    if (i < nl) v.look[i] = 0ull;   // the brick allocation's chained scan
  }
}

// markBricks (voxel.ts:359-376): one thread per triangle; every lane walks the same levels so that the list appends
// are warp-aggregated.
__global__ void __launch_bounds__(256, 4) k_mark_bricks(VoxDev v, SceneDev s) {
  grid_dep_wait();
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  bool live = i < s.threads;
  uint32_t t = 0, L0 = 0;
  Tri T;
  T.a = T.b = T.c = mk(0.0f, 0.0f, 0.0f);
  T.idx = make_uint4(0u, 0u, 0u, 0u);
  if (live) { t = work_at(s, i, L0); T = load_tri(s, t); }
  for (uint32_t L = 0; L < v.levels; L++) {
    bool big = false;
    Range r;
    r.lo = r.n = mki(0, 0, 0);
    int n = 0;
    if (live && L >= L0) {
      r = vox_range(v, T, L, true);
      n = r.n.x * r.n.y * r.n.z;
      if (n != 0 && !finer_holds_range(v, L, r, 8)) big = n > 8;
      else n = 0;
    }
    uint32_t k = warp_append(&v.hdr[24 + L], big);
    if (big) {
      if (k < v.big_cap) v.big[(8u + L) * v.big_cap + k] = t; else atomicAdd(&v.hdr[3], 1u);
    }
    SmallItem it;
    it.T = T; it.t = t; it.r = r; it.n = n;
    warp_deal(it, (!big && n > 0) ? (uint32_t)n : 0u, [&](const SmallItem &w, int j) {
      mark_one(v, w.T, L, w.r, (uint32_t)w.n, (uint32_t)j);
    });
  }
}

// The list entry of global item w among the levels' lists starting at segment seg0 (markBricksBig / voxelizeBig
// level walk, voxel.ts:378-384).  Returns false past the end.
__device__ __forceinline__ bool big_item(const VoxDev &v, uint32_t seg0, uint32_t hdr0, uint32_t w, uint32_t &L, uint32_t &t) {
  uint32_t k = w;
  for (L = 0; L < v.levels; L++) {
    uint32_t n = min(v.hdr[hdr0 + L], v.big_cap);
    if (k < n) { t = v.big[(seg0 + L) * v.big_cap + k]; return true; }
    k -= n;
  }
  return false;
}

// markBricksBig (voxel.ts:377-387): one warp per big (triangle, level), lanes over the range's bricks.
__global__ void __launch_bounds__(256, 4) k_mark_bricks_big(VoxDev v, SceneDev s) {
  grid_dep_wait();
  uint32_t lane = threadIdx.x & 31u;
  for (;;) {
    uint32_t w = 0;
    if (lane == 0) w = atomicAdd(&v.work[0], 1u);   // warps take items from a queue: long items do not stall others
    w = __shfl_sync(0xffffffffu, w, 0);
    uint32_t L, t;
    if (!big_item(v, 8u, 24u, w, L, t)) break;
    Tri T = load_tri(s, t);
    Range r = vox_range(v, T, L, true);
    uint32_t n = (uint32_t)(r.n.x * r.n.y * r.n.z);
    for (uint32_t j = lane; j < n; j += 32u) mark_one(v, T, L, r, n, j);
  }
}

// ---- ordered allocation of the marked bricks (countMarks / scanMarks / allocBricks, voxel.ts:411-470) ---------------
// Order space o in [0, levels * G^3): level levels-1 first, pointer index within a level.
// The ordered brick allocation takes 256 * k pointer entries per block, k per thread: k = 1 unless the block sums
// would not fit the scan buffer (alloc_per_thread)

__device__ __forceinline__ uint32_t order_to_ptr(uint32_t o, uint32_t per, uint32_t NL) {
  return (NL - 1u - o / per) * per + o % per;
}

// allocBricks (voxel.ts:411-470: countMarks, scanMarks, allocBricks) in the fixed order, one pass: each block takes
// 256 * kpt consecutive entries of the order space, kpt per thread.
__global__ void __launch_bounds__(256) k_alloc_bricks(VoxDev v, uint32_t kpt, uint32_t nblocks) {
  grid_dep_wait();
  uint32_t per = v.G * v.G * v.G, NL = v.levels, n = NL * per, G = v.G;
  uint32_t blk = chain_ticket(v.look);
  uint32_t o0 = blk * 256u * kpt;
  uint32_t flags = 0, c = 0;
  for (uint32_t k = 0; k < kpt; k++) {
    uint32_t o = o0 + threadIdx.x * kpt + k;
    bool m = o < n && v.ptr[order_to_ptr(o, per, NL)] == GI_MARK;
    flags |= (m ? 1u : 0u) << k;
    c += m ? 1u : 0u;
  }
  uint32_t tot;
  uint32_t ex = block_scan_256(c, &tot);
  __shared__ uint32_t s_pre;
  if (threadIdx.x == 0) {
    uint32_t pre = chain_prefix(v.look, blk, tot, v.hdr, v.scan_hold);
    s_pre = pre;
    if (blk == nblocks - 1u) { v.hdr[0] = pre + tot; v.hdr[5] = pre + tot; }
  }
  __syncthreads();
  ex += s_pre;
  for (uint32_t k = 0; k < kpt; k++) {
    if (!((flags >> k) & 1u)) continue;
    uint32_t o = o0 + threadIdx.x * kpt + k;
    uint32_t i = order_to_ptr(o, per, NL);
    uint32_t idx = ex++;
    if (idx >= v.max_bricks) { v.ptr[i] = GI_DROP; atomicAdd(&v.hdr[2], 1u); continue; }
    uint32_t L = i / per, r = i % per;
    atomicAdd(&v.hdr[8 + L], 1u);
    v.ptr[i] = idx;
    v.base[idx] = 0u;
    v.code[idx] = (L << 27) | ((r % G) << 18) | (((r / G) % G) << 9) | (r / (G * G));
  }
}

// The rest of the brick init and clearKeys (voxel.ts:467, :471-474): zero the occupancy (64 B) and representatives
// (2 KB) of every allocated brick, over the whole grid.
__global__ void __launch_bounds__(256) k_init_bricks(VoxDev v) {
  grid_dep_wait();
  uint32_t nb = min(v.hdr[0], v.max_bricks);
  uint4 z = make_uint4(0u, 0u, 0u, 0u);
  uint4 *occ = reinterpret_cast<uint4 *>(v.occ), *rep = reinterpret_cast<uint4 *>(v.rep);
  if (blockIdx.x == 0 && threadIdx.x == 0) v.work[1] = 0u;   // the voxBitsBig item counter
  for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < nb * 132u; q += gridDim.x * blockDim.x) {
    if (q < nb * 4u) occ[q] = z;
    else rep[q - nb * 4u] = z;
  }
}

// closestBary (voxel.ts:250-267)
__device__ __forceinline__ f3 closest_bary(f3 p, f3 a, f3 b, f3 c) {
  f3 ab = b - a, ac = c - a, ap = p - a;
  float d1 = dot(ab, ap), d2 = dot(ac, ap);
  if (d1 <= 0.0f && d2 <= 0.0f) return mk(1.0f, 0.0f, 0.0f);
  f3 bp = p - b;
  float d3 = dot(ab, bp), d4 = dot(ac, bp);
  if (d3 >= 0.0f && d4 <= d3) return mk(0.0f, 1.0f, 0.0f);
  float vc = d1 * d4 - d3 * d2;
  if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) { float w = d1 / (d1 - d3); return mk(1.0f - w, w, 0.0f); }
  f3 cp = p - c;
  float d5 = dot(ab, cp), d6 = dot(ac, cp);
  if (d6 >= 0.0f && d5 <= d6) return mk(0.0f, 0.0f, 1.0f);
  float vb = d5 * d2 - d1 * d6;
  if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) { float w = d2 / (d2 - d6); return mk(1.0f - w, 0.0f, w); }
  float va = d3 * d6 - d5 * d4;
  if (va <= 0.0f && (d4 - d3) >= 0.0f && (d5 - d6) >= 0.0f) {
    float w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
    return mk(0.0f, 1.0f - w, w);
  }
  float dn = 1.0f / (va + vb + vc);
  float vv = vb * dn, ww = vc * dn;
  return mk(1.0f - vv - ww, vv, ww);
}

// surfaceAt's alpha test (voxel.ts:325-332): a masked material keeps the cell when its alpha — the base colour texture
// at level 3 + L at the voxel centre's closest point on the triangle, times the factor; the factor alone untextured —
// reaches the cutoff
__device__ __forceinline__ bool alpha_passes(const SceneDev &s, const Tri &T, f3 p, uint32_t L) {
  const gi_material &m = s.mats[T.idx.w];
  if ((m.flags & 1u) == 0u) return true;
  float a = m.base_color[3];
  const uint32_t layer = tex_layer_of(s, m);
  if (layer) {
    const f3 w = closest_bary(p, T.a, T.b, T.c);
    const float2 uv = tri_uv(s, T.idx, w.x, w.y, w.z);
    a = tex_sample(s, layer, uv.x, uv.y, 3u + L).w * m.base_color[3];
  }
  return !(a < m.alpha_cutoff);
}

// voxelizeOne (voxel.ts:476-490)

__device__ __forceinline__ void voxelize_one(const VoxDev &v, const SceneDev &s, const Tri &T, uint32_t t, uint32_t L,
                                             i3 c, bool single, uint32_t brick_overflow) {
  if (finer_built(v, L, c, brick_overflow)) return;
  const uint32_t ptr = v.ptr[ptr_index(v, L, mki(c.x >> 3, c.y >> 3, c.z >> 3))];   // in flight during the box test
  float vs = vox_size(v, L);
  f3 p = region_lo(v, L) + adds(vi2f(c), 0.5f) * vs;
  float hh = 0.5f * vs * 1.0001f;
  if (!single && !tri_box(p, mk(hh, hh, hh), T.a, T.b, T.c)) return;
  if (ptr >= GI_MARK) return;
  uint32_t bit = (uint32_t)((c.x & 7) + 8 * (c.y & 7) + 64 * (c.z & 7));
  if (!alpha_passes(s, T, p, L)) return;
  uint32_t wi = ptr * 16u + (bit >> 5);
  uint32_t msk = 1u << (bit & 31u);
  uint32_t ri = ptr * 512u + bit;
  // unconditional reductions (their results unused): the warp does not wait for a read of the word first
  atomicOr(&v.occ[wi], msk);
  atomicMax(&v.rep[ri], t + 1u);
}

// The big items' work for k_vox_bits_big: every big (triangle, level) of voxBits is cut into chunks of
// 2^chunk_log2 cells (a wall triangle clipped to a window covers ~10^4 cells; one warp per triangle left one warp working
// long after the rest).  The warp reserves its items' chunks with one atomic, item after item; the item's first chunk
// goes to cpre[slot] and, below citem_cap, the slot of every chunk to citem (written by the whole warp).  An item with
// chunks at or past citem_cap is listed for k_vox_bits_big to walk from there to its end with one warp.  All lanes call
// it (nch = 0: no item).  Which chunk numbers an item gets does not change the voxels: the occupancy and
// representative updates are ORs and maxima.
__device__ __forceinline__ void big_chunks(const VoxDev &v, uint32_t slot, uint32_t nch) {
  const uint32_t lane = threadIdx.x & 31u;
  uint32_t incl = nch;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, d);
    if (lane >= (uint32_t)d) incl += y;
  }
  const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
  if (total == 0u) return;
  uint32_t base = 0;
  if (lane == 31u) base = atomicAdd(&v.work[2], total);
  base = __shfl_sync(0xffffffffu, base, 31);
  const uint32_t first = base + incl - nch;
  if (nch != 0u) {
    v.cpre[slot] = first;
    if (first + nch > v.citem_cap) v.big[8u * v.big_cap + atomicAdd(&v.work[3], 1u)] = slot;
  }
  for (uint32_t m = __ballot_sync(0xffffffffu, nch != 0u); m != 0u; m &= m - 1u) {
    const int src = __ffs(m) - 1;
    const uint32_t f = __shfl_sync(0xffffffffu, first, src), c = __shfl_sync(0xffffffffu, nch, src);
    const uint32_t sl = __shfl_sync(0xffffffffu, slot, src);
    for (uint32_t j = lane; j < c && f + j < v.citem_cap; j += 32u) v.citem[f + j] = sl;
  }
}

// voxBits (voxel.ts:492-513)
__global__ void __launch_bounds__(256, 4) k_vox_bits(VoxDev v, SceneDev s) {
  grid_dep_wait();
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  bool live = i < s.threads;
  uint32_t bo = v.hdr[2];
  uint32_t t = 0, L0 = 0;
  Tri T;
  T.a = T.b = T.c = mk(0.0f, 0.0f, 0.0f);
  T.idx = make_uint4(0u, 0u, 0u, 0u);
  if (live) { t = work_at(s, i, L0); T = load_tri(s, t); }
  for (uint32_t L = 0; L < v.levels; L++) {
    bool big = false;
    Range r;
    r.lo = r.n = mki(0, 0, 0);
    int n = 0;
    if (live && L >= L0) {
      r = vox_range(v, T, L, false);
      n = r.n.x * r.n.y * r.n.z;
      bool skip = n == 0 || (bo == 0u && finer_holds_range(v, L, r, 1));
      if (skip) n = 0;
      else big = (uint32_t)n > GI_BIG_SMALL;
    }
    uint32_t k = warp_append(&v.hdr[16 + L], big);
    uint32_t slot = 0, nch = 0;
    if (big) {
      if (k < v.big_cap) {
        slot = L * v.big_cap + k;
        v.big[slot] = t;
        nch = ((uint32_t)n + (1u << v.chunk_log2) - 1u) >> v.chunk_log2;
      } else {
        atomicAdd(&v.hdr[3], 1u);
      }
    }
    big_chunks(v, slot, nch);
    SmallItem it;
    it.T = T; it.t = t; it.r = r; it.n = n;
    warp_deal(it, (!big && n > 0) ? (uint32_t)n : 0u, [&](const SmallItem &w, int q) {
      voxelize_one(v, s, w.T, w.t, L, range_cell_small(w.r, q), w.n == 1, bo);
    });
  }
}

// voxelizeOne's tests (voxel.ts:477-485) without the writes: true and the occupancy word / bit / representative slot
// when the voxel takes the triangle.
__device__ __forceinline__ bool voxel_takes(const VoxDev &v, const SceneDev &s, const Tri &T, uint32_t L, i3 c,
                                            uint32_t brick_overflow, uint32_t &wi, uint32_t &msk, uint32_t &ri) {
  if (finer_built(v, L, c, brick_overflow)) return false;
  const uint32_t ptr = v.ptr[ptr_index(v, L, mki(c.x >> 3, c.y >> 3, c.z >> 3))];   // in flight during the box test
  float vs = vox_size(v, L);
  f3 p = region_lo(v, L) + adds(vi2f(c), 0.5f) * vs;
  float hh = 0.5f * vs * 1.0001f;
  if (!tri_box(p, mk(hh, hh, hh), T.a, T.b, T.c)) return false;
  if (ptr >= GI_MARK) return false;
  if (!alpha_passes(s, T, p, L)) return false;
  uint32_t bit = (uint32_t)((c.x & 7) + 8 * (c.y & 7) + 64 * (c.z & 7));
  wi = ptr * 16u + (bit >> 5);
  msk = 1u << (bit & 31u);
  ri = ptr * 512u + bit;
  return true;
}

// voxBitsBig (voxel.ts:515-534), balanced: one warp per chunk of a big item, taken from a queue (big_chunks cut the
// items); then one warp per item listed with chunks past the table, from its first untabulated chunk to its end.  The
// lanes' occupancy bits are ORed per word inside the warp (neighbouring cells share a word), one atomic per word.
__global__ void __launch_bounds__(256, 4) k_vox_bits_big(VoxDev v, SceneDev s) {
  grid_dep_wait();
  uint32_t lane = threadIdx.x & 31u;
  uint32_t bo = v.hdr[2];
  const uint32_t tab = min(v.work[2], v.citem_cap);   // chunks found through the table
  const uint32_t work = tab + v.work[3];               // + the listed items
  // the attribute allocation's chained scan (the brick allocation's is done)
  for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q <= v.scan_cap; q += gridDim.x * blockDim.x) v.look[q] = 0ull;
  for (;;) {
    uint32_t ch = 0;
    if (lane == 0) ch = atomicAdd(&v.work[1], 1u);
    ch = __shfl_sync(0xffffffffu, ch, 0);
    if (ch >= work) break;
    const bool whole = ch >= tab;
    const uint32_t slot = whole ? v.big[8u * v.big_cap + (ch - tab)] : v.citem[ch];
    const uint32_t first = v.cpre[slot];
    const uint32_t part = whole ? max(first, v.citem_cap) - first : ch - first;
    const uint32_t L = slot / v.big_cap, t = v.big[slot];
    Tri T = load_tri(s, t);
    Range r = vox_range(v, T, L, false);
    int n = r.n.x * r.n.y * r.n.z;
    int q_end = whole ? n : min(n, (int)((part + 1u) << v.chunk_log2));
    // the lane's cell, then 32 cells further in range order per step: 32 = dz * nx * ny + dy * nx + dx
    int q = (int)(part << v.chunk_log2) + (int)lane;
    i3 cell = range_cell(r, q);
    const int nxy = r.n.x * r.n.y, dz = 32 / nxy, dy = (32 - dz * nxy) / r.n.x, dx = 32 - dz * nxy - dy * r.n.x;
    for (; q - (int)lane < q_end; q += 32) {
      uint32_t wi = 0xffffffffu, msk = 0u, ri = 0u;
      bool ok = q < q_end && voxel_takes(v, s, T, L, cell, bo, wi, msk, ri);
      cell = mki(cell.x + dx, cell.y + dy, cell.z + dz);
      if (cell.x >= r.lo.x + r.n.x) { cell.x -= r.n.x; cell.y++; }
      if (cell.y >= r.lo.y + r.n.y) { cell.y -= r.n.y; cell.z++; }
      uint32_t any = __ballot_sync(0xffffffffu, ok);
      if (any == 0u) continue;
      uint32_t grp = __match_any_sync(0xffffffffu, ok ? wi : 0xffffffffu);
      uint32_t m = __reduce_or_sync(grp, msk);
      if (ok) {
        if ((uint32_t)(__ffs(grp) - 1) == lane) atomicOr(&v.occ[wi], m);
        atomicMax(&v.rep[ri], t + 1u);
      }
    }
  }
}

// reduce (voxel.ts:540-577) for every level at once.  The reference runs reduce(L) for L = 1 .. levels-1 in turn, each
// ORing the occupancy of level L-1 (its own voxels and what reduce(L-1) put there) into level L and taking the maximum
// of the representatives, through the parent brick when it is allocated.  OR and max are associative, so level L ends
// with its own voxels and those of every finer level l whose parent bricks l+1 .. L are all allocated: here one thread
// per occupancy word of a level 0 .. levels-2 brick walks up the levels, the word's 8 x 4 cells becoming 4 x 2 parent
// cells, then 2 x 1, then 1, and stops at the first level without a brick.  Same final state, one launch.
__global__ void __launch_bounds__(256) k_reduce(VoxDev v) {
  grid_dep_wait();
  const uint32_t NL = v.levels, nb = min(v.hdr[0], v.max_bricks);
  const uint32_t first = v.hdr[8 + NL - 1u];   // bricks are allocated coarse levels first: the finer ones follow
  const int lim = (int)v.G * 8;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < (nb - first) * 16u; i += gridDim.x * blockDim.x) {
    uint32_t ptr = first + (i >> 4), w = i & 15u;
    uint32_t word = v.occ[ptr * 16u + w];
    if (word == 0u) continue;
    uint32_t code = v.code[ptr];
    uint32_t l = code >> 27;
    i3 b = mki((int)((code >> 18) & 511u), (int)((code >> 9) & 511u), (int)(code & 511u));
    // the word's first cell in level-l cells from the world origin
    i3 oc = org(v, l);
    i3 wc = mki(oc.x * 8 + b.x * 8, oc.y * 8 + b.y * 8 + (int)((w & 1u) * 4u), oc.z * 8 + b.z * 8 + (int)(w >> 1));
    // 4 x 2 parent cells: occupancy (bit px + 4 py) and representatives; the word's 32 representatives in 8
    // independent 128-bit loads; bit k = x + 8 y of the word, parent (x/2, y/2)
    uint32_t lo[4] = {0, 0, 0, 0}, hi[4] = {0, 0, 0, 0}, m1 = 0;
    const uint4 *rp = reinterpret_cast<const uint4 *>(v.rep + ptr * 512u + w * 32u);
    uint4 rq[8];
#pragma unroll
    for (int q = 0; q < 8; q++) rq[q] = rp[q];
#pragma unroll
    for (int q = 0; q < 8; q++) {
      uint32_t b4 = (word >> (4 * q)) & 15u;
      uint32_t px = 2u * (uint32_t)(q & 1);
      uint32_t a = max((b4 & 1u) ? rq[q].x : 0u, (b4 & 2u) ? rq[q].y : 0u);
      uint32_t c = max((b4 & 4u) ? rq[q].z : 0u, (b4 & 8u) ? rq[q].w : 0u);
      if (q < 4) { lo[px] = max(lo[px], a); lo[px + 1u] = max(lo[px + 1u], c); }
      else { hi[px] = max(hi[px], a); hi[px + 1u] = max(hi[px + 1u], c); }
      uint32_t pa = ((b4 & 3u) ? 1u : 0u) | ((b4 & 12u) ? 2u : 0u);   // parents px, px + 1 of this row
      m1 |= pa << (px + (q < 4 ? 0u : 4u));
    }
    for (uint32_t L = l + 1u, s = 1u; L < NL; L++, s++) {
      wc = mki(wc.x >> 1, wc.y >> 1, wc.z >> 1);
      i3 ol = org(v, L);
      i3 pc = mki(wc.x - ol.x * 8, wc.y - ol.y * 8, wc.z - ol.z * 8);
      if (pc.x < 0 || pc.y < 0 || pc.z < 0 || pc.x >= lim || pc.y >= lim || pc.z >= lim) break;
      uint32_t pptr = v.ptr[ptr_index(v, L, mki(pc.x >> 3, pc.y >> 3, pc.z >> 3))];
      if (pptr >= GI_MARK) break;
      uint32_t pbit0 = (uint32_t)((pc.x & 7) + 8 * (pc.y & 7) + 64 * (pc.z & 7));
      if (s == 2u) {   // 4 x 2 -> 2 x 1
        lo[0] = max(max(lo[0], lo[1]), max(hi[0], hi[1]));
        lo[1] = max(max(lo[2], lo[3]), max(hi[2], hi[3]));
        m1 = ((m1 & 0x33u) ? 1u : 0u) | ((m1 & 0xCCu) ? 2u : 0u);
      } else if (s == 3u) {   // 2 x 1 -> 1
        lo[0] = max(lo[0], lo[1]);
        m1 = m1 ? 1u : 0u;
      }
      const uint32_t nx = s == 1u ? 4u : (s == 2u ? 2u : 1u), ny = s == 1u ? 2u : 1u;
      uint32_t mask = 0;
      for (uint32_t py = 0; py < ny; py++)
        for (uint32_t px = 0; px < nx; px++)
          if ((m1 >> (px + nx * py)) & 1u) mask |= 1u << ((pbit0 + px + 8u * py) & 31u);
      uint32_t wi = pptr * 16u + (pbit0 >> 5);
      if ((v.occ[wi] & mask) != mask) atomicOr(&v.occ[wi], mask);
      for (uint32_t py = 0; py < ny; py++)
        for (uint32_t px = 0; px < nx; px++) {
          uint32_t rv = py == 0u ? lo[px] : hi[px];
          if (rv == 0u) continue;
          uint32_t ri = pptr * 512u + pbit0 + px + 8u * py;
          if (v.rep[ri] < rv) atomicMax(&v.rep[ri], rv);
        }
    }
  }
}

// ---- allocVoxels (voxel.ts:579-588): attribute bases as an exclusive scan of the bricks' popcounts -------------------
constexpr uint32_t VOX_CHUNK = 256;   // bricks per block

__device__ __forceinline__ uint32_t brick_pop(const VoxDev &v, uint32_t b) {
  const uint4 *o = reinterpret_cast<const uint4 *>(v.occ) + b * 4u;
  uint32_t n = 0;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    uint4 q = o[k];
    n += __popc(q.x) + __popc(q.y) + __popc(q.z) + __popc(q.w);
  }
  return n;
}

// allocVoxels in one pass: each block takes 256 bricks (chained scan of their popcounts).
__global__ void __launch_bounds__(256) k_alloc_voxels(VoxDev v, uint32_t nblocks) {
  grid_dep_wait();
  uint32_t nb = min(v.hdr[0], v.max_bricks);
  uint32_t blk = chain_ticket(v.look);
  // the grid covers the pool; only the parts that hold bricks take part in the scan (a part waits on smaller tickets
  // only, so the parts past the bricks can leave at once)
  const uint32_t used = max((nb + VOX_CHUNK - 1u) / VOX_CHUNK, 1u);
  if (blk >= used) return;
  nblocks = used;
  uint32_t b = blk * VOX_CHUNK + threadIdx.x;
  uint32_t c = b < nb ? brick_pop(v, b) : 0u;
  uint32_t tot;
  uint32_t ex = block_scan_256(c, &tot);
  __shared__ uint32_t s_pre;
  if (threadIdx.x == 0) s_pre = chain_prefix(v.look, blk, tot, v.hdr);
  __syncthreads();
  uint32_t first = ex + s_pre;
  if (b < nb) {
    if (first + c > v.max_voxels) { v.base[b] = GI_EMPTY; atomicAdd(&v.hdr[4], 1u); }
    else v.base[b] = first;
    v.vpre[b] = first;
    if (b == nb - 1u) v.vpre[nb] = first + c;
  }
  if (nb == 0u && b == 0u) v.vpre[0] = 0u;
  if (blk == nblocks - 1u && threadIdx.x == 255u) v.hdr[1] = first + c;
}


// resolveAttr (voxel.ts:596-620): one thread per voxel of the attribute pool (voxel ai of brick b is rank
// ai - vpre[b] of b's occupancy), so every occupied voxel is resolved in parallel and the attribute writes are
// contiguous.  With a shadow map the same thread runs voxSun (the reference's next stage) on what it stored.
__global__ void __launch_bounds__(256) k_resolve_attr(VoxDev v, SceneDev s) {
  grid_dep_wait();
  uint32_t nb = min(v.hdr[0], v.max_bricks);
  uint32_t nv = nb ? min(v.vpre[nb], v.max_voxels) : 0u;
  for (uint32_t ai = blockIdx.x * blockDim.x + threadIdx.x; ai < nv; ai += gridDim.x * blockDim.x) {
    uint32_t lo = 0, hi = nb;   // the last brick b with vpre[b] <= ai
    while (hi - lo > 1u) {
      uint32_t m = (lo + hi) >> 1;
      if (v.vpre[m] <= ai) lo = m; else hi = m;
    }
    uint32_t ptr = lo;
    if (v.base[ptr] == GI_EMPTY) continue;   // past the voxel pool: no attributes (voxel.ts:586)
    uint32_t r = ai - v.vpre[ptr];
    const uint4 *o4 = reinterpret_cast<const uint4 *>(v.occ) + ptr * 4u;
    uint32_t bit = 0;
#pragma unroll
    for (int q = 0; q < 4; q++) {
      uint4 o = o4[q];
      uint32_t ws[4] = {o.x, o.y, o.z, o.w};
#pragma unroll
      for (int j = 0; j < 4; j++) {
        uint32_t pc = __popc(ws[j]);
        if (r < pc && bit == 0u) {
          uint32_t wd = ws[j];
          bit = (uint32_t)(q * 4 + j) * 32u + nth_set_bit(wd, r) + 1u;   // + 1: found
        }
        if (bit == 0u) r -= pc;
      }
    }
    if (bit == 0u) continue;   // rank past the brick's voxels: only after a scan that gave up (header word 6)
    bit -= 1u;
    uint32_t code = v.code[ptr];
    uint32_t L = code >> 27;
    i3 b = mki((int)((code >> 18) & 511u), (int)((code >> 9) & 511u), (int)(code & 511u));
    i3 c = mki(b.x * 8 + (int)(bit & 7u), b.y * 8 + (int)((bit >> 3) & 7u), b.z * 8 + (int)(bit >> 6));
    f3 p = region_lo(v, L) + adds(vi2f(c), 0.5f) * vox_size(v, L);
    uint32_t rv = v.rep[ptr * 512u + bit];
    if (rv == 0u || rv > s.key_limit) {   // no representative (cannot happen for a set bit): no attributes
      v.attr[ai] = make_uint4(0u, 0u, 0u, 0u); v.plane[ai] = 0.0f;
      v.sunvis[ai] = v.shadow ? voxel_sun(v.sun_frame, v.shadow, v.shadow_size, v.shadow_layers, p, vox_size(v, L), 0u,
                                          0.0f) : 1.0f;
      continue;
    }
    Tri T = load_tri(s, rv - 1u);
    const gi_material &m = s.mats[T.idx.w];
    // surfaceAt(..., wantAttr = true) (voxel.ts:325-336), untextured
    f3 wb = closest_bary(p, T.a, T.b, T.c);
    f3 n0 = ld3(s.nrm[T.idx.x]), n1 = ld3(s.nrm[T.idx.y]), n2 = ld3(s.nrm[T.idx.z]);
    f3 n = (n0 * wb.x + n1 * wb.y) + n2 * wb.z;
    if (!(dot(n, n) > 1e-12f)) n = cross(T.b - T.a, T.c - T.a);
    n = normalize3(n);
    f3 q = (T.a * wb.x + T.b * wb.y) + T.c * wb.z;
    float toon = (m.flags & 4u) ? 1.0f : 0.0f;
    // octEnc (voxel.ts:590-594)
    float sa = fabsf(n.x) + fabsf(n.y) + fabsf(n.z);
    float ox = n.x / sa, oy = n.y / sa;
    if (n.z < 0.0f) {
      float tx = ox, ty = oy;
      ox = (1.0f - fabsf(ty)) * (tx >= 0.0f ? 1.0f : -1.0f);
      oy = (1.0f - fabsf(tx)) * (ty >= 0.0f ? 1.0f : -1.0f);
    }
    uint4 rec;
    // the albedo: the base colour texture at level 3 + L at the closest point, times the factor (surfaceAt)
    float ar = m.base_color[0], ag = m.base_color[1], ab = m.base_color[2];
    const uint32_t layer = tex_layer_of(s, m);
    if (layer) {
      const float2 uv = tri_uv(s, T.idx, wb.x, wb.y, wb.z);
      const float4 t = tex_sample(s, layer, uv.x, uv.y, 3u + L);
      ar = t.x * m.base_color[0]; ag = t.y * m.base_color[1]; ab = t.z * m.base_color[2];
    }
    rec.x = pack4x8unorm(ar, ag, ab, toon);
    rec.y = pack2x16snorm(ox, oy);
    rec.z = (uint32_t)f2h(m.emissive[0]) | ((uint32_t)f2h(m.emissive[1]) << 16);
    rec.w = (uint32_t)f2h(m.emissive[2]);
    v.attr[ai] = rec;
    float pl = dot(n, q - p);
    v.plane[ai] = pl;
    // voxSun (voxel.ts:633-671) from the values just stored
    v.sunvis[ai] = v.shadow ? voxel_sun(v.sun_frame, v.shadow, v.shadow_size, v.shadow_layers, p, vox_size(v, L), rec.y,
                                        pl) : 1.0f;
  }
}

}  // namespace gi

using namespace gi;

// The rebuild's launches (VOX_STAGES minus sun, voxel.ts:708), stream-ordered.
cudaError_t gi_launch_vox_build(const VoxDev &v, const SceneDev &s, uint32_t sm_count, cudaStream_t st) {
  uint32_t per = v.G * v.G * v.G, nptr = v.levels * per;
  uint32_t persist = sm_count * v.blocks;   // blocks of 256 threads per SM for the grid-stride passes (default 8)
  GI_TRY(gi_launch(k_clear, min((nptr + 255u) / 256u + 1u, persist), 256, st, v));
  uint32_t tb = (s.threads + 255u) / 256u;   // threads of the triangle passes (the work items' triangles)
  if (tb) GI_TRY(gi_launch(k_mark_bricks, tb, 256, st, v, s));
  GI_TRY(gi_launch(k_mark_bricks_big, persist, 256, st, v, s));
  uint32_t kpt = 1;
  while ((nptr + 256u * kpt - 1u) / (256u * kpt) > v.scan_cap && kpt < 32u) kpt *= 2u;
  uint32_t ab = (nptr + 256u * kpt - 1u) / (256u * kpt);
  GI_TRY(gi_launch(k_alloc_bricks, ab, 256, st, v, kpt, ab));
  GI_TRY(gi_launch(k_init_bricks, persist, 256, st, v));
  if (tb) GI_TRY(gi_launch(k_vox_bits, tb, 256, st, v, s));
  GI_TRY(gi_launch(k_vox_bits_big, persist, 256, st, v, s));
  if (v.levels > 1) GI_TRY(gi_launch(k_reduce, persist, 256, st, v));
  uint32_t vb = (v.max_bricks + VOX_CHUNK - 1u) / VOX_CHUNK;
  GI_TRY(gi_launch(k_alloc_voxels, vb, 256, st, v, vb));
  GI_TRY(gi_launch(k_resolve_attr, persist, 256, st, v, s));
  return cudaGetLastError();
}
