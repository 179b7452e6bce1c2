// Headless G-buffer on sm_100a: reversed-Z depth (depth32float) and the rgba16float shading normal that the
// reference's raster pass writes (src/core/gbuffer.ts:82-103), defined here as one primary-ray sample per pixel
// centre (there is no graphics pipeline on a compute-only box):
//   ray    origin = eye, direction = worldAt(px, 1) - eye (the point on the near plane, frame.ts:22-26)
//   hit    Moller-Trumbore against the triangles whose near-clipped screen box (one pixel of margin) holds the pixel;
//          w = t * dot(dir, fwd) must be >= near, depth = near / w
//   depth  the largest wins (reversed Z, compare 'greater'); equal depths keep the smaller triangle index
//          (the larger key depth bits << 32 | ~triangle, so the result does not depend on the order of the tests)
//   normal normalize(interpolated vertex normal) * (front ? 1 : -1) (gbuffer.ts:94-95), stored as f16; w = 0
//
// Binned in 16 x 16 pixel tiles: k_rs_setup gives every triangle its screen box, tile range and a depth bound,
// k_rs_bin lists each triangle in the tiles its box touches (count, scan, fill), and one block per tile keeps its
// 256 pixels' keys in registers while it walks the tile's list front to back by depth bound, in sorted chunks of 256.
// A triangle whose bound is below the depth every pixel of the tile already holds cannot win anywhere in the tile
// and ends the chunk; below one pixel's depth it is skipped for that pixel.  Skipped pairs are exactly pairs whose
// key would lose, so the result equals testing every (pixel, triangle whose box holds it) pair.  Triangles beyond the
// list capacity go to an overflow list that every tile walks, so the result never depends on the capacity.
#include <cuda_runtime.h>

#include "gi_dev.cuh"
#include "gi_internal.h"

namespace gi {

constexpr uint32_t RT = 16;               // tile edge in pixels; one thread per pixel
constexpr float DEPTH_MARGIN = 1.03125f;  // slack on the depth bound for the rounding of the ray test

// Moller-Trumbore with the edges precomputed (e1 = b - a, e2 = c - a: the same f32 values as computing them here)
__device__ __forceinline__ bool ray_tri(f3 o, f3 dir, f3 a, f3 e1, f3 e2, float &t, float &u, float &v) {
  f3 pv = cross(dir, e2);
  float det = dot(e1, pv);
  if (det == 0.0f) return false;
  float inv = 1.0f / det;
  f3 tv = o - a;
  float uu = dot(tv, pv) * inv;
  if (uu < 0.0f || uu > 1.0f) return false;
  f3 qv = cross(tv, e1);
  float vv = dot(dir, qv) * inv;
  if (vv < 0.0f || uu + vv > 1.0f) return false;
  float tt = dot(e2, qv) * inv;
  if (!(tt > 0.0f)) return false;
  t = tt; u = uu; v = vv;
  return true;
}

// Screen box of the triangle clipped to w >= near, one pixel of margin, clamped.  False when empty.  min_w: the
// smallest clip w of the clipped polygon (near when an edge crosses the near plane).
__device__ __forceinline__ bool screen_box(const float *__restrict__ F, uint32_t W, uint32_t H, const f3 p[3], int box[4],
                                           float &min_w) {
  const float *m = F + F_VP;
  float near = F[F_EYE + 3];
  float cl[3][4];
#pragma unroll
  for (int k = 0; k < 3; k++)
#pragma unroll
    for (int i = 0; i < 4; i++) cl[k][i] = m[i] * p[k].x + m[4 + i] * p[k].y + m[8 + i] * p[k].z + m[12 + i] * 1.0f;
  float x0 = 1e30f, x1 = -1e30f, y0 = 1e30f, y1 = -1e30f;
  int np = 0;
  min_w = 3.0e38f;
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const float *a = cl[k], *b = cl[(k + 1) % 3];
    bool ina = a[3] >= near, inb = b[3] >= near;
    float px[2], py[2];
    int cnt = 0;
    if (ina) { px[cnt] = a[0] / a[3]; py[cnt] = a[1] / a[3]; cnt++; min_w = mn(min_w, a[3]); }
    if (ina != inb) {
      float t = (a[3] - near) / (a[3] - b[3]);
      float x = a[0] + (b[0] - a[0]) * t, y = a[1] + (b[1] - a[1]) * t;
      px[cnt] = x / near; py[cnt] = y / near; cnt++;
      min_w = mn(min_w, near);
    }
    for (int j = 0; j < cnt; j++) {
      float sx = (px[j] * 0.5f + 0.5f) * (float)W, sy = (0.5f - py[j] * 0.5f) * (float)H;
      x0 = mn(x0, sx); x1 = mx(x1, sx); y0 = mn(y0, sy); y1 = mx(y1, sy);
      np++;
    }
  }
  if (np == 0) return false;
  if (!(x1 >= -1.0f) || !(y1 >= -1.0f) || !(x0 <= (float)W + 1.0f) || !(y0 <= (float)H + 1.0f)) return false;
  box[0] = iclamp(f2i(floorf(mx(x0, -2.0f))) - 1, 0, (int)W - 1);
  box[1] = iclamp(f2i(floorf(mn(x1, (float)W + 2.0f))) + 1, 0, (int)W - 1);
  box[2] = iclamp(f2i(floorf(mx(y0, -2.0f))) - 1, 0, (int)H - 1);
  box[3] = iclamp(f2i(floorf(mn(y1, (float)H + 2.0f))) + 1, 0, (int)H - 1);
  return true;
}

// The key of (pixel ray, triangle): depth bits << 32 | ~t, or 0 when the ray misses or the hit is nearer than near
__device__ __forceinline__ unsigned long long pixel_key(const float *__restrict__ F, f3 eye, f3 dir, f3 a, f3 e1, f3 e2,
                                                        uint32_t t, float &uu, float &vv) {
  float tt;
  if (!ray_tri(eye, dir, a, e1, e2, tt, uu, vv)) return 0ull;
  float w = tt * dot(dir, mk(F[F_FWD], F[F_FWD + 1], F[F_FWD + 2]));
  float near = F[F_EYE + 3];
  if (!(w >= near)) return 0ull;
  float depth = near / w;
  return ((unsigned long long)__float_as_uint(depth) << 32) | (unsigned long long)(0xffffffffu - t);
}

__device__ __forceinline__ uint32_t block_sum_256(uint32_t x, uint32_t *excl) {
  __shared__ uint32_t ws[8];
  __shared__ uint32_t tot;
  uint32_t lane = threadIdx.x & 31u, wid = threadIdx.x >> 5, inc = x;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, inc, d);
    if (lane >= (uint32_t)d) inc += y;
  }
  if (lane == 31u) ws[wid] = inc;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t a = 0;
    for (int k = 0; k < 8; k++) { uint32_t q = ws[k]; ws[k] = a; a += q; }
    tot = a;
  }
  __syncthreads();
  *excl = ws[wid] + inc - x;
  uint32_t r = tot;
  __syncthreads();
  return r;
}

// Per triangle: the record (a, bound; e1, x0 | x1 << 16; e2, y0 | y1 << 16), the tile count of its box, and the
// exclusive prefix of the tile counts within its block of 256 triangles (block totals to sums)
__global__ void __launch_bounds__(256) k_rs_setup(SceneDev s, const float *__restrict__ F, uint32_t W, uint32_t H,
                                                  RasterDev rd) {
  grid_dep_wait();
  uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  for (uint32_t i = t; i <= rd.ntiles; i += gridDim.x * blockDim.x) rd.tile_cnt[i] = 0u;   // counted by k_rs_bin
  uint32_t nt = 0;
  if (t < s.ntris) {
    f3 off;
    uint4 idx = drawn_tri(s, t, off);
    f3 p[3];
    p[0] = ld3(s.pos[idx.x]); p[1] = ld3(s.pos[idx.y]); p[2] = ld3(s.pos[idx.z]);
    if (s.inst) { p[0] = p[0] + off; p[1] = p[1] + off; p[2] = p[2] + off; }
    int box[4];
    float min_w;
    if (screen_box(F, W, H, p, box, min_w)) {
      float near = F[F_EYE + 3];
      // every hit of the triangle has w >= min_w up to rounding, so its depth near / w is at most near / min_w
      float bound = min_w > near ? near / min_w * DEPTH_MARGIN : 3.0e38f;
      f3 e1 = p[1] - p[0], e2 = p[2] - p[0];
      rd.rec[3u * t] = make_float4(p[0].x, p[0].y, p[0].z, bound);
      rd.rec[3u * t + 1u] = make_float4(e1.x, e1.y, e1.z, __uint_as_float((uint32_t)box[0] | ((uint32_t)box[1] << 16)));
      rd.rec[3u * t + 2u] = make_float4(e2.x, e2.y, e2.z, __uint_as_float((uint32_t)box[2] | ((uint32_t)box[3] << 16)));
      nt = ((uint32_t)box[1] / RT - (uint32_t)box[0] / RT + 1u) * ((uint32_t)box[3] / RT - (uint32_t)box[2] / RT + 1u);
    }
    rd.ntile[t] = nt;
  }
  uint32_t ex;
  uint32_t tot = block_sum_256(nt, &ex);
  if (t < s.ntris) rd.pre[t] = ex;
  if (threadIdx.x == 0) rd.sums[blockIdx.x] = tot;
}

// Block offsets of the triangle prefix (in place in sums) and the pair total; clears the overflow count
__global__ void __launch_bounds__(256) k_rs_scan(uint32_t nblk, RasterDev rd) {
  grid_dep_wait();
  __shared__ uint32_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (uint32_t b0 = 0; b0 < nblk; b0 += 256u) {
    uint32_t i = b0 + threadIdx.x;
    uint32_t ex;
    uint32_t tot = block_sum_256(i < nblk ? rd.sums[i] : 0u, &ex);
    if (i < nblk) rd.sums[i] = carry + ex;
    __syncthreads();
    if (threadIdx.x == 0) carry += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) { rd.counter[0] = carry; rd.counter[1] = 0u; }
}

// Every (triangle, tile) pair: FILL = false counts the pairs of each tile and lists the triangles that do not fit the
// list capacity; FILL = true writes each pair's triangle into its tile's range of the list
template <bool FILL>
__global__ void __launch_bounds__(256) k_rs_bin(uint32_t ntris, uint32_t tiles_x, RasterDev rd) {
  grid_dep_wait();
  uint32_t total = rd.counter[0];
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < total; p += gridDim.x * blockDim.x) {
    uint32_t lo = 0, hi = ntris;   // the last triangle whose first pair is <= p: the owner (it has pairs)
    while (hi - lo > 1u) {
      uint32_t m = (lo + hi) >> 1;
      if (rd.pre[m] + rd.sums[m >> 8] <= p) lo = m; else hi = m;
    }
    uint32_t first = rd.pre[lo] + rd.sums[lo >> 8], nt = rd.ntile[lo];
    if (first + nt > rd.list_cap) {
      if (!FILL && p == first) rd.over[atomicAdd(&rd.counter[1], 1u)] = lo;
      continue;
    }
    uint32_t bx = __float_as_uint(rd.rec[3u * lo + 1u].w), by = __float_as_uint(rd.rec[3u * lo + 2u].w);
    uint32_t tx0 = (bx & 0xffffu) / RT, tw = (bx >> 16) / RT - tx0 + 1u, ty0 = (by & 0xffffu) / RT;
    uint32_t i = p - first;
    uint32_t tile = (ty0 + i / tw) * tiles_x + tx0 + i % tw;
    if (!FILL) {
      atomicAdd(&rd.tile_cnt[tile], 1u);
    } else {
      uint32_t slot = atomicAdd(&rd.tile_fill[tile], 1u);
      rd.list[rd.tile_cnt[tile] + slot] = lo;
    }
  }
}

// Exclusive scan of the tile counts in place (tile_cnt becomes the list offsets, tile_cnt[ntiles] the end); clears
// the fill cursors
__global__ void __launch_bounds__(1024) k_rs_tile_scan(RasterDev rd) {
  grid_dep_wait();
  __shared__ uint32_t ws[32];
  __shared__ uint32_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  uint32_t lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
  for (uint32_t b0 = 0; b0 < rd.ntiles; b0 += 1024u) {
    uint32_t i = b0 + threadIdx.x;
    uint32_t x = i < rd.ntiles ? rd.tile_cnt[i] : 0u, inc = x;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, inc, d);
      if (lane >= (uint32_t)d) inc += y;
    }
    if (lane == 31u) ws[wid] = inc;
    __syncthreads();
    if (wid == 0) {
      uint32_t v = ws[lane], vi = v;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, vi, d);
        if (lane >= (uint32_t)d) vi += y;
      }
      ws[lane] = vi - v;
    }
    __syncthreads();
    if (i < rd.ntiles) { rd.tile_cnt[i] = carry + ws[wid] + inc - x; rd.tile_fill[i] = 0u; }
    __syncthreads();
    if (threadIdx.x == 1023u) carry += ws[wid] + inc;
    __syncthreads();
  }
  if (threadIdx.x == 0) rd.tile_cnt[rd.ntiles] = carry;
}

// Smallest depth bits held by the block's 256 pixels (pixels off the screen hold +inf)
__device__ __forceinline__ uint32_t block_min_256(uint32_t x, uint32_t *ws) {
  uint32_t m = __reduce_min_sync(0xffffffffu, x);
  if ((threadIdx.x & 31u) == 0) ws[threadIdx.x >> 5] = m;
  __syncthreads();
  uint32_t r = ws[0];
#pragma unroll
  for (int k = 1; k < 8; k++) r = min(r, ws[k]);
  __syncthreads();
  return r;
}

// One block per tile: the tile's list, then the overflow list, in chunks of 256 sorted by depth bound (largest
// first), fragments of alpha-masked materials whose alpha falls below the cutoff left out; then the winner's depth,
// normal and style tag
__global__ void __launch_bounds__(256) k_rs_tiles(SceneDev s, const float *__restrict__ F, uint32_t W, uint32_t H,
                                                  uint32_t tiles_x, RasterDev rd, float *depth, uint2 *normal,
                                                  uint8_t *tag) {
  grid_dep_wait();
  __shared__ float4 sa[256], se1[256], se2[256];
  __shared__ uint32_t skey[256], sval[256];
  __shared__ uint32_t ws[8];
  uint32_t tile = blockIdx.x;
  uint32_t x = (tile % tiles_x) * RT + (threadIdx.x % RT), y = (tile / tiles_x) * RT + (threadIdx.x / RT);
  bool inside = x < W && y < H;
  f3 eye = mk(F[F_EYE], F[F_EYE + 1], F[F_EYE + 2]);
  f3 dir = mk(0.0f, 0.0f, 0.0f);
  if (inside) dir = world_at(F, (int)x, (int)y, 1.0f) - eye;
  unsigned long long best = 0ull;
  uint32_t my_depth = inside ? 0u : 0x7f800000u;   // depth bits of best (positive floats order as integers)
  for (int pass = 0; pass < 2; pass++) {
    uint32_t beg = pass == 0 ? rd.tile_cnt[tile] : 0u, end = pass == 0 ? rd.tile_cnt[tile + 1u] : rd.counter[1];
    const uint32_t *lst = pass == 0 ? rd.list : rd.over;
    for (uint32_t c0 = beg; c0 < end; c0 += 256u) {
      uint32_t n = min(256u, end - c0);
      uint32_t t = 0, kb = 0;   // empty slots sort last (every bound is > 0)
      if (threadIdx.x < n) {
        t = lst[c0 + threadIdx.x];
        kb = __float_as_uint(rd.rec[3u * t].w);
      }
      skey[threadIdx.x] = kb;
      sval[threadIdx.x] = t;
      __syncthreads();
      for (uint32_t k = 2; k <= 256u; k <<= 1) {      // bitonic sort, descending
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
          uint32_t i = threadIdx.x, l = i ^ j;
          if (l > i) {
            uint32_t a = skey[i], b = skey[l];
            if ((i & k) == 0 ? a < b : a > b) {
              skey[i] = b; skey[l] = a;
              uint32_t v = sval[i]; sval[i] = sval[l]; sval[l] = v;
            }
          }
          __syncthreads();
        }
      }
      if (threadIdx.x < n) {
        uint32_t u = sval[threadIdx.x];
        sa[threadIdx.x] = rd.rec[3u * u];
        se1[threadIdx.x] = rd.rec[3u * u + 1u];
        se2[threadIdx.x] = rd.rec[3u * u + 2u];
      }
      __syncthreads();
      uint32_t far = 0;
      for (uint32_t j = 0; j < n; j++) {
        if ((j & 31u) == 0) far = block_min_256(my_depth, ws);   // every thread reaches it at the same j
        float4 a = sa[j];
        uint32_t bound = __float_as_uint(a.w);
        if (bound < far) break;                     // no pixel of the tile can take this or a later triangle
        if (!inside || bound < my_depth) continue;  // this pixel cannot
        float4 e1 = se1[j], e2 = se2[j];
        uint32_t bx = __float_as_uint(e1.w), by = __float_as_uint(e2.w);
        if (x < (bx & 0xffffu) || x > (bx >> 16) || y < (by & 0xffffu) || y > (by >> 16)) continue;
        float uu = 0.0f, vv = 0.0f;
        unsigned long long k = pixel_key(F, eye, dir, mk(a.x, a.y, a.z), mk(e1.x, e1.y, e1.z), mk(e2.x, e2.y, e2.z),
                                         sval[j], uu, vv);
        if (k > best) {
          if (s.masked) {   // an alpha-masked fragment is discarded (gbuffer.ts:94)
            f3 off;
            if (!raster_alpha_ok(s, drawn_tri(s, sval[j], off), (1.0f - uu) - vv, uu, vv)) continue;
          }
          best = k; my_depth = (uint32_t)(k >> 32);
        }
      }
      __syncthreads();
    }
  }
  if (!inside) return;
  size_t q = (size_t)y * W + x;
  if (best == 0ull) { depth[q] = 0.0f; normal[q] = make_uint2(0u, 0u); tag[q] = 0u; return; }
  uint32_t t = 0xffffffffu - (uint32_t)(best & 0xffffffffull);
  depth[q] = __uint_as_float((uint32_t)(best >> 32));
  float4 a4 = rd.rec[3u * t], e14 = rd.rec[3u * t + 1u], e24 = rd.rec[3u * t + 2u];
  f3 a = mk(a4.x, a4.y, a4.z), e1 = mk(e14.x, e14.y, e14.z), e2 = mk(e24.x, e24.y, e24.z);
  float tt = 0.0f, uu = 0.0f, vv = 0.0f;
  ray_tri(eye, dir, a, e1, e2, tt, uu, vv);
  f3 off;
  uint4 idx = drawn_tri(s, t, off);
  f3 n0 = ld3(s.nrm[idx.x]), n1 = ld3(s.nrm[idx.y]), n2 = ld3(s.nrm[idx.z]);
  f3 nn = (n0 * (1.0f - uu - vv) + n1 * uu) + n2 * vv;
  float flip = dot(cross(e1, e2), eye - a) > 0.0f ? 1.0f : -1.0f;
  nn = normalize3(nn) * flip;
  normal[q] = make_uint2((uint32_t)f2h(nn.x) | ((uint32_t)f2h(nn.y) << 16), (uint32_t)f2h(nn.z));
  // the albedo's alpha (gbuffer.ts:2): 1 toon, 0.5 another measured object, 0 photoreal, as an 8-bit unorm
  const uint32_t fl = s.mats[idx.w].flags;
  tag[q] = (fl & 4u) ? 255u : ((fl & 8u) ? 128u : 0u);
}

}  // namespace gi

using namespace gi;

namespace gi {
// Level 0 of every layer: the texels decoded (rgb through the sRGB table, alpha k / 255)
__global__ void k_tex_decode(const uint8_t *__restrict__ rgba8, const float *__restrict__ lut, float4 *tex, uint32_t size,
                             uint32_t layers, uint32_t per) {
  const uint64_t n = (uint64_t)size * size;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n * layers; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t l = i / n, t = i - l * n;
    const uchar4 c = reinterpret_cast<const uchar4 *>(rgba8)[i];
    tex[l * per + t] = make_float4(lut[c.x], lut[c.y], lut[c.z], (float)c.w / 255.0f);
  }
}
// Level k + 1 of every layer (size m) from level k (size 2m): the mean of its 2 x 2 texels, ((a + b) + (c + d)) / 4
__global__ void k_tex_mip(float4 *tex, uint32_t m, uint32_t src_off, uint32_t dst_off, uint32_t layers, uint32_t per) {
  const uint64_t n = (uint64_t)m * m;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n * layers; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t l = i / n, t = i - l * n;
    const uint32_t x = (uint32_t)(t % m), y = (uint32_t)(t / m), w = 2u * m;
    const float4 *s = tex + l * per + src_off;
    const float4 a = s[(2u * y) * w + 2u * x], b = s[(2u * y) * w + 2u * x + 1u];
    const float4 c = s[(2u * y + 1u) * w + 2u * x], d = s[(2u * y + 1u) * w + 2u * x + 1u];
    tex[l * per + dst_off + t] = make_float4(((a.x + b.x) + (c.x + d.x)) * 0.25f, ((a.y + b.y) + (c.y + d.y)) * 0.25f,
                                             ((a.z + b.z) + (c.z + d.z)) * 0.25f, ((a.w + b.w) + (c.w + d.w)) * 0.25f);
  }
}
}  // namespace gi

cudaError_t gi_launch_tex_build(const uint8_t *rgba8, const float *lut, float4 *tex, uint32_t size, uint32_t levels,
                                uint32_t layers, uint32_t per) {
  k_tex_decode<<<1184, 256>>>(rgba8, lut, tex, size, layers, per);
  uint32_t off = 0;
  for (uint32_t k = 0; k + 1u < levels; k++) {
    const uint32_t n = size >> k;
    k_tex_mip<<<1184, 256>>>(tex, n / 2u, off, off + n * n, layers, per);
    off += n * n;
  }
  return cudaGetLastError();
}

uint32_t gi_raster_tiles(uint32_t W, uint32_t H) { return ((W + RT - 1u) / RT) * ((H + RT - 1u) / RT); }

cudaError_t gi_launch_gbuffer(const SceneDev &s, const float *frame_dev, uint32_t W, uint32_t H, float *depth,
                              uint2 *normal, uint8_t *tag, const RasterDev &rd, uint32_t sm_count, cudaStream_t st) {
  uint32_t tiles_x = (W + RT - 1u) / RT;
  uint32_t nblk = s.ntris ? (s.ntris + 255u) / 256u : 1u;
  GI_TRY(gi_launch(k_rs_setup, nblk, 256, st, s, frame_dev, W, H, rd));
  GI_TRY(gi_launch(k_rs_scan, 1, 256, st, nblk, rd));
  if (s.ntris) GI_TRY(gi_launch(k_rs_bin<false>, sm_count * 8u, 256, st, s.ntris, tiles_x, rd));
  GI_TRY(gi_launch(k_rs_tile_scan, 1, 1024, st, rd));
  if (s.ntris) GI_TRY(gi_launch(k_rs_bin<true>, sm_count * 8u, 256, st, s.ntris, tiles_x, rd));
  GI_TRY(gi_launch(k_rs_tiles, rd.ntiles, 256, st, s, frame_dev, W, H, tiles_x, rd, depth, normal, tag));
  return cudaGetLastError();
}
