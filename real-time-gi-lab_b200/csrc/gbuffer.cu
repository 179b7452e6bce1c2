// Headless G-buffer on sm_100a: reversed-Z depth (depth32float) and the rgba16float shading normal that the
// reference's raster pass writes (src/core/gbuffer.ts:82-103), defined here as one primary-ray sample per pixel
// centre (there is no graphics pipeline on a compute-only box):
//   ray    origin = eye, direction = worldAt(px, 1) - eye (the point on the near plane, frame.ts:22-26)
//   hit    Moller-Trumbore against the triangles whose near-clipped screen box (one pixel of margin) holds the pixel;
//          w = t * dot(dir, fwd) must be >= near, depth = near / w
//   depth  the largest wins (reversed Z, compare 'greater'); equal depths keep the smaller triangle index
//          (one 64-bit atomicMax of depth bits << 32 | ~triangle per sample, order independent)
//   normal normalize(interpolated vertex normal) * (front ? 1 : -1) (gbuffer.ts:94-95), stored as f16; w = 0
// Triangles whose box covers more than 256 pixels go to a list, cut into 256-pixel tiles taken from a queue.
#include <cuda_runtime.h>

#include "gi_dev.cuh"
#include "gi_internal.h"

namespace gi {

constexpr uint32_t RASTER_SMALL = 256;

__device__ __forceinline__ bool ray_tri(f3 o, f3 dir, f3 a, f3 b, f3 c, float &t, float &u, float &v) {
  f3 e1 = b - a, e2 = c - a;
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

// Screen box of the triangle clipped to w >= near, one pixel of margin, clamped.  False when empty.
__device__ __forceinline__ bool screen_box(const float *__restrict__ F, uint32_t W, uint32_t H, const f3 p[3], int box[4]) {
  const float *m = F + F_VP;
  float near = F[F_EYE + 3];
  float cl[3][4];
#pragma unroll
  for (int k = 0; k < 3; k++)
#pragma unroll
    for (int i = 0; i < 4; i++) cl[k][i] = m[i] * p[k].x + m[4 + i] * p[k].y + m[8 + i] * p[k].z + m[12 + i] * 1.0f;
  float x0 = 1e30f, x1 = -1e30f, y0 = 1e30f, y1 = -1e30f;
  int np = 0;
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const float *a = cl[k], *b = cl[(k + 1) % 3];
    bool ina = a[3] >= near, inb = b[3] >= near;
    float px[2], py[2];
    int cnt = 0;
    if (ina) { px[cnt] = a[0] / a[3]; py[cnt] = a[1] / a[3]; cnt++; }
    if (ina != inb) {
      float t = (a[3] - near) / (a[3] - b[3]);
      float x = a[0] + (b[0] - a[0]) * t, y = a[1] + (b[1] - a[1]) * t;
      px[cnt] = x / near; py[cnt] = y / near; cnt++;
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

__device__ __forceinline__ void sample_pixel(const float *__restrict__ F, uint32_t W, int x, int y, const f3 p[3],
                                             uint32_t t, unsigned long long *keys) {
  f3 eye = mk(F[F_EYE], F[F_EYE + 1], F[F_EYE + 2]);
  f3 dir = world_at(F, x, y, 1.0f) - eye;
  float tt, uu, vv;
  if (!ray_tri(eye, dir, p[0], p[1], p[2], tt, uu, vv)) return;
  float w = tt * dot(dir, mk(F[F_FWD], F[F_FWD + 1], F[F_FWD + 2]));
  float near = F[F_EYE + 3];
  if (!(w >= near)) return;
  float depth = near / w;
  unsigned long long k = ((unsigned long long)__float_as_uint(depth) << 32) | (unsigned long long)(0xffffffffu - t);
  unsigned long long *kp = &keys[(size_t)y * W + (size_t)x];
  if (k > *kp) atomicMax(kp, k);
}

__global__ void __launch_bounds__(256) k_raster_small(SceneDev s, const float *__restrict__ F, uint32_t W, uint32_t H,
                                                      unsigned long long *keys, uint32_t *big, uint32_t big_cap,
                                                      uint32_t *counter) {
  uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  bool live = t < s.ntris;
  f3 p[3];
  int box[4] = {0, -1, 0, -1};
  bool any = false;
  if (live) {
    uint4 idx = s.tri[t];
    p[0] = ld3(s.pos[idx.x]); p[1] = ld3(s.pos[idx.y]); p[2] = ld3(s.pos[idx.z]);
    any = screen_box(F, W, H, p, box);
  }
  uint32_t area = any ? (uint32_t)(box[1] - box[0] + 1) * (uint32_t)(box[3] - box[2] + 1) : 0u;
  bool is_big = area > RASTER_SMALL;
  uint32_t k = warp_append(counter, is_big);
  if (is_big) {
    if (k < big_cap) big[k] = t;
    return;
  }
  if (!any) return;
  for (int y = box[2]; y <= box[3]; y++)
    for (int x = box[0]; x <= box[1]; x++) sample_pixel(F, W, x, y, p, t, keys);
}

// Big triangles, balanced: each one's box is cut into tiles of 256 pixels; k_raster_count gives every listed triangle
// its tile count and an exclusive prefix within blocks of 256 triangles, k_raster_scan the block offsets and the
// total, and blocks of k_raster_big take tiles from a queue (counter[1]) and find their triangle by binary search.
__device__ __forceinline__ bool big_box(const SceneDev &s, const float *__restrict__ F, uint32_t W, uint32_t H,
                                        uint32_t t, f3 p[3], int box[4]) {
  uint4 idx = s.tri[t];
  p[0] = ld3(s.pos[idx.x]); p[1] = ld3(s.pos[idx.y]); p[2] = ld3(s.pos[idx.z]);
  return screen_box(F, W, H, p, box);
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

__global__ void __launch_bounds__(256) k_raster_count(SceneDev s, const float *__restrict__ F, uint32_t W, uint32_t H,
                                                      const uint32_t *big, uint32_t big_cap, uint32_t *counter,
                                                      uint32_t *pre, uint32_t *sums) {
  uint32_t items = min(counter[0], big_cap);
  uint32_t nblk = (items + 255u) / 256u;
  for (uint32_t b = blockIdx.x; b < nblk; b += gridDim.x) {
    uint32_t it = b * 256u + threadIdx.x, tiles = 0;
    if (it < items) {
      f3 p[3];
      int box[4];
      if (big_box(s, F, W, H, big[it], p, box))
        tiles = ((uint32_t)(box[1] - box[0] + 1) * (uint32_t)(box[3] - box[2] + 1) + 255u) / 256u;
    }
    uint32_t ex;
    uint32_t tot = block_sum_256(tiles, &ex);
    if (it < items) pre[it] = ex;
    if (threadIdx.x == 0) sums[b] = tot;
  }
}

__global__ void __launch_bounds__(256) k_raster_scan(uint32_t big_cap, uint32_t *counter, uint32_t *sums) {
  uint32_t nblk = (min(counter[0], big_cap) + 255u) / 256u;
  __shared__ uint32_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (uint32_t b0 = 0; b0 < nblk; b0 += 256u) {
    uint32_t i = b0 + threadIdx.x;
    uint32_t ex;
    uint32_t tot = block_sum_256(i < nblk ? sums[i] : 0u, &ex);
    if (i < nblk) sums[i] = carry + ex;
    __syncthreads();
    if (threadIdx.x == 0) carry += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) { counter[2] = carry; counter[1] = 0u; }
}

__global__ void __launch_bounds__(256) k_raster_big(SceneDev s, const float *__restrict__ F, uint32_t W, uint32_t H,
                                                    unsigned long long *keys, const uint32_t *big, uint32_t big_cap,
                                                    uint32_t *counter, const uint32_t *pre, const uint32_t *sums) {
  uint32_t items = min(counter[0], big_cap);
  uint32_t tiles = counter[2];
  __shared__ uint32_t s_tile;
  for (;;) {
    if (threadIdx.x == 0) s_tile = atomicAdd(&counter[1], 1u);
    __syncthreads();
    uint32_t tile = s_tile;
    __syncthreads();
    if (tile >= tiles) break;
    uint32_t lo = 0, hi = items;   // the last triangle whose first tile is <= tile
    while (hi - lo > 1u) {
      uint32_t m = (lo + hi) >> 1;
      if (pre[m] + sums[m >> 8] <= tile) lo = m; else hi = m;
    }
    uint32_t t = big[lo];
    f3 p[3];
    int box[4];
    if (!big_box(s, F, W, H, t, p, box)) continue;
    uint32_t bw = (uint32_t)(box[1] - box[0] + 1), bh = (uint32_t)(box[3] - box[2] + 1);
    uint32_t q = (tile - (pre[lo] + sums[lo >> 8])) * 256u + threadIdx.x;
    if (q < bw * bh) sample_pixel(F, W, box[0] + (int)(q % bw), box[2] + (int)(q / bw), p, t, keys);
  }
}

__global__ void __launch_bounds__(256) k_raster_resolve(SceneDev s, const float *__restrict__ F, uint32_t W, uint32_t H,
                                                        const unsigned long long *keys, float *depth, uint2 *normal) {
  uint32_t x = blockIdx.x * 16u + (threadIdx.x & 15u), y = blockIdx.y * 16u + (threadIdx.x >> 4);
  if (x >= W || y >= H) return;
  size_t q = (size_t)y * W + x;
  unsigned long long k = keys[q];
  if (k == 0ull) { depth[q] = 0.0f; normal[q] = make_uint2(0u, 0u); return; }
  uint32_t t = 0xffffffffu - (uint32_t)(k & 0xffffffffull);
  depth[q] = __uint_as_float((uint32_t)(k >> 32));
  uint4 idx = s.tri[t];
  f3 a = ld3(s.pos[idx.x]), b = ld3(s.pos[idx.y]), c = ld3(s.pos[idx.z]);
  f3 eye = mk(F[F_EYE], F[F_EYE + 1], F[F_EYE + 2]);
  f3 dir = world_at(F, (int)x, (int)y, 1.0f) - eye;
  float tt = 0.0f, uu = 0.0f, vv = 0.0f;
  ray_tri(eye, dir, a, b, c, tt, uu, vv);
  f3 n0 = ld3(s.nrm[idx.x]), n1 = ld3(s.nrm[idx.y]), n2 = ld3(s.nrm[idx.z]);
  f3 nn = (n0 * (1.0f - uu - vv) + n1 * uu) + n2 * vv;
  float flip = dot(cross(b - a, c - a), eye - a) > 0.0f ? 1.0f : -1.0f;
  nn = normalize3(nn) * flip;
  normal[q] = make_uint2((uint32_t)f2h(nn.x) | ((uint32_t)f2h(nn.y) << 16), (uint32_t)f2h(nn.z));
}

}  // namespace gi

using namespace gi;

cudaError_t gi_launch_gbuffer(const SceneDev &s, const float *frame_dev, uint32_t W, uint32_t H, float *depth,
                              uint2 *normal, unsigned long long *keys, uint32_t *big, uint32_t big_cap,
                              uint32_t *counter, uint32_t *pre, uint32_t *sums, uint32_t sm_count, cudaStream_t st) {
  cudaMemsetAsync(keys, 0, (size_t)W * H * sizeof(unsigned long long), st);
  cudaMemsetAsync(counter, 0, 4 * sizeof(uint32_t), st);
  if (s.ntris) k_raster_small<<<(s.ntris + 255u) / 256u, 256, 0, st>>>(s, frame_dev, W, H, keys, big, big_cap, counter);
  k_raster_count<<<sm_count * 2u, 256, 0, st>>>(s, frame_dev, W, H, big, big_cap, counter, pre, sums);
  k_raster_scan<<<1, 256, 0, st>>>(big_cap, counter, sums);
  k_raster_big<<<sm_count * 8u, 256, 0, st>>>(s, frame_dev, W, H, keys, big, big_cap, counter, pre, sums);
  dim3 g((W + 15u) / 16u, (H + 15u) / 16u);
  k_raster_resolve<<<g, 256, 0, st>>>(s, frame_dev, W, H, keys, depth, normal);
  return cudaGetLastError();
}
