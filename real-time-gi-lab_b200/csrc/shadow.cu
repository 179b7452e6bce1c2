// Sun shadow map on sm_100a (the reference's shadow pass, src/core/lighting.ts:133-140, 175-189: depth32float cleared
// to 1, compare 'less', depthBias 2, depthBiasSlopeScale 2, cull none, alpha-masked fragments discarded), defined for
// a compute-only device as a raster of the light's orthographic clip space at texel centres:
//   clip     c_k = M * (p_k, 1), summed in column order; w = 1 (orthographic).  M is the layer's matrix: layer 0
//            lightViewProj (frame words 64-79), layer 1 of a world's camera-following pair lightViewProjFar (140-155);
//            each layer is one launch sequence into its own S x S slice
//   cover    texel (i, j) centre x = (i + 0.5) / S * 2 - 1, y = 1 - (j + 0.5) / S * 2 is inside when its three edge
//            functions w_k = (b - a) x (centre - a) are all >= 0 or all <= 0 (either winding, edges included)
//   depth    z = (w0 z0 + w1 z1 + w2 z2) / (w0 + w1 + w2), kept when 0 <= z <= 1
//   bias     2 r + 2 m: r = 2^(e - 23) for the exponent e of the largest |z_k|, m the larger of |dz/dx|, |dz/dy| per
//            texel (Vulkan's depth-bias terms for a float depth buffer)
//   stored   the smallest z + bias over the covering triangles, 1 where none; so the result does not depend on the
//            order in which the triangles are drawn
//   alpha    an alpha-masked material whose factor's alpha is below the cutoff draws nothing untextured; textured, a
//            texel is left out where the texture at level 0 at its barycentric weights w_k / (w0 + w1 + w2), times
//            the factor, falls below the cutoff
//
// Work: k_sm_setup gives every triangle its clip record, texel box and the number of 128-texel chunks of that box
// (prefix within blocks of 256 triangles); k_sm_scan turns the block sums into offsets and the chunk total; warps of
// k_sm_raster take chunks in turn, find their triangle with a 32-way search of the prefix, and test 32 texels per step
// (one texel per lane), keeping the smallest depth with atomicMin on the depth bits (non-negative floats order as
// their bits).
#include <cuda_runtime.h>

#include "gi_dev.cuh"
#include "gi_internal.h"

namespace gi {

constexpr uint32_t SM_CHUNK = 128;   // texels of a triangle's box per work item

__device__ __forceinline__ uint32_t sm_block_scan(uint32_t x, uint32_t *total) {
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
  uint32_t ex = ws[wid] + inc - x;
  *total = tot;
  __syncthreads();
  return ex;
}

// 2^(e - 23) for the exponent e of |z| (zero and subnormals take the smallest normal exponent)
__device__ __forceinline__ float sm_bias_unit(float zmax) {
  int eb = (int)((__float_as_uint(zmax) >> 23) & 0xffu);
  eb = eb < 1 ? 1 : eb;
  return ldexpf(1.0f, eb - 127 - 23);
}

// Per triangle: rec[4t] = (c0, bias), [4t+1] = (c1, i0 | j0 << 16), [4t+2] = (c2, bw | bh << 16), the chunk count,
// its exclusive prefix within the block and the block's sum.  Also clears the map (grid-stride).
__global__ void __launch_bounds__(256) k_sm_setup(SceneDev s, const float *__restrict__ M, uint32_t S, ShadowRaster sr) {
  grid_dep_wait();
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < (size_t)S * S; i += (size_t)gridDim.x * blockDim.x)
    sr.map[i] = 1.0f;
  uint32_t t = blockIdx.x * blockDim.x + threadIdx.x, nch = 0;
  if (t < s.ntris) {
    f3 off;
    uint4 idx = drawn_tri(s, t, off);
    const gi_material &mt = s.mats[idx.w];
    // an alpha-masked material: untextured, every fragment or none; textured, each texel tested (record word 12)
    const bool per_texel = (mt.flags & 1u) != 0u && tex_layer_of(s, mt) != 0u;
    if (per_texel || !((mt.flags & 1u) != 0u && mt.base_color[3] < mt.alpha_cutoff)) {
      f3 a = ld3(s.pos[idx.x]), b = ld3(s.pos[idx.y]), c = ld3(s.pos[idx.z]);
      if (s.inst) { a = a + off; b = b + off; c = c + off; }
      f3 c0 = light_clip(M, a), c1 = light_clip(M, b), c2 = light_clip(M, c);
      float det = (c1.x - c0.x) * (c2.y - c0.y) - (c2.x - c0.x) * (c1.y - c0.y);
      if (det != 0.0f) {
        const float inv = 1.0f / (float)S, fS = (float)S;
        float dzx = ((c1.z - c0.z) * (c2.y - c0.y) - (c2.z - c0.z) * (c1.y - c0.y)) / det;
        float dzy = ((c2.z - c0.z) * (c1.x - c0.x) - (c1.z - c0.z) * (c2.x - c0.x)) / det;
        float slope = mx(fabsf(dzx), fabsf(dzy)) * (2.0f * inv);
        float zmax = mx(mx(fabsf(c0.z), fabsf(c1.z)), fabsf(c2.z));
        float bias = 2.0f * sm_bias_unit(zmax) + 2.0f * slope;
        float xa = (c0.x + 1.0f) * 0.5f * fS, xb = (c1.x + 1.0f) * 0.5f * fS, xc = (c2.x + 1.0f) * 0.5f * fS;
        float ya = (1.0f - c0.y) * 0.5f * fS, yb = (1.0f - c1.y) * 0.5f * fS, yc = (1.0f - c2.y) * 0.5f * fS;
        float x0 = mn(mn(xa, xb), xc), x1 = mx(mx(xa, xb), xc), y0 = mn(mn(ya, yb), yc), y1 = mx(mx(ya, yb), yc);
        if (x1 >= -1.0f && y1 >= -1.0f && x0 <= fS + 1.0f && y0 <= fS + 1.0f) {
          int i0 = iclamp(__float2int_rd(mx(x0, -2.0f)) - 1, 0, (int)S - 1);
          int i1 = iclamp(__float2int_rd(mn(x1, fS + 2.0f)) + 1, 0, (int)S - 1);
          int j0 = iclamp(__float2int_rd(mx(y0, -2.0f)) - 1, 0, (int)S - 1);
          int j1 = iclamp(__float2int_rd(mn(y1, fS + 2.0f)) + 1, 0, (int)S - 1);
          uint32_t bw = (uint32_t)(i1 - i0 + 1), bh = (uint32_t)(j1 - j0 + 1);
          nch = (bw * bh + SM_CHUNK - 1u) / SM_CHUNK;
          sr.rec[4u * t] = make_float4(c0.x, c0.y, c0.z, bias);
          sr.rec[4u * t + 1u] = make_float4(c1.x, c1.y, c1.z, __uint_as_float((uint32_t)i0 | ((uint32_t)j0 << 16)));
          sr.rec[4u * t + 2u] = make_float4(c2.x, c2.y, c2.z, __uint_as_float(bw | (bh << 16)));
          sr.rec[4u * t + 3u] = make_float4(per_texel ? 1.0f : 0.0f, 0.0f, 0.0f, 0.0f);
        }
      }
    }
  }
  uint32_t tot;
  uint32_t ex = sm_block_scan(nch, &tot);
  if (t < s.ntris) sr.pre[t] = ex;
  if (threadIdx.x == 0) sr.sums[blockIdx.x] = tot;
}

// Block offsets of the chunk prefix (in place) and the chunk total (counter[0])
__global__ void __launch_bounds__(256) k_sm_scan(uint32_t nblk, ShadowRaster sr) {
  grid_dep_wait();
  __shared__ uint32_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (uint32_t b0 = 0; b0 < nblk; b0 += 256u) {
    uint32_t i = b0 + threadIdx.x, tot;
    uint32_t ex = sm_block_scan(i < nblk ? sr.sums[i] : 0u, &tot);
    if (i < nblk) sr.sums[i] = carry + ex;
    __syncthreads();
    if (threadIdx.x == 0) carry += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) sr.counter[0] = carry;
}

__device__ __forceinline__ uint32_t sm_first(const ShadowRaster &sr, uint32_t t) { return sr.pre[t] + sr.sums[t >> 8]; }

__global__ void __launch_bounds__(256) k_sm_raster(SceneDev s, uint32_t ntris, uint32_t S, ShadowRaster sr) {
  grid_dep_wait();
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t nwarps = gridDim.x * (blockDim.x >> 5), w0 = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const uint32_t total = sr.counter[0];
  const float inv = 1.0f / (float)S;
  for (uint32_t ch = w0; ch < total; ch += nwarps) {
    // the owner: the last triangle whose first chunk is <= ch, by a 32-way search (lane k probes lo + span k / 32)
    uint32_t lo = 0, hi = ntris;
    while (hi - lo > 1u) {
      uint32_t span = hi - lo;
      uint32_t m = lo + (uint32_t)(((unsigned long long)span * lane) >> 5);
      uint32_t ok = __ballot_sync(0xffffffffu, sm_first(sr, m) <= ch);
      uint32_t k = 31u - (uint32_t)__clz(ok);   // lane 0 probes lo, which always qualifies
      uint32_t nlo = lo + (uint32_t)(((unsigned long long)span * k) >> 5);
      hi = k == 31u ? hi : lo + (uint32_t)(((unsigned long long)span * (k + 1u)) >> 5);
      lo = nlo;
    }
    const uint32_t t = lo;
    const float4 ra = sr.rec[4u * t], rb = sr.rec[4u * t + 1u], rc = sr.rec[4u * t + 2u];
    const f3 c0 = mk(ra.x, ra.y, ra.z), c1 = mk(rb.x, rb.y, rb.z), c2 = mk(rc.x, rc.y, rc.z);
    const float bias = ra.w;
    const bool per_texel = sr.rec[4u * t + 3u].x != 0.0f;
    f3 toff;
    const uint4 tidx = per_texel ? drawn_tri(s, t, toff) : make_uint4(0u, 0u, 0u, 0u);
    const uint32_t ij = __float_as_uint(rb.w), wh = __float_as_uint(rc.w);
    const int i0 = (int)(ij & 0xffffu), j0 = (int)(ij >> 16), bw = (int)(wh & 0xffffu), bh = (int)(wh >> 16);
    const int area = bw * bh;
    int q = (int)((ch - sm_first(sr, t)) * SM_CHUNK) + (int)lane;
    const int q_end = min(area, q - (int)lane + (int)SM_CHUNK);
    // the lane's texel in the box (row-major), then 32 texels further per step: 32 = dy * bw + dx
    int yy = q / bw, xx = q - yy * bw;
    const int dy = 32 / bw, dx = 32 - dy * bw;
    for (; q - (int)lane < q_end; q += 32) {
      if (q < q_end) {
        const int i = i0 + xx, j = j0 + yy;
        float x = ((float)i + 0.5f) * inv * 2.0f - 1.0f;
        float y = 1.0f - ((float)j + 0.5f) * inv * 2.0f;
        float e0 = (c2.x - c1.x) * (y - c1.y) - (c2.y - c1.y) * (x - c1.x);
        float e1 = (c0.x - c2.x) * (y - c2.y) - (c0.y - c2.y) * (x - c2.x);
        float e2 = (c1.x - c0.x) * (y - c0.y) - (c1.y - c0.y) * (x - c0.x);
        bool in = (e0 >= 0.0f && e1 >= 0.0f && e2 >= 0.0f) || (e0 <= 0.0f && e1 <= 0.0f && e2 <= 0.0f);
        if (in) {
          float sum = (e0 + e1) + e2;
          if (sum != 0.0f) {
            float z = ((e0 * c0.z + e1 * c1.z) + e2 * c2.z) / sum;
            if (z >= 0.0f && z <= 1.0f && (!per_texel || raster_alpha_ok(s, tidx, e0 / sum, e1 / sum, e2 / sum))) {
              uint32_t zb = __float_as_uint(z + bias);
              uint32_t *d = reinterpret_cast<uint32_t *>(sr.map) + (size_t)j * S + (size_t)i;
              if (zb < *d) atomicMin(d, zb);
            }
          }
        }
      }
      xx += dx; yy += dy;
      if (xx >= bw) { xx -= bw; yy++; }
    }
  }
}

}  // namespace gi

using namespace gi;

cudaError_t gi_launch_shadow(const SceneDev &s, const float *matrix_dev, uint32_t S, const ShadowRaster &sr,
                             uint32_t sm_count, cudaStream_t st) {
  uint32_t nblk = s.ntris ? (s.ntris + 255u) / 256u : 1u;
  GI_TRY(gi_launch(k_sm_setup, nblk, 256, st, s, matrix_dev, S, sr));
  GI_TRY(gi_launch(k_sm_scan, 1, 256, st, nblk, sr));
  if (s.ntris) GI_TRY(gi_launch(k_sm_raster, sm_count * 8u, 256, st, s, s.ntris, S, sr));
  return cudaGetLastError();
}
