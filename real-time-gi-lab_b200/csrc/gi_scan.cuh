// Block scans and chained single-pass scans (decoupled look-back) shared by the voxel rebuild and the world probes.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace gi {

// Block-wide exclusive scan of one value per thread (256 threads).  Returns the exclusive prefix; *total = sum.
__device__ __forceinline__ uint32_t block_scan_256(uint32_t x, uint32_t *total) {
  __shared__ uint32_t warp_sums[8];
  __shared__ uint32_t s_total;
  uint32_t lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
  uint32_t inc = x;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, inc, d);
    if (lane >= (uint32_t)d) inc += y;
  }
  if (lane == 31u) warp_sums[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    uint32_t ws = lane < 8u ? warp_sums[lane] : 0u;
    uint32_t wi = ws;
#pragma unroll
    for (int d = 1; d < 8; d <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, wi, d);
      if (lane >= (uint32_t)d) wi += y;
    }
    if (lane < 8u) warp_sums[lane] = wi - ws;   // exclusive prefix of the warps
    if (lane == 7u) s_total = wi;
  }
  __syncthreads();
  uint32_t excl = warp_sums[wid] + inc - x;
  if (total) *total = s_total;
  __syncthreads();   // the next call may overwrite warp_sums / s_total
  return excl;
}

// ---- chained scans: one pass, decoupled look-back ---------------------------------------------------------------
// look[0] hands out tickets (the order in which blocks take their part of the scan: every smaller ticket belongs to
// a block that is already running); look[1 + k] is part k's state, status << 32 | value with status 1 = the part's
// own sum, 2 = the inclusive prefix through the part.  A part waits only on smaller tickets, so every wait ends; the
// spin is bounded all the same, and a part that gives up sets header word 6 and takes what it has (the host reports
// it as GI_ERR_TIMEOUT when it reads the counters).
constexpr uint32_t LOOK_SPIN = 1u << 20;

__device__ __forceinline__ void st_release_u64(unsigned long long *p, unsigned long long x) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(x) : "memory");
}
__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long *p) {
  unsigned long long x;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(x) : "l"(p) : "memory");
  return x;
}

// The block's ticket (block-uniform; all threads call it).
__device__ __forceinline__ uint32_t chain_ticket(unsigned long long *look) {
  __shared__ uint32_t s_ticket;
  if (threadIdx.x == 0) s_ticket = (uint32_t)atomicAdd(look, 1ull);
  __syncthreads();
  uint32_t t = s_ticket;
  __syncthreads();
  return t;
}

// One thread per block: publishes part k's sum, looks back for its exclusive prefix, publishes the inclusive prefix.
// hold = k + 1 makes part k publish nothing (a test of the bounded wait: the parts after it give up), else 0.
__device__ __forceinline__ uint32_t chain_prefix(unsigned long long *look, uint32_t k, uint32_t sum, uint32_t *hdr,
                                                 uint32_t hold = 0u) {
  if (hold != 0u && hold == k + 1u) return 0u;
  unsigned long long *st = look + 1;
  if (k == 0u) { st_release_u64(st, (2ull << 32) | sum); return 0u; }
  st_release_u64(st + k, (1ull << 32) | sum);
  uint32_t excl = 0, j = k - 1u, spins = 0;
  for (;;) {
    unsigned long long x = ld_acquire_u64(st + j);
    uint32_t f = (uint32_t)(x >> 32);
    if (f == 0u) {
      if (++spins > LOOK_SPIN) { atomicExch(&hdr[6], 1u); break; }
      __nanosleep(32);
      continue;
    }
    excl += (uint32_t)x;
    if (f == 2u || j == 0u) break;
    j--;
  }
  st_release_u64(st + k, (2ull << 32) | (excl + sum));
  return excl;
}

}  // namespace gi
