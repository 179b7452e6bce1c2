// Host/device shared declarations of the library (not part of the C-ABI).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "gi_dev.cuh"

namespace gi {

struct CascDev {
  uint32_t probe_off, rad_off, res, tile_size, tiles_x, tiles_y, ray_off, dir_off;
  float b0, b1;
  uint32_t dirs_log2, np;   // log2(res * res) (res is a power of two); probes (tiles_x * tiles_y)
};

struct ProbeDev { float4 pos; float4 nrm; int4 grid; };   // rc.ts:157 Probe, 48 bytes

// Radiance-cascade state of one solve in device memory.
struct RcDev {
  uint32_t cascades, width, height, atlas;
  CascDev c[8];
  float vox_scale, vox_offset, level_map, vox_skip;
  uint32_t dda_cap, stats, probes_total, rays_total;
  uint32_t trace_order, trace_rays, pad_t[2];   // tuning of k_trace (gi_rc_tuning)
  const float *frame;      // 160 words (packFrame)
  const float *depth;      // W*H
  const uint2 *normal;     // W*H rgba16f
  ProbeDev *probes;
  uint32_t *plevel;        // per probe: voxLevel(s0, c) (rc.ts:210-213), computed once by setupScreen
  const float4 *dirs;      // per cascade, res^2 texel directions dirOf(di, res) (rc.ts:308), computed at creation
  void *rad;               // rays_total atlas elements
  void *sh;                // probes of cascade 0 x 8 atlas elements
  void *irr;               // W*H: float4 (atlas F32) or rgba16f (uint2)
  uint32_t *counts;        // 80 words
  uint4 *hits;             // optional: per ray (level, brick, bit, tIn bits)
  void *rad_traced;        // optional: copy of the atlas after the trace
  float4 *mavg[2];         // merge: quad averages of the cascade above (ping-pong by cascade parity)
};

// Scratch of the binned G-buffer raster (gbuffer.cu)
struct RasterDev {
  float4 *rec;                     // 3 per triangle: (a, depth bound), (e1, x0 | x1 << 16), (e2, y0 | y1 << 16)
  uint32_t *ntile, *pre, *sums;    // per triangle: tiles its box touches, prefix within its block; block offsets
  uint32_t *counter;               // [0] (triangle, tile) pairs, [1] overflow triangles
  uint32_t *list, *over;           // per-tile triangle lists (list_cap entries), overflow triangles (ntris)
  uint32_t *tile_cnt, *tile_fill;  // per tile: count, then list offset (ntiles + 1); fill cursor (ntiles)
  uint32_t list_cap, ntiles;
};

}  // namespace gi

cudaError_t gi_launch_vox_build(const gi::VoxDev &v, const gi::SceneDev &s, uint32_t sm_count, cudaStream_t st);
// ev (optional, 5 events): recorded after giBuild (setupScreen), giTrace, giMerge (merge + projectSH), giGather.
// Launch shapes of the cascade passes (the result does not depend on them)
struct RcLaunch { uint32_t trace_blocks, gather_shape, merge_threads; };
cudaError_t gi_launch_rc_solve(const gi::RcDev &r, const gi::VoxDev &v, uint32_t sm_count, cudaStream_t st,
                               cudaEvent_t *ev = nullptr, const RcLaunch *ls = nullptr);
uint32_t gi_raster_tiles(uint32_t W, uint32_t H);
cudaError_t gi_launch_gbuffer(const gi::SceneDev &s, const float *frame_dev, uint32_t W, uint32_t H, float *depth,
                              uint2 *normal, const gi::RasterDev &rd, uint32_t sm_count, cudaStream_t st);
cudaError_t gi_launch_normal_f32_to_f16(const float4 *src, uint2 *dst, uint32_t n, cudaStream_t st);
cudaError_t gi_launch_irr_to_f32(const gi::RcDev &r, float4 *dst, cudaStream_t st);
cudaError_t gi_launch_init_dirs(const gi::RcDev &r, float4 *dirs, uint32_t ndirs, cudaStream_t st);
// FP64 reference of merge + SH + gather from the f32 traced atlas: rad64 rays_total x 4 doubles, sh64 27 doubles per
// cascade-0 probe, irr64 W*H x 4 doubles.
cudaError_t gi_launch_merge_gather_f64(const gi::RcDev &r, const float4 *traced, void *rad64, double *sh64, void *irr64,
                                       cudaStream_t st);
