// Host/device shared declarations of the library (not part of the C-ABI).
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "gi_dev.cuh"

namespace gi {

struct CascDev {
  uint32_t probe_off, rad_off, res, tile_size, tiles_x, tiles_y, ray_off, dir_off;
  float b0, b1;
  uint32_t dirs_log2, np;   // log2(res * res) (res is a power of two); probes (tiles_x * tiles_y)
  float inv_tile;           // 1 / tile_size when tile_size is a power of two (x * inv_tile == x / tile_size), else 0
  uint32_t pad3[3];
};

// x / tile_size: a multiplication when the tile is a power of two (exact), else the division
__device__ __forceinline__ float div_tile(float x, const CascDev &L) {
  return L.inv_tile != 0.0f ? x * L.inv_tile : x / (float)L.tile_size;
}

struct ProbeDev { float4 pos; float4 nrm; int4 grid; };   // rc.ts:157 Probe, 48 bytes

// Radiance-cascade state of one solve in device memory.
struct RcDev {
  uint32_t cascades, width, height, atlas;
  CascDev c[8];
  float vox_scale, vox_offset, level_map, vox_skip;
  uint32_t dda_cap, stats, probes_total, rays_total;
  uint32_t trace_order, trace_rays;   // tuning of k_trace (gi_rc_tuning; trace_order 2: walk-length order)
  uint32_t f32_out;                   // SH and irradiance stored as f32 whatever the atlas
  uint32_t irr_f16;                   // irradiance stored as rgba16f whatever the atlas and f32_out
  uint32_t tag_any, pad_tag;          // nonzero once a G-buffer with style tags was set or drawn (world gather)
  const float *frame;      // 160 words (packFrame)
  const float *depth;      // W*H
  const uint2 *normal;     // W*H rgba16f
  const uint8_t *tag;      // W*H: the G-buffer albedo's alpha byte (style tag: 255 toon, 128 object, 0 photoreal)
  uint8_t *rsteps;         // trace_order 2: per atlas element the key of its last walk (steps, hit); null otherwise
  uint32_t *rperm;         // trace_order 2: the trace order (atlas indices by descending key)
  uint32_t *rhist;         // trace_order 2: 128 key counts, then 128 scatter cursors
  ProbeDev *probes;
  uint32_t *plevel;        // per probe: voxLevel(s0, c) (rc.ts:210-213), computed once by setupScreen
  const float4 *dirs;      // per cascade, res^2 texel directions dirOf(di, res) (rc.ts:308), computed at creation
  const float4 *idirs;     // the same directions' 1 / d (tiny components clamped as traceVox does), after dirs
  void *rad;               // rays_total atlas elements
  void *sh;                // probes of cascade 0 x 8 atlas elements
  void *irr;               // W*H: float4 (atlas F32 or f32_out, without irr_f16) or rgba16f (uint2)
  uint32_t *counts;        // 80 words
  uint4 *hits;             // optional: per ray (level, brick, bit, tIn bits)
  void *rad_traced;        // optional: copy of the atlas after the trace
  float4 *mavg[2];         // merge: quad averages of the cascade above (ping-pong by cascade parity)
  const float *unorm8;     // [k] = k / 255.0f, [256 + k] = (k / 255.0f) / pi for k = 0..255 (IEEE quotients, host)
  const uint4 *bn_inj;     // multi-bounce on: per voxel the bounce volume's irradiance on its two sides (bnInject)
  const uint32_t *dyn_hdr; // the dynamic layer the traces read (gi_rc_set_dyn; null: none): header, pointers, data
  const uint32_t *dyn_ptr;
  uint32_t *dyn_data;      // (written only by dynInject, objects on)
  const uint32_t *dyn_meta;  // slot -> brick pointer index (dynInject)
  uint32_t dyn_nb;
  uint32_t objects;        // token obj (phase 31): the layer receives the bounce volume and the volume's rays read it
};

// The dynamic layer (dynlayer.ts): header (64 words), a pointer per brick of every level (slot, DYN_EMPTY or
// DYN_DROPPED), two bitsets of wanted bricks (bit order: coarse levels first), slot -> brick, per slot 16 words of its
// non-zero voxels, per voxel of a slot 13 words (P+x P-x P+y P-y P+z P-z, area, area x radiance, area x albedo),
// level 0 in fixed point (x 65536), the levels above as f32 after the resolve.
struct DynDev {
  uint32_t nb, albedo, first, end;   // brick pool; splat the albedo words; dynamic triangles [first, end)
  uint32_t *hdr, *ptr, *bits, *meta, *mask, *data;
  unsigned long long *look;          // the allocation's chained scan: ticket and block states
  uint32_t look_cap, pad;
};
constexpr uint32_t DYN_W = 13, DYN_EMPTY = 0xffffffffu, DYN_DROPPED = 0xfffffffdu;
constexpr float DYN_FIX = 65536.0f;   // level-0 words: fixed point x 65536

// World probes (the method 'world', rc.ts:253-570): per cascade a hash table of probe keys, the probes compacted from
// it in slot order, and the parents each probe merges; the c0 history of two solves.  Probes and atlas entries are laid
// out by capacity (RcDev.c[c].probe_off / rad_off); the counts are device-side.
struct WorldDev {
  uint32_t hash_off[8], hash_mask[8], cap[8], look_off[8];
  uint32_t hash_total, look_total, relocate, hist_h;   // relocate: 0 'gbuffer', 1 'none', 2 'voxel'; hist_h = hash size of c0
  uint32_t *keys;                  // hash_total: key or 0
  uint32_t *slot_probe;            // hash_total: the key's probe or NONE
  uint32_t *parents;               // probes * 8: the probes of the cascade above a probe merges (NONE: none)
  uint32_t *state;                 // [0] the history parity of the current solve, [8 + c] probes of cascade c (min(keys,
                                   // cap)), [16 + c] first ray of cascade c in the trace order (c <= cascades)
  unsigned long long *look;        // the compactions' chained scans, cascade c at look_off[c]
  uint32_t *hist_tab;              // 2 * hist_h: probe + 1 or 0, per parity
  int4 *hist_grid;                 // 2 * cap0: grid point and LOD of each probe, per parity
  float4 *hist_sh;                 // 2 * cap0 * 8: the SH as stored, per parity
};

// The multi-bounce volume (bounce.ts): dx x dy x dz irradiance probes around the camera, rebuilt every frame from the
// voxels, each an ambient cube (six axes: rgb irradiance, alpha the reach along the axis), stored rgba16f in two
// volumes that swap every frame (this frame's is written, the previous one read by the probes' own rays).
struct BounceDev {
  float cell, v0;              // probe spacing (m); the clipmap's level-0 voxel size (the reach tolerance)
  uint32_t dx, dy, dz, rays, div, n, levels;   // n = dx dy dz probes
  const float4 *dirs;          // sfDir(r, rays) (bounce.ts:147-152), computed on the host
  uint2 *vol[2];               // dx * dy * (6 dz + 1) texels, texel (x, y, z) at (z dy + y) dx + x; z = a dz + probe z,
                               // texel (0, 0, 6 dz) holds the volume's origin in probe coordinates
  uint32_t *list;              // [0] probes listed this frame, [1] frame counter, [2] this frame's volume, [4..) list
  uint4 *inj;                  // per voxel: front rg, front b | 0, back rg, back b | 0 (f16 pairs)
  float4 *ray_out;             // n * (rays + 6): each listed probe's ray results (rgb, reach) before the sums
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

// Sun shadow-map raster scratch (shadow.cu) and its output
struct ShadowRaster {
  float *map;                      // S x S depths
  float4 *rec;                     // 4 per triangle: (c0, bias), (c1, i0 | j0 << 16), (c2, bw | bh << 16), unused
  uint32_t *pre, *sums, *counter;  // per triangle chunk prefix within its block; block offsets; [0] chunk total
};

// Per-level constants of a voxel world computed once on the host with the same f32 operations the kernels would do:
// the voxel size ldexpf(v0, L) (a power-of-two scaling, exact) and voxRange's cell limit f2i(G * size * 8 / cell)
// (voxel.ts:295) for voxel cells (cell = size) and brick cells (cell = size * 8).  Call after v0 and G are set.
static inline int32_t f2i_host(float q) {   // f32 -> i32 truncation, saturating (the kernels' f2i)
  return q >= 2147483648.0f ? 2147483647 : (q <= -2147483648.0f ? (-2147483647 - 1) : (q != q ? 0 : (int32_t)q));
}
inline void vox_derived(VoxDev &d) {
  for (uint32_t L = 0; L < 8; L++) {
    volatile float vs = ldexpf(d.v0, (int)L);
    volatile float a = (float)d.G * vs;
    volatile float b = a * 8.0f;
    volatile float cb = vs * 8.0f;
    volatile float qv = b / vs, qb = b / cb;
    volatile float iv = 1.0f / vs;
    d.vs[L] = vs;
    d.inv_vs[L] = iv;
    d.lim_vox[L] = f2i_host(qv);
    d.lim_brick[L] = f2i_host(qb);
  }
}
// Per-level box of the clipmap window after the origins are set, with the f32 operations traceVox uses
// (voxel.ts:124-125: lo = (origin * vs) * 8, hi = lo + (G * vs) * 8; voxInside's lo = origin * (vs * 8) and
// hi = lo + G * (vs * 8), voxel.ts:108-112, are the same numbers, a scaling by 8 being exact).
inline void vox_bounds(VoxDev &d) {
  for (uint32_t L = 0; L < 8; L++) {
    volatile float vs = d.vs[L];
    volatile float gs = (float)d.G * vs;
    volatile float ext = gs * 8.0f;
    for (int a = 0; a < 3; a++) {
      volatile float o = (float)d.origin[L][a];
      volatile float ov = o * vs;
      volatile float lo = ov * 8.0f;
      volatile float hi = lo + ext;
      d.box_lo[L][a] = lo;
      d.box_hi[L][a] = hi;
    }
    d.box_lo[L][3] = d.box_hi[L][3] = 0.0f;
  }
}

}  // namespace gi

cudaError_t gi_launch_vox_build(const gi::VoxDev &v, const gi::SceneDev &s, uint32_t sm_count, cudaStream_t st);
// One build of the dynamic layer (mark .. resolve) in the voxel world's windows; frame: sun, style, light view; shadow:
// the sun's map of `layers` S x S layers, or null (visibility 1)
cudaError_t gi_launch_dyn_build(const gi::DynDev &d, const gi::VoxDev &v, const gi::SceneDev &s, const float *frame,
                                const float *shadow, uint32_t S, uint32_t layers, uint32_t sm_count, cudaStream_t st);
cudaError_t gi_launch_shadow(const gi::SceneDev &s, const float *matrix_dev, uint32_t S, const gi::ShadowRaster &sr,
                             uint32_t sm_count, cudaStream_t st);
// ev (optional, 5 events): recorded after giBuild (setupScreen), giTrace, giMerge (merge + projectSH), giGather.
// Kernel launch with programmatic dependent launch allowed: the next kernel in the stream (or graph) may be scheduled
// while this one's last blocks drain, hiding the launch gap between dependent kernels.  Every kernel launched this
// way starts with grid_dep_wait(), so nothing it reads or writes is touched before its predecessor has finished.
template <typename... P, typename... Args>
inline cudaError_t gi_launch(void (*k)(P...), dim3 grid, dim3 block, cudaStream_t st, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k, args...);
}
#define GI_TRY(...)                                   \
  do {                                                \
    cudaError_t e_ = (__VA_ARGS__);                   \
    if (e_ != cudaSuccess) return e_;                 \
  } while (0)

// Launch shapes of the cascade passes (the result does not depend on them)
struct RcLaunch { uint32_t trace_blocks, gather_shape, merge_threads; };

// A batch of solves run pass by pass: one launch per pass over the work of every solve.  The solves' descriptors and
// the work prefixes live in device memory; each block (each 32-ray fetch of the trace) belongs to one solve, found by
// a binary search of the prefix.
namespace gi {
struct BatchDev {
  const RcDev *rc;
  const VoxDev *vox;
  uint32_t n, max_casc;
  const uint32_t *setup_blk;    // n + 1: first setup block of each solve (256 probes a block)
  const uint32_t *ray_pre;      // n + 1: first ray of each solve in the batch's trace order (rays padded to 32)
  const uint32_t *merge_blk;    // max_casc x (n + 1): per merge step k (cascade C - 1 - k), first block of each solve
  const uint32_t *gather_blk;   // n + 1: first gather block of each solve
  uint32_t *counter;            // [0]: rays handed out by the batched trace
};
// host copies of the launch sizes
struct BatchSizes { uint32_t setup_blocks, merge_blocks[8], gather_blocks, atlas, P0; };
}  // namespace gi
cudaError_t gi_launch_batch_passes(const gi::BatchDev &b, const gi::BatchSizes &z, uint32_t sm_count, cudaStream_t st);
// The world probes' device tables (segment sample positions); called before their first solve
cudaError_t gi_world_tables();
// w: world probes (nullptr: screen probes)
cudaError_t gi_launch_rc_solve(const gi::RcDev &r, const gi::VoxDev &v, uint32_t sm_count, cudaStream_t st,
                               cudaEvent_t *ev = nullptr, const RcLaunch *ls = nullptr, const gi::BounceDev *bn = nullptr,
                               const gi::WorldDev *w = nullptr);
uint32_t gi_raster_tiles(uint32_t W, uint32_t H);
cudaError_t gi_launch_gbuffer(const gi::SceneDev &s, const float *frame_dev, uint32_t W, uint32_t H, float *depth,
                              uint2 *normal, uint8_t *tag, const gi::RasterDev &rd, uint32_t sm_count, cudaStream_t st);
cudaError_t gi_launch_normal_f32_to_f16(const float4 *src, uint2 *dst, uint32_t n, cudaStream_t st);
cudaError_t gi_launch_normal_rgb_to_rgba(const uint16_t *src, uint2 *dst, uint32_t n, cudaStream_t st);
cudaError_t gi_launch_iota(uint32_t *dst, uint32_t n, cudaStream_t st);
// Base colour textures: rgba8 (sRGB rgb, linear alpha) decoded to linear float4 through lut, then every layer's mip
// chain (levels of size >> k, per texels a layer), on the null stream
cudaError_t gi_launch_tex_build(const uint8_t *rgba8, const float *lut, float4 *tex, uint32_t size, uint32_t levels,
                                uint32_t layers, uint32_t per);
cudaError_t gi_launch_irr_to_f32(const gi::RcDev &r, float4 *dst, cudaStream_t st);
cudaError_t gi_launch_init_dirs(const gi::RcDev &r, float4 *dirs, uint32_t ndirs, cudaStream_t st);
// FP64 reference of merge + SH + gather from the f32 traced atlas: rad64 rays_total x 4 doubles, sh64 27 doubles per
// cascade-0 probe, irr64 W*H x 4 doubles.
cudaError_t gi_launch_merge_gather_f64(const gi::RcDev &r, const float4 *traced, void *rad64, double *sh64, void *irr64,
                                       uint32_t f16_cascades, cudaStream_t st);
