/*
 * gi_oracle — CPU restatement of the real-time-gi-lab GI hot path, used ONLY as test infrastructure.
 *
 * This library is the checker for the CUDA path: tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg are the only callers.  It is never linked into, or called by, the product library.
 *
 * It restates, sequentially and in plain C, the WGSL of the reference renderer (owoDra/real-time-gi-lab):
 *   - the voxel clipmap rebuild            src/core/voxel.ts:205-620 (build WGSL), :868-892 (writeUniform)
 *   - the two-level voxel DDA              src/core/voxel.ts:75-203  (voxRank, voxAt, voxLevelFor, traceVox)
 *   - hit shading                          src/core/rc.ts:95-141, src/core/style.ts:16-26
 *   - screen probes, trace, merge, SH,     src/core/rc.ts:210-310, :572-622, :679-774, :819-829, :929-954
 *     gather
 *   - the headless G-buffer raster         src/core/gbuffer.ts:82-103 (conventions only; the reference draws it
 *                                          with a graphics pipeline, restated here as a scanline raster)
 *   - the sun shadow map and voxSun        src/core/lighting.ts:133-189, frame.ts:35-52, voxel.ts:633-671
 *   - world probes (method 'world')        src/core/rc.ts:248-570, :688-708, :775-927
 *
 * Arithmetic follows the WGSL expression order exactly (left-associative, no contraction: build with
 * -ffp-contract=off).  Where the WGSL leaves a builtin implementation-defined, the choice made here is stated
 * at the function (normalize = v / sqrt(dot), round(log2(x)) exact, pack* = the WGSL spec formulas, f16 = RNE).
 *
 * Pinning: the reference cannot run here (WGSL through Dawn/Vulkan on Node).  The voxel build is pinned against
 * the brick/voxel counters the reference recorded for its procedural leak rooms
 * (docs/reference/measurements/s2-voxel-stratabrick/leak-<t>/world-32-voxel.summary.json, static.vox); the
 * tracer, merge and gather have no recorded reference output for a reproducible scene: parity unpinned there.
 */
#ifndef GI_ORACLE_H
#define GI_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_HDR 64
#define ORC_EMPTY 0xffffffffu
#define ORC_DROP 0xfffffffeu
#define ORC_MARK 0xfffffffdu

/* Material: baseColorFactor, flags (1 alpha mask, 2 double-sided, 4 toon, 8 object; scene_gpu.ts:95-104),
 * alpha cutoff, and the emissive radiance this build adds (the reference has no emission). 48 bytes. */
typedef struct {
  float base_color[4];
  uint32_t flags;
  float alpha_cutoff;
  float emissive[3];
  uint32_t base_color_tex;   /* 1 + texture layer; 0 untextured */
  uint32_t reserved[2];
} orc_material;

typedef struct {
  const float *pos;        /* xyz per vertex */
  const float *nrm;        /* xyz per vertex */
  uint32_t nverts;
  const uint32_t *tri;     /* (i0, i1, i2, material) per triangle: triangleTable, voxel.ts:730 */
  uint32_t ntris;
  const orc_material *mats;
  uint32_t nmats;
  /* World work items (world.ts; voxel.ts:270-288), NULL items: one contiguous item over every row, instance 0.
   * items: nitems x (first thread, source, instance, first level), the source an offset into lists or
   * 0x80000000 | first row; a triangle's key is instance * key_stride + row; inst: 4 floats per instance (offset). */
  const uint32_t *items;
  uint32_t nitems, threads, key_stride, ninst;
  const uint32_t *lists;
  const float *inst;
  /* The rasters (G-buffer, shadow map): rows [0, ndraw) at draw_ninst instances (4 floats each, draw_inst; NULL:
   * one instance at the origin), drawn triangle i * ndraw + row; ndraw 0: every row */
  uint32_t ndraw, draw_ninst;
  const float *draw_inst;
  /* Base colour textures (tex.c): a uv per vertex (2 floats), every layer's mip chain of linear rgba f32 texels
   * (orc_tex_build); uv or tex NULL: every material untextured */
  const float *uv;
  const float *tex;
  uint32_t tex_size, tex_levels, tex_layers, tex_layer_texels;
} orc_scene;

/* Textures (tex.c): levels of a size (and texels a layer); decode + mip chain of `layers` rgba8 images into out
 * (layers x per-layer texels x 4 floats); 1 + layer of a material's texture or 0; a bilinear sample at a level; the uv
 * at barycentric weights. */
uint32_t orc_tex_levels(uint32_t size, uint32_t *per_layer);
void orc_tex_build(const uint8_t *rgba8, uint32_t size, uint32_t layers, float *out);
uint32_t orc_tex_layer_of(const orc_scene *s, const orc_material *m);
void orc_tex_sample(const orc_scene *s, uint32_t layer1, float u, float v, uint32_t lod, float out[4]);
void orc_tri_uv(const orc_scene *s, const uint32_t idx[3], float wx, float wy, float wz, float uv[2]);
/* The rasters' alpha test (gbuffer.ts:94, the shadow pass's discard): a masked material's alpha at barycentric weights
 * (the texture at level 0 times the factor; the factor alone untextured) against the cutoff; 1 when kept. */
int orc_raster_alpha_ok(const orc_scene *s, const uint32_t idx[4], float wa, float wb, float wc);

/* Voxel world state, laid out exactly as the CUDA path lays it out in device memory (struct of arrays). */
typedef struct {
  /* parameters (VoxParams, voxel.ts:31) */
  float v0;
  uint32_t levels, G, max_bricks, max_voxels;
  uint32_t big_cap;                /* entries per big-triangle segment (BIG_CAP, voxel.ts:224) */
  uint32_t coarse_from_triangles;  /* 1: every level voxelised from the triangles (the pre-phase-21 build); pin runs only */
  int32_t origin[8][4];            /* per level: first brick of the window (world brick coordinates) */
  /* buffers (caller-allocated) */
  uint32_t *hdr;                   /* ORC_HDR counter words (voxel.ts:11) */
  uint32_t *ptr;                   /* levels * G^3 brick pointers */
  uint32_t *occ;                   /* max_bricks * 16 occupancy words */
  uint32_t *base;                  /* max_bricks: first attribute */
  uint32_t *code;                  /* max_bricks: level << 27 | bx << 18 | by << 9 | bz */
  uint32_t *rep;                   /* max_bricks * 512: representative triangle + 1 */
  uint32_t *big;                   /* 16 * big_cap: segments 0-7 voxBits per level, 8-15 markBricks per level */
  uint32_t *attr;                  /* max_voxels * 4: albedo, normal, emissive rg (f16x2), emissive b (f16) */
  float *plane;                    /* max_voxels: representative plane offset from the voxel centre */
  float *sunvis;                   /* max_voxels: sun visibility of the voxel (1 when no visibility pass runs) */
  const float *bn_inj;             /* NULL, or max_voxels * 6: the bounce volume's irradiance on the voxel's two sides
                                      (front rgb, back rgb, f16 values; orc_bounce_frame writes it) */
  const struct orc_dyn_s *dyn;     /* NULL, or the dynamic layer the cascades' traces read (traceDyn, rc.ts:227-231) */
} orc_vox;

/* The dynamic layer (src/core/dynlayer.ts), laid out as the CUDA path lays it out in device memory: the 64 header
 * words (dynlayer.ts:53-55), a pointer per brick of every level (slot, DYN_EMPTY or DYN_DROPPED), the two brick
 * bitsets (bit order: coarse levels first), slot -> brick, per slot 16 words of its non-zero voxels, per voxel of a
 * slot 13 words (P+x P-x P+y P-y P+z P-z, area, area x radiance rgb, area x albedo rgb), level 0 in fixed point
 * (x 65536), levels above as f32 after the resolve. */
typedef struct orc_dyn_s {
  uint32_t nb;                     /* brick pool (DYN_MAX_BRICKS) */
  uint32_t albedo;                 /* 1: the splat writes the albedo words (configs whose objects receive light) */
  uint32_t *hdr;                   /* 64 */
  uint32_t *ptr;                   /* levels * G^3 */
  uint32_t *bits;                  /* 2 * levels * G^3 / 32 */
  uint32_t *meta;                  /* nb */
  uint32_t *mask;                  /* nb * 16 */
  uint32_t *data;                  /* nb * 512 * 13 */
} orc_dyn;

/* createDynLayer's initial state (dynlayer.ts:690-694) over the voxel world's levels and G. */
void orc_dyn_init(const orc_vox *vx, orc_dyn *dl);
/* One build (mark .. resolve, dynlayer.ts:592) of the dynamic triangles [first, end) of the scene in the voxel world's
 * current windows, shaded with the frame's sun and style and the sun shadow map (map NULL: visibility 1). */
int orc_dyn_build(const orc_scene *s, const orc_vox *vx, orc_dyn *dl, uint32_t first, uint32_t end, const float *frame,
                  const float *map, uint32_t S);
/* traceDyn (dynlayer.ts:118-162): covered radiance (rgb) and coverage of [t0, t1] along d from o, cone width k * t. */
void orc_trace_dyn(const orc_vox *vx, float o[3], float d[3], float t0, float t1, float k, float out[4]);
/* log2 as this library defines it (the reference's WGSL log2 is implementation-defined). */
float orc_log2(float x);

/* Host writeUniform (voxel.ts:868-876): per level origin = floor(eye / bs) - G/2, bs = v0 * 2^L * 8 (f64 host math). */
void orc_vox_origins(float v0, uint32_t levels, uint32_t G, const double eye[3], int32_t origin_out[8][4]);
/* The whole rebuild (VOX_STAGES minus sun): clear .. resolveAttr.  Returns 0. */
int orc_vox_build(const orc_scene *s, orc_vox *vx);

/* Cascade layout (rc.ts:1024-1035) for the screen method. */
typedef struct {
  uint32_t probe_off, cap, rad_off, res, tile_size, tiles_x, tiles_y, pad;
  float b0, b1, pad2[2];
} orc_casc;

typedef struct {
  uint32_t cascades;
  orc_casc c[8];
  /* wp: voxScale, voxOffset, levelMap, voxSkip */
  float vox_scale, vox_offset, level_map, vox_skip;
  uint32_t dda_cap;       /* DDA step cap (the reference hard-codes 1024, voxel.ts:142) */
  uint32_t stats;         /* 0 off, 1 DDA step counters (rc.ts:232-235) */
  uint32_t atlas;         /* 0: f32 storage, 1: f16 (the reference's rgba16 packing), 2: bf16 */
  uint32_t f32_out;       /* 1: SH and irradiance stored as f32 whatever the atlas */
  uint32_t irr_f16;       /* 1: irradiance stored as rgba16float whatever the atlas and f32_out */
} orc_layout;

/* One probe (rc.ts:157): pos.xyz + s0, nrm.xyz + view depth, grid. 48 bytes. */
typedef struct { float pos[4]; float nrm[4]; int32_t grid[4]; } orc_probe;

typedef struct {
  const float *frame;       /* 160 words (packFrame, frame.ts:76) */
  uint32_t width, height;
  const float *depth;       /* W*H reversed-Z depth (0 = background) */
  const float *normal;      /* W*H*4, the G-buffer normal as read from its rgba16float texture */
  const uint8_t *tag;       /* W*H style tags (the albedo's alpha byte: 255 toon, 128 object, 0), or NULL (all 0) */
} orc_gbuf;

typedef struct {
  orc_probe *probes;        /* sum of caps */
  float *rad;               /* sum over cascades of cap * res^2 * 4 (values after the atlas rounding) */
  float *sh;                /* cap0 * 32 (27 used), after the atlas rounding */
  float *irr;               /* W*H*4 (rgb + alpha), after the output rounding (f16 unless atlas = f32) */
  uint32_t *counts;         /* 80 words (rc.ts:173-175) */
  /* optional debug (may be NULL): per traced ray of every cascade, the hit: level, brick pointer, bit, tIn bits */
  uint32_t *hit;            /* 4 words per ray, rad order */
} orc_rc_out;

/* setupScreen (all cascades) + trace (all cascades).  rad holds the traced (unmerged) intervals. */
int orc_rc_trace(const orc_vox *vx, const orc_layout *ly, const orc_gbuf *g, orc_rc_out *o);
/* mergeScreen (N-1 .. 0) + projectSH + gatherScreen on o->rad (in place). */
int orc_rc_merge_gather(const orc_layout *ly, const orc_gbuf *g, orc_rc_out *o);
/* The same in float64 throughout (no intermediate rounding): the FP64 accuracy oracle of the merge and gather.
 * rad_in: traced intervals (f32, unmerged).  irr_out: W*H*4 doubles. */
int orc_rc_merge_gather_f64(const orc_layout *ly, const orc_gbuf *g, const orc_probe *probes, const float *rad_in,
                            double *irr_out);
/* The same with the atlas storage of the cascades in bit mask f16_cascades rounded to f16 (ties to even): their traced
 * intervals, and above cascade 0 their merged radiances as the cascade below reads them; every stage in double. */
int orc_rc_merge_gather_f64_rounded(const orc_layout *ly, const orc_gbuf *g, const orc_probe *probes,
                                    const float *rad_in, unsigned f16_cascades, double *irr_out);

/* Headless G-buffer: depth (reversed Z, infinite far) and the shading normal (interpolated vertex normal,
 * flipped to the viewer for back faces), one sample at each pixel centre.  normal_out is rgba, w = 0.
 * tri_out (optional) receives the winning triangle per pixel (0xffffffff: none). */
int orc_raster_gbuffer(const orc_scene *s, const float *frame, uint32_t width, uint32_t height, float *depth_out,
                       float *normal_out, uint32_t *tri_out);

/* Sun shadow map (lighting.ts:133-140, 175-189, restated as a per-texel-centre raster of the light's orthographic
 * clip space; the rules are stated in shadow.c): per layer S*S depths, 1 where nothing is drawn; layer 0 from the
 * frame's lightViewProj (frame words 64-79), layer 1 (frames with shadow.x = 2, word 156) from lightViewProjFar
 * (words 140-155) at map + S*S. */
int orc_shadow_render(const orc_scene *s, const float *frame, uint32_t S, float *map);
/* shadowTap (frame.ts:35-52): the 'less-equal' comparison of x's biased light depth (bias: frame word 157, layer 1:
 * 158) with the layer x projects into, bilinear over the four texels around it; 1 outside every layer. */
float orc_sun_tap(const float *frame, const float *map, uint32_t S, const float x[3]);
/* toonReceive (style.ts:30-42) on c = (c0, c1y, c1z, c1x) as 12 floats: out = (E rgb, band, contrast). */
void orc_toon_receive(const float c[12], const float n[3], float soft, float out[5]);
/* The frame's layer count: 2 when shadow.x (word 156) >= 1.5, else 1. */
uint32_t orc_shadow_layers(const float *frame);
/* voxSun (voxel.ts:633-671): the sun visibility of every occupied voxel of a built world (after orc_vox_build). */
int orc_vox_sun(orc_vox *vx, const float *frame, const float *map, uint32_t S);

/* The multi-bounce volume (bounce.ts): dx * dy * dz probes around the camera, each an ambient cube (6 axes x rgba),
 * stored in f16 (kept here as the f16 values in floats), two volumes swapped every frame.  Caller-allocated buffers. */
typedef struct {
  float cell, v0;                 /* probe spacing; the clipmap's level-0 voxel size */
  uint32_t dx, dy, dz, rays, div;
  const float *dirs;              /* rays * 4: sfDir(r, rays) (the same table the GPU path uses) */
  float *vol[2];                  /* dx * dy * (6 dz + 1) * 4 each, texel (x, y, z) at ((z dy + y) dx + x) * 4 */
  uint32_t *list;                 /* 4 + dx dy dz words: [0] listed, [1] frame counter, [2] this frame's volume */
  uint32_t objects;               /* token obj (phase 31): with a dynamic layer in the voxel world (vx->dyn), its
                                     voxels receive the previous volume first (dynInject) and the volume's irradiance
                                     rays read it (bnTraceDyn) */
} orc_bounce;
/* One frame of the volume (Bounce.encode, bounce.ts:356-368) over a built voxel world: (objects: dynInject into
 * vx->dyn,) clear, classify, update, inject (into inj_out, max_voxels * 6).  The list order is the probe order (the GPU's atomics order it otherwise;
 * the result does not depend on it). */
int orc_bounce_frame(orc_bounce *b, const orc_vox *vx, const float *frame, float *inj_out);

/* World probes (method 'world', rc.ts:253-570, 688-708, 775-927; world.c states the choices it makes).  The layout
 * reuses orc_layout for the per-cascade probe / atlas offsets, capacities (caps), resolutions and intervals. */
typedef struct {
  orc_layout base;
  uint32_t hash_off[8], hash_mask[8];   /* per cascade: its hash table's first slot, size - 1 (size = nextPow2(2 cap)) */
  uint32_t hash_total;
  uint32_t relocate;                     /* 0 'gbuffer' (relocate), 1 'none', 2 'voxel' (relocateVox + segOccluded) */
} orc_wlayout;
/* State a world solve keeps across solves (caller-allocated, zeroed before the first solve). */
typedef struct {
  uint32_t *keys, *slot_probe;   /* hash_total each */
  uint32_t *parents;             /* probes * 8: the upper probes each probe merges (NONE = 0xffffffff) */
  uint32_t *hist_tab;            /* 2 * H0 (H0 = hash_mask[0] + 1): the c0 history's tables, probe index + 1 or 0 */
  int32_t *hist_grid;            /* 2 * cap0 * 4: per probe of each parity its grid point and LOD */
  float *hist_sh;                /* 2 * cap0 * 32: per probe of each parity its SH as stored */
  uint32_t hist_par;             /* parity of the last solve (0 before the first) */
} orc_wstate;
/* One solve: clearKeys .. linkParents, trace, mergeWorld N-1 .. 0, projectSH with the history, gatherWorld.
 * o->probes / rad / sh / irr / counts / hit as for the screen method (rad indexed by the cap-based offsets). */
int orc_world_solve(const orc_vox *vx, const orc_wlayout *wl, const orc_gbuf *g, orc_wstate *ws, orc_rc_out *o);
uint32_t orc_hash32(uint32_t x);
int32_t orc_lod_for(const float *frame, float dist);

/* WGSL builtins as the oracle defines them (exported for the known-answer tests). */
uint32_t orc_pack4x8unorm(const float v[4]);
uint32_t orc_pack2x16snorm(float a, float b);
uint16_t orc_f32_to_f16(float x);
float orc_f16_to_f32(uint16_t h);
uint16_t orc_f32_to_bf16(float x);
float orc_bf16_to_f32(uint16_t h);
int orc_tri_box(const float c[3], const float h[3], const float a[3], const float b[3], const float cc[3]);
uint32_t orc_round_log2(float x);
float orc_gi_exp(float x);

#ifdef __cplusplus
}
#endif
#endif
