/*
 * gi.h — C-ABI of the B200 GI hot path: the voxel clipmap rebuild, the voxel DDA radiance cascades, and the cascade
 * merge plus irradiance gather of the real-time-gi-lab renderer, as sm_100a CUDA kernels.
 *
 * The entry points replace the WebGPU dispatch of the reference's `vox` and `giBuild/giTrace/giMerge/giGather`
 * passes (src/core/rcrun.ts:18, :283-298).  They mirror the reference's two host objects:
 *   VoxWorld  src/core/voxel.ts:710-727   -> gi_vox_*   (createVoxWorld voxel.ts:746)
 *   Rc        src/core/rc.ts:980-992      -> gi_rc_*    (createRc rc.ts:1019)
 * plus the scene upload (src/core/scene_gpu.ts:56 uploadScene) and the frame uniform (src/core/frame.ts:76 packFrame).
 *
 * Conventions.  Every function returns a gi_status (0 = GI_OK, negative = error); gi_last_error() returns the
 * message of the calling thread's last error (the reference throws `new Error(msg)`, e.g. voxel.ts:749).  Pool
 * overflows are counters, not errors (voxel.ts:463, :586).  Handles own their device memory and free it in
 * gi_*_destroy (voxel.ts:923, rc.ts:1234).  Host pointers are borrowed for the duration of the call.  `stream` is a
 * cudaStream_t (NULL: the legacy default stream); work is stream-ordered and asynchronous except where a function
 * says it synchronises.  A handle may be used by one host thread at a time.
 */
#ifndef GI_H
#define GI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GI_ABI_VERSION 1

typedef enum {
  GI_OK = 0,
  GI_ERR_INVALID = -1,   /* bad argument or unsupported parameter combination */
  GI_ERR_OOM = -2,       /* device or pinned host allocation failed */
  GI_ERR_CUDA = -3,      /* a CUDA runtime error (message in gi_last_error) */
  GI_ERR_TIMEOUT = -4,   /* a bounded device wait gave up */
  GI_ERR_OVERFLOW = -5,  /* a fixed-capacity structure of the call itself overflowed */
  GI_ERR_STATE = -6      /* call out of order (e.g. solve before a frame was set) */
} gi_status;

/* Cascade atlas storage.  F16 is the reference's own packing (pack2x16float, rc.ts:309-310, SH rc.ts:768-771,
 * rgba16float irradiance rc.ts:1073); F32 keeps every intermediate in f32; BF16 stores the atlases as bfloat16.
 * Accumulation is f32 in every mode. */
typedef enum { GI_ATLAS_F32 = 0, GI_ATLAS_F16 = 1, GI_ATLAS_BF16 = 2 } gi_atlas;

typedef struct gi_ctx gi_ctx;
typedef struct gi_scene gi_scene;
typedef struct gi_vox gi_vox;
typedef struct gi_rc gi_rc;
typedef struct gi_dyn gi_dyn;

/* Material (scene_gpu.ts:95-106 `struct Material`): base colour factor, flags (1 alpha mask, 2 double-sided,
 * 4 toon, 8 object), alpha cutoff.  emissive: radiance added at a voxel hit (no counterpart in the reference,
 * whose materials do not emit).  base_color_tex: 1 + the base colour texture layer (gi_scene_set_textures) the
 * colour is sampled from and multiplied by the factor; 0: untextured, the factor alone (the reference's white
 * default layer, layers.x = 0).  48 bytes. */
typedef struct {
  float base_color[4];
  uint32_t flags;
  float alpha_cutoff;
  float emissive[3];
  uint32_t base_color_tex;
  uint32_t reserved[2];
} gi_material;

/* VoxParams (voxel.ts:31-38).  levels <= 8; G a multiple of 4, <= 256 (brick coordinates are packed in 9 bits). */
typedef struct {
  double v0;             /* finest voxel size (m); the window origins use it in f64 like the reference's numbers,
                            the kernels in f32 like its uniform */
  uint32_t levels;
  uint32_t G;
  uint32_t max_bricks;
  uint32_t max_voxels;
  uint32_t dyn_bricks;   /* accepted for parity with VoxParams; the dynamic layer is not part of this library */
  uint32_t reserved;
} gi_vox_params;

/* The RcParams fields the screen-probe / voxel-tracer path reads (rc.ts:42-84; parseConfig runner/configs.ts:47). */
typedef struct {
  uint32_t cascades;     /* <= 8 */
  uint32_t P;            /* pixels between c0 probes (tile size of cascade 0) */
  float k_interval;      /* c0 interval length in units of s0 */
  float vox_scale;       /* c0 voxel size relative to the c0 probe spacing */
  float vox_offset;      /* voxel traces start vox_offset voxels along the probe normal */
  float vox_skip;        /* occupied voxels entered within vox_skip voxels are ignored */
  float level_map;       /* voxel level grows by level_map per cascade */
  uint32_t res_cap;      /* directions stop growing above this cascade */
  uint32_t dda_cap;      /* DDA step cap (the reference hard-codes 1024, voxel.ts:142) */
  uint32_t stats;        /* 0 off, 1 DDA step counters (rc.ts:232-235) */
  uint32_t atlas;        /* gi_atlas */
  uint32_t f32_out;      /* 1: SH and irradiance stored as f32 whatever the atlas (the reference stores both f16,
                            rc.ts:768-773, :1073); 0: stored like the atlas, f16 for F16/BF16 */
  uint32_t irr_f16;      /* 1: the irradiance stored as rgba16float whatever the atlas and f32_out (the format of the
                            reference's rc.irr texture, rc.ts:1073): every pass before the store keeps its precision,
                            the store rounds to nearest even; half the bytes of an f32 readback */
  uint32_t reserved[3];
} gi_rc_params;

/* World probes (RcParams.method 'world', rc.ts:253-570): probes on a world-space grid registered from the G-buffer's
 * pixels, LOD by distance (spacing sMin * 2^lod, frame word 104; P, frame word 106), kept in one hash table per cascade,
 * relocated out of the surface, merged through their parents, with a history on the c0 SH (rc.ts:775-816). */
enum { GI_RELOCATE_GBUFFER = 0, GI_RELOCATE_NONE = 1, GI_RELOCATE_VOXEL = 2 };
typedef struct {
  uint32_t relocate;     /* params.relocate: GI_RELOCATE_GBUFFER (default), _NONE, _VOXEL (config token vrel) */
  uint32_t caps[8];      /* params.caps: probes per cascade (default 2^18, 2^16, 2^14, 2^12, 2^11, 2^10, 2^9, 2^8) */
  uint32_t reserved[3];
} gi_world_params;

int gi_version(void);
const char *gi_status_string(int status);
/* Message of the calling thread's last failed call ("" when none). */
const char *gi_last_error(void);

/* ---- context --------------------------------------------------------------------------------------------------- */
/* Binds CUDA device `device` (env.ts createNativeDevice is the reference's counterpart). */
int gi_ctx_create(int device, gi_ctx **out);
int gi_ctx_destroy(gi_ctx *ctx);

/* ---- scene (scene_gpu.ts:56 uploadScene, voxel.ts:730 triangleTable) --------------------------------------------- */
/* pos, nrm: nverts x 3 floats.  tri4: ntris x (i0, i1, i2, material), absolute vertex indices. */
int gi_scene_upload(gi_ctx *ctx, const float *pos, const float *nrm, uint32_t nverts, const uint32_t *tri4,
                    uint32_t ntris, const gi_material *mats, uint32_t nmats, gi_scene **out);
/* Base colour textures (scene_gpu.ts:60-89; voxel.ts:325-336 surfaceAt; gbuffer.ts:90-94 and the shadow pass's
 * alpha test; dynlayer.ts:451-454 shadeSample).  rgba8: layers x size x size texels, rgb sRGB-encoded and alpha
 * linear (the reference's rgba8unorm-srgb), row-major; uv: nverts x 2 floats per vertex.  The library decodes the
 * texels to linear f32 and builds each layer's mip chain on the device (level k + 1: the mean of 2 x 2 texels of level
 * k, sums in a fixed order); a sample is bilinear within one level, repeat addressing, texel centres at (i + 0.5) /
 * size.  The voxel passes sample at level 3 + L (the reference's textureSampleLevel), the rasters' alpha test and the
 * dynamic layer likewise at their levels (G-buffer and shadow map: level 0, where the reference's hardware picks a
 * level from derivatives).  size a power of two, 1 .. 4096; layers >= 1; the data is copied (stream-ordered on the
 * null stream, synchronised before return).  Calling it again replaces the textures. */
int gi_scene_set_textures(gi_scene *scene, const uint8_t *rgba8, uint32_t size, uint32_t layers, const float *uv);
/* Replaces vertices [first, first + count) (the per-frame pose of moving objects, rcrun.ts:206-214). */
int gi_scene_update_vertices(gi_scene *scene, uint32_t first, uint32_t count, const float *pos, const float *nrm,
                             void *stream);
/* The rasters (G-buffer, shadow map) draw rows [0, count); rows past it are voxelised only (a world's clustered
 * copies, world.ts:20-24).  All rows by default. */
int gi_scene_set_draw_count(gi_scene *scene, uint32_t count);
/* The rows the voxel rebuild reads: [0, count) (createVoxWorld's firstDynamicTri, voxel.ts:746); the rows after it are
 * the dynamic triangles, which go to a dynamic layer (gi_dyn_create) instead.  count = the scene's rows: all (the
 * default).  The rasters still draw every row. */
int gi_scene_set_static_count(gi_scene *scene, uint32_t count);
/* The rasters draw those rows at n instance offsets (3 floats each, instance 0 at the origin; n <= 1: once), drawn
 * triangle i * count + row for instance i (the instanced draws of a world, world.ts:4-6). */
int gi_scene_set_draw_instances(gi_scene *scene, const float *offsets, uint32_t n);
int gi_scene_destroy(gi_scene *scene);

/* ---- voxel world (voxel.ts VoxWorld) ------------------------------------------------------------------------------ */
int gi_vox_create(gi_scene *scene, const gi_vox_params *params, gi_vox **out);
/* update(eye) (voxel.ts:868-892 writeUniform): the per-level windows around eye (f64, as the reference's numbers). */
int gi_vox_update(gi_vox *vox, const double eye[3]);
/* Worlds (world.ts; voxel.ts:270-288, :765-885): the scene's rows placed at ninst instance offsets (3 floats each,
 * instance 0 at the origin), chunk row lists `lists` (table rows), key_stride = the scene's rows (a triangle's key is
 * instance * key_stride + row).  From then on the rebuild reads only this frame's work items (gi_vox_set_items), not
 * every row.  ninst 0 returns to every row once. */
int gi_vox_set_world(gi_vox *vox, const float *instances, uint32_t ninst, const uint32_t *lists, uint32_t nlists,
                     uint32_t key_stride);
/* This frame's work items (selectItems, world.ts:179-199): nitems x (first thread, source, instance, first level), the
 * source an offset into the lists or 0x80000000 | first row of a contiguous range; threads = the items' triangles.
 * Set after gi_vox_update (the items follow the windows); a captured graph keeps the thread count it was captured
 * with. */
int gi_vox_set_items(gi_vox *vox, const uint32_t *items, uint32_t nitems, uint32_t threads);
/* encode(pass) (voxel.ts:897-899): the whole rebuild, clear .. resolveAttr, stream-ordered. */
int gi_vox_build(gi_vox *vox, void *stream);
/* readCounters (voxel.ts:908-918): the 64 header words (0 bricks marked, 1 voxels, 2-4 brick/big/voxel overflow,
 * 6 nonzero if a chained scan of the rebuild stopped waiting for a block (never expected), 8-15 bricks per level,
 * 16-23 voxBits big triangles per level, 24-31 markBricks big triangles per level).
 * Synchronises the stream.  The words are copied out in every case; returns GI_ERR_TIMEOUT when word 6 is set (the
 * rebuild's state is then not valid), as the reference's counters report its overflows (voxel.ts:463,586). */
int gi_vox_read_counters(gi_vox *vox, uint32_t hdr[64], void *stream);
/* Test hook for failure detection, no counterpart in the reference: part `part` (0-based, in ticket order) of the
 * next rebuilds' brick-allocation scan publishes nothing, so the part after it waits until its bounded wait gives up
 * (well under a second) and sets header word 6; gi_vox_read_counters then returns GI_ERR_TIMEOUT.  part < 0 turns it
 * off.  A held rebuild's voxel state is not valid; nothing reads outside its buffers. */
int gi_vox_debug_hold_scan(gi_vox *vox, int32_t part);
/* usedBytes (voxel.ts:919-922) of the last counters read: persistent and build-temporary bytes. */
int gi_vox_used_bytes(gi_vox *vox, uint64_t *persistent, uint64_t *build_temp);
/* Copies the voxel world's buffers to the host (any pointer may be NULL).  Sizes: ptr levels*G^3, occ
 * max_bricks*16, base/code max_bricks, rep max_bricks*512, attr max_voxels*4, plane/sunvis max_voxels words.
 * Synchronises the stream. */
int gi_vox_read_state(gi_vox *vox, uint32_t *ptr, uint32_t *occ, uint32_t *base, uint32_t *code, uint32_t *rep,
                      uint32_t *attr, float *plane, float *sunvis, void *stream);
int gi_vox_destroy(gi_vox *vox);
/* Bytes of device memory a voxel world / a scene holds (voxel.ts VoxWorld.bytes; the serving loop's HBM budget). */
int gi_vox_bytes(gi_vox *vox, uint64_t *bytes);
int gi_scene_bytes(gi_scene *scene, uint64_t *bytes);
/* Capacity, in entries, of the G-buffer raster's per-tile triangle lists (default 8 per triangle, at least 2^20).
 * Triangles past it are tested by every tile instead: slower, the same G-buffer.  Frees the old list (which waits for
 * work still using it). */
int gi_scene_set_raster_capacity(gi_scene *scene, uint32_t entries);
/* Rigid objects (no counterpart in the reference's static scene upload; its moving objects go through dynlayer.ts):
 * vertices [first, first + verts_per_object * n_objects) become n_objects rigid bodies whose current vertices are
 * their rest vertices (copied now) under a per-object transform.  gi_scene_rigid_upload copies n_objects row-major
 * 3x4 transforms [R | t] (12 floats each; R a rotation) from host memory (pinned: asynchronous); gi_scene_rigid_apply
 * writes position = R * rest + t and normal = R * rest normal on the device (graph-capturable). */
int gi_scene_rigid_define(gi_scene *scene, uint32_t first, uint32_t verts_per_object, uint32_t n_objects);
int gi_scene_rigid_upload(gi_scene *scene, const float *m34, void *stream);
int gi_scene_rigid_apply(gi_scene *scene, void *stream);
/* The voxel rebuild for callers that cannot allocate device memory (no counterpart in the reference).  Some callers
 * cannot call cudaMalloc: a renderer that hands out every buffer from its own fixed device pool, a thread that is
 * capturing a CUDA graph, a serving loop that must not stall the GPU with an allocation mid-request.  This entry point
 * takes the scene and every output in the caller's device memory and allocates nothing: its scratch (representatives,
 * big-triangle lists, scan sums) is a static device array of 14.2 MiB that the library holds on every GPU it is loaded
 * on.  Limits: max_bricks <= 4096, levels * G^3 <= 2^25, 65,536 big triangles per list (more count as bigOverflow,
 * header word 3; gi_vox_build keeps up to 262,144, so past 65,536 the two give different voxels and only this one
 * reports the overflow).  Inputs: pos4/nrm4 4 floats per vertex (w ignored), tri4 (i0, i1, i2, material) with indices below
 * nverts / nmats (not checked: they are device memory), mats device gi_material[nmats]; pos4, nrm4, tri4, occ, attr
 * 16-byte aligned.  Outputs as gi_vox_read_state lays them out (hdr 64 words, ptr levels*G^3, occ max_bricks*16,
 * base/code max_bricks, attr max_voxels*4, plane/sunvis max_voxels).  Runs on the current device and `stream`; the
 * first call on a device looks up the scratch's address there, in the device's primary context (the one the CUDA
 * runtime uses); the address stays valid until that context is reset.  All calls share the scratch: two calls that overlap
 * on the GPU race and corrupt each other, so serialise them. */
int gi_vox_build_noalloc(const gi_vox_params *params, const double eye[3], const float *pos4, const float *nrm4,
                         uint32_t nverts, const uint32_t *tri4, uint32_t ntris, const gi_material *mats, uint32_t nmats,
                         uint32_t *hdr, uint32_t *ptr, uint32_t *occ, uint32_t *base, uint32_t *code, uint32_t *attr,
                         float *plane, float *sunvis, void *stream);

/* ---- radiance cascades (rc.ts Rc), screen probes traced in the voxel world --------------------------------------- */
int gi_rc_create(gi_ctx *ctx, const gi_rc_params *params, uint32_t width, uint32_t height, gi_rc **out);
/* createRc with params.method 'world' (rc.ts:1019) and the voxel world tracer: the same cascades (P unused, the
 * frame's P and sMin set the probe spacing), probes and atlas laid out by capacity.  Every later gi_rc_solve /
 * gi_solve runs registerPixels .. linkParents, the trace, mergeWorld, projectSH with the c0 history and gatherWorld;
 * the history keeps one solve (a host that reorders or skips frames changes the result, as in the reference). */
int gi_rc_create_world(gi_ctx *ctx, const gi_rc_params *params, const gi_world_params *world, uint32_t width,
                       uint32_t height, gi_rc **out);
/* The 640-byte Frame uniform exactly as packFrame (frame.ts:76-94) writes it. */
int gi_rc_set_frame(gi_rc *rc, const void *frame640, void *stream);
/* G-buffer from host memory: depth (W*H f32, reversed Z, 0 = background) and the shading normal, either as
 * rgba f32 (normal4) or in the reference's rgba16float texture format (normal_rgba16f, 4 halves per pixel). */
int gi_rc_set_gbuffer(gi_rc *rc, const float *depth, const float *normal4, void *stream);
int gi_rc_set_gbuffer_f16(gi_rc *rc, const float *depth, const uint16_t *normal_rgba16f, void *stream);
/* The same with the normal as three halves per pixel (the rgba16float texture's r, g, b; the path reads no alpha):
 * 6 bytes a pixel over the bus instead of 8, expanded on the device (stream-ordered, alpha 0 as the raster writes). */
int gi_rc_set_gbuffer_rgb16f(gi_rc *rc, const float *depth, const uint16_t *normal_rgb16f, void *stream);
/* The G-buffer's style tag (gbuffer.ts:2: the alpha byte of its rgba8 albedo: 1 toon, 0.5 another measured object,
 * 0 photoreal), W*H bytes from host memory.  gatherWorld applies the receiving operator to toon pixels
 * (rc.ts:877-926: the interpolated L0/L1 SH through toonReceive, style.ts:30-42, output alpha 2 + band + 2 contrast)
 * and counts only photoreal pixels as black.  All zero at creation; gi_rc_render_gbuffer writes it from the
 * materials' flags (4 toon, 8 object).  The screen method does not read it. */
int gi_rc_set_gbuffer_tag(gi_rc *rc, const uint8_t *tag, void *stream);
/* G-buffer drawn on the device from the scene and the frame (one primary-ray sample per pixel centre). */
int gi_rc_render_gbuffer(gi_rc *rc, gi_scene *scene, void *stream);
/* The sun shadow map (encodeShadow, lighting.ts:175-189; depth32float, compare less, depth bias 2 + slope 2, cull
 * none) drawn on the device from the frame's lightViewProj (words 64-79) over the scene's triangles: size x size
 * f32 depths owned by the rc, 1 where nothing is drawn.  While the rc holds one, gi_solve's rebuild also runs voxSun
 * (voxel.ts:633-671) with it, the frame's sun direction and shadow bias (word 157); without one every voxel's sun
 * visibility is 1.  size 0 releases it.  Draw it again when the light matrix or the scene moves; a graph captured
 * before a change of size must be captured again. */
int gi_rc_render_shadow(gi_rc *rc, gi_scene *scene, uint32_t size, void *stream);
/* The rebuild (gi_vox_build) with voxSun from rc's shadow map and frame, as gi_solve runs it, for callers that solve
 * several cascade sets over one voxel world (gi_rc_solve each); the same as gi_vox_build when rc holds no map. */
int gi_vox_build_sun(gi_vox *vox, gi_rc *rc, void *stream);
/* Multi-bounce (bounce.ts; BounceParams, DEFAULT_BOUNCE {1.2, [32, 16, 32], 16, 2}): a camera-centred volume of
 * dx*dy*dz irradiance probes `cell` metres apart, rebuilt every solve from the voxels (each probe near a surface traces
 * `rays` rays plus six axis rays, every `div` solves by its position) and injected into the voxels, whose hits then
 * add albedo / pi times it.  Bound to one voxel world (the volume's rays and the injected irradiance are its voxels');
 * gi_solve / gi_rc_solve with another world fail.  rays <= 26.  params NULL turns it off.  The volume keeps one frame
 * of history (the probes' rays read the previous volume), so results depend on the sequence of solves. */
typedef struct {
  float cell;
  uint32_t dx, dy, dz, rays, div;
  uint32_t reserved[2];
} gi_bounce_params;
int gi_rc_set_bounce(gi_rc *rc, gi_vox *vox, const gi_bounce_params *params);
/* encode(enc) (rc.ts:1169-1222): giBuild (setupScreen), giTrace, giMerge (mergeScreen N-1..0, projectSH),
 * giGather (gatherScreen) over the voxel world's current state. */
int gi_rc_solve(gi_rc *rc, gi_vox *vox, void *stream);
/* One frame of the GI path: gi_vox_build then gi_rc_solve. */
int gi_solve(gi_rc *rc, gi_vox *vox, void *stream);
/* readIrradiance (rcrun.ts:131-149): W*H rgba f32 (rgb irradiance, a = 1 valid / 0 background). Synchronises. */
int gi_rc_read_irradiance(gi_rc *rc, float *rgba, void *stream);
/* The irradiance as stored: rgba16float (atlas F16/BF16) or rgba f32 (atlas F32).  Synchronises. */
int gi_rc_read_irradiance_raw(gi_rc *rc, void *out, size_t bytes, void *stream);
/* The same without synchronising: a stream-ordered copy into `out`, host or device memory (pinned host memory makes
 * it asynchronous). */
int gi_rc_read_irradiance_async(gi_rc *rc, void *out, size_t bytes, void *stream);
/* readCounts (rc.ts:1223-1232): the 80 counter words (rc.ts:173-175).  Synchronises.  World probes: returns
 * GI_ERR_TIMEOUT (the words copied out) when a bounded wait of the solve's compaction gave up. */
int gi_rc_read_counts(gi_rc *rc, uint32_t counts[80], void *stream);
/* setStats (rc.ts:1233): 0 off, 1 DDA step counters. */
int gi_rc_set_stats(gi_rc *rc, uint32_t level);
/* CUDA graph of one gi_solve(rc, vox) captured on `stream` (not the legacy default stream), replayed by
 * gi_rc_graph_launch.  The graph reads the frame, G-buffer and scene vertices from their device buffers at replay, so
 * gi_rc_set_frame / gi_rc_set_gbuffer* / gi_scene_update_vertices before a launch take effect; the voxel windows
 * (gi_vox_update) and the parameters are those of capture time: capture again after moving the windows. */
int gi_rc_graph_capture(gi_rc *rc, gi_vox *vox, void *stream);
/* CUDA graph of one whole frame: the scene's rigid objects posed from their last uploaded transforms (when defined),
 * the G-buffer drawn, gi_solve, and the irradiance as stored copied into irr_out (pinned host or device memory,
 * gi_rc_read_irradiance_raw's layout; NULL: no copy).  Replayed by gi_rc_graph_launch: per frame a caller uploads
 * the transforms and launches.  The same conditions as gi_rc_graph_capture; the voxel world must be built from
 * `scene`. */
int gi_rc_graph_capture_frame(gi_rc *rc, gi_vox *vox, gi_scene *scene, void *irr_out, void *stream);
int gi_rc_graph_launch(gi_rc *rc, void *stream);
/* Batches (no counterpart in the reference, which solves one frame per queue submit): n independent solves, each
 * an (rc, vox) pair with its own frame, G-buffer and scene, captured into ONE CUDA graph whose n solve chains are
 * parallel branches, so the GPU runs the small kernels of uneven solves side by side.  Every handle may appear once.
 * gi_batch_capture needs a stream that is not the legacy default stream; the graph reads frames, G-buffers and
 * vertices at launch; capture again after moving a voxel window. */
typedef struct gi_batch gi_batch;
int gi_batch_create(gi_ctx *ctx, gi_rc *const *rcs, gi_vox *const *voxes, uint32_t n, gi_batch **out);
int gi_batch_capture(gi_batch *batch, void *stream);
/* The same batch captured pass by pass: the n voxel rebuilds as parallel branches, then ONE launch per cascade pass
 * over the work of every solve (setup, a persistent trace over all the rays, one merge launch per cascade step, the
 * gather).  All solves need the same atlas format and probe spacing (8, 16 or 32 pixels); the solves' launch tuning
 * does not apply to these launches (results are the same bits either way); a solve with multi-bounce on is
 * refused (GI_ERR_INVALID: capture its chain with gi_batch_capture).  Replaces a graph captured before. */
int gi_batch_capture_passes(gi_batch *batch, void *stream);
int gi_batch_launch(gi_batch *batch, void *stream);
int gi_batch_destroy(gi_batch *batch);
/* Pass timing (the reference's per-pass timestamps, rcrun.ts:325-372): when on, every solve records CUDA events
 * between its passes; gi_rc_pass_times then gives the last solve's milliseconds of [vox (gi_solve only), giBuild,
 * giTrace, giMerge, giGather] (synchronises on the last event). */
int gi_rc_set_timing(gi_rc *rc, int on);
int gi_rc_pass_times(gi_rc *rc, float ms[5]);
/* Bytes of device memory the handle holds (rc.ts `bytes`). */
int gi_rc_bytes(gi_rc *rc, uint64_t *bytes);

/* Debug readback of an internal buffer (synchronises).  what: */
enum {
  GI_RC_PROBES = 0,     /* 48 bytes per probe (pos.xyz, s0; nrm.xyz, view depth; grid), all cascades */
  GI_RC_RAD = 1,        /* the cascade atlas as stored (4 components per ray) */
  GI_RC_SH = 2,         /* 32 components per c0 probe as stored (27 used) */
  GI_RC_DEPTH = 3,      /* W*H f32 */
  GI_RC_NORMAL = 4,     /* W*H*4 halves */
  GI_RC_HITS = 5,       /* per ray: level, brick, bit, tIn bits (only after gi_rc_set_debug_hits(rc, 1)) */
  GI_RC_RAD_TRACED = 6, /* the atlas right after the trace, before the merge (only with debug hits on) */
  GI_RC_SHADOW = 7,     /* layers*size*size f32, the sun shadow map (only after gi_rc_render_shadow) */
  GI_RC_BOUNCE_VOL = 8, /* the two bounce volumes, dx*dy*(6dz+1) rgba16f texels each (only with multi-bounce on) */
  GI_RC_BOUNCE_INJ = 9, /* per voxel the injected irradiance: 8 halves (front rgb, 0, back rgb, 0) (multi-bounce on) */
  GI_RC_BOUNCE_LIST = 10, /* 4 + dx*dy*dz words: listed probes, frame counter, current volume, then the list */
  GI_RC_WORLD_KEYS = 11,  /* world probes: every cascade's hash table of probe keys (0 = empty) */
  GI_RC_WORLD_SLOTS = 12, /* world probes: per hash slot the key's probe (0xffffffff: none, or past the capacity) */
  GI_RC_WORLD_PARENTS = 13, /* world probes: per probe the 8 probes of the cascade above it merges (0xffffffff: none) */
  GI_RC_WORLD_STATE = 14, /* world probes: 64 words: [0] history parity, [7] nonzero if a compaction's scan stopped
                             waiting (never expected), [8 + c] probes of cascade c, [16 + c] first ray of cascade c */
  GI_RC_TAG = 15          /* W*H bytes: the G-buffer's style tag (its albedo's alpha byte: 255 toon, 128 object, 0) */
};
int gi_rc_read_buffer(gi_rc *rc, int what, void *out, size_t bytes, void *stream);
int gi_rc_buffer_bytes(gi_rc *rc, int what, size_t *bytes);
int gi_rc_set_debug_hits(gi_rc *rc, int on);
/* FP64 reference of the merge, SH projection and gather (no counterpart in the reference, whose atlases are f16): the
 * last solve's traced intervals, kept in f32 by gi_rc_set_debug_hits, merged (mergeScreen rc.ts:710-743), projected
 * (projectSH rc.ts:752-774) and gathered (gatherScreen rc.ts:929-954) in double precision with no rounding between
 * the stages.  The yardstick of the f32/f16/bf16 atlas error.  Needs an F32 atlas with debug hits on (GI_ERR_STATE
 * otherwise); allocates its f64 buffers (32 bytes per ray and per pixel) on the first call.  Stream-ordered. */
int gi_rc_merge_gather_f64(gi_rc *rc, void *stream);
/* The same with the atlas storage of the cascades in bit mask f16_cascades rounded to f16 (round to nearest even) and
 * every stage still in double: their traced intervals as they are read, and (cascades above 0) their merged radiances
 * as they are stored for the cascade below.  The storage error of a per-cascade f16/f32 atlas apart from the f32
 * arithmetic; mask 0 is gi_rc_merge_gather_f64.  No counterpart in the reference. */
int gi_rc_merge_gather_f64_rounded(gi_rc *rc, uint32_t f16_cascades, void *stream);
/* W*H*4 doubles (rgb, a = 1 valid / 0 background) of the last gi_rc_merge_gather_f64, into host or device memory.
 * Synchronises. */
int gi_rc_read_irradiance_f64(gi_rc *rc, double *rgba, void *stream);
/* Launch tuning (no counterpart in the reference; results do not depend on it, tested bit-exact).  Picked per solve
 * shape by the autotuner (rtgi/autotune.py); takes effect at the next solve or graph capture. */
typedef struct gi_rc_tuning {
  uint32_t trace_order;    /* 0: probe-major (a warp's lanes take an 8 x 4 tile of a probe's direction map, or all
                              of a small map: neighbouring directions walk alike; atlas writes in 128-byte runs), 1: direction-major (a warp's lanes take one direction of 32 neighbouring probes,
                              coherent voxel paths), 2: walk-length order (screen probes; the rays by the previous
                              solve's DDA step count and hit, longest first, so a warp's lanes walk alike: for a camera
                              that holds still, as the keys come from the previous solve's rays and screen probes move
                              with the camera; 5 bytes per ray, allocated when chosen).  Default 0 */
  uint32_t trace_rays;     /* rays per lane per queue fetch: 1, 2 or 4 (default 1) */
  uint32_t trace_blocks;   /* resident 256-thread blocks per SM of the persistent trace: 1..16 (default 8) */
  uint32_t gather_shape;   /* gather: 0, 1, 2 blocks of 16x16, 32x8, 8x32 pixels; 3 (default) warps on pixel tiles
                              aligned to the probe cells, the shared probes staged in shared memory (cascade-0 tile
                              size 8, 16 or 32; otherwise 16x16) */
  uint32_t merge_threads;  /* threads per merge block: 64, 128, 256 (default) or 512 */
  uint32_t reserved[3];
} gi_rc_tuning;
int gi_rc_set_tuning(gi_rc *rc, const gi_rc_tuning *t);
int gi_rc_get_tuning(gi_rc *rc, gi_rc_tuning *t);
typedef struct gi_vox_tuning {
  uint32_t chunk_cells;    /* cells per big-triangle work item of voxBits: a power of two 32..1024 (default 128) */
  uint32_t blocks;         /* resident 256-thread blocks per SM of the grid-stride rebuild passes: 1..16 (default 8) */
  uint32_t reserved[6];
} gi_vox_tuning;
int gi_vox_set_tuning(gi_vox *vox, const gi_vox_tuning *t);
int gi_vox_get_tuning(gi_vox *vox, gi_vox_tuning *t);
int gi_rc_destroy(gi_rc *rc);

/* ---- the dynamic layer (src/core/dynlayer.ts) ---------------------------------------------------------------------
 * Moving triangles (the scene's rows from first_dynamic on; gi_scene_set_static_count keeps them out of the voxel
 * rebuild) splatted every frame into a layer of coverage and mean radiance per voxel of the clipmap's levels (fixed
 * point at level 0, prefiltered to the coarser levels), which the cascades' traces read at the width of a direction
 * bin's cone (traceDyn, rc.ts:223-231).  createDynLayer (dynlayer.ts:680): `bricks` is VoxParams.dynBricks (the
 * reference's default 512); albedo 1 writes the area x albedo words (the reference's DYN_ALB, configs with the token
 * obj, whose objects receive light: gi_rc_set_objects).  G^3 must be a multiple of 32. */
int gi_dyn_create(gi_vox *vox, uint32_t bricks, uint32_t first_dynamic, uint32_t albedo, gi_dyn **out);
/* DynLayer.encode (dynlayer.ts:738-741): mark .. resolve at the voxel world's current windows, shaded with the rc's
 * frame (sun, style) and its sun shadow map when it has one.  Stream-ordered.  gi_solve runs it after the static
 * rebuild when the layer is bound to the rc (gi_rc_set_dyn). */
int gi_dyn_build(gi_dyn *dyn, gi_rc *rc, void *stream);
/* readCounters (dynlayer.ts:749-759): the 64 header words (0 wanted bricks, 1 dropped, 2-7 bounds in cm + 2^30,
 * 8 allocated, 9 triangles outside every clipmap, 10 frame counter, 16 + L first slot and 24 + L bricks of level L).
 * Synchronises; GI_ERR_TIMEOUT when the allocation's bounded scan wait gave up (word 12). */
int gi_dyn_read_counters(gi_dyn *dyn, uint32_t hdr[64], void *stream);
/* The layer's arrays (any may be NULL): ptr levels*G^3, bits 2*levels*G^3/32, meta bricks, mask bricks*16, data
 * bricks*512*13 words.  Synchronises. */
int gi_dyn_read_state(gi_dyn *dyn, uint32_t *ptr, uint32_t *bits, uint32_t *meta, uint32_t *mask, uint32_t *data,
                      void *stream);
int gi_dyn_bytes(gi_dyn *dyn, uint64_t *bytes);
int gi_dyn_destroy(gi_dyn *dyn);
/* The layer the rc's traces read, or NULL for none (dyn[0] = 0 in the reference: no dynamic objects).  Drops a
 * captured graph (it was captured without the layer). */
int gi_rc_set_dyn(gi_rc *rc, gi_dyn *dyn);
/* The token obj (RcParams.objects, rc.ts:79-80; phase 31, off by default): with multi-bounce on (gi_rc_set_bounce) and a
 * layer bound, every solve's trace pass first adds to the layer's voxels the light they receive from the previous
 * frame's bounce volume (dynInject, dynlayer.ts:165-191, with bounce.ts:265-296's dynE), and the volume's irradiance
 * rays read the layer in front of their static hits (bnTraceDyn, bounce.ts:169-174).  The layer should be created
 * with albedo 1 (DynLayer.setAlbedo): without its albedo words the received light is 0.  Captured graphs made before
 * the change are refused (GI_ERR_STATE). */
int gi_rc_set_objects(gi_rc *rc, int on);

#ifdef __cplusplus
}
#endif
#endif /* GI_H */
