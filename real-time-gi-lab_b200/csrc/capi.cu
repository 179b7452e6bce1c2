// C-ABI of the GI path (include/gi.h): handle lifetimes, device memory, argument checks and the launch sequences.
#include <cuda_runtime.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <new>
#include <string>
#include <vector>

#include "gi_dev.cuh"
#include "gi_internal.h"

using namespace gi;

namespace {

thread_local std::string g_err;

int fail(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

int cuda_fail(cudaError_t e, const char *what) {
  if (e == cudaErrorMemoryAllocation) return fail(GI_ERR_OOM, "%s: out of device memory", what);
  return fail(GI_ERR_CUDA, "%s: %s (%s)", what, cudaGetErrorString(e), cudaGetErrorName(e));
}

#define CK(expr, what)                         \
  do {                                         \
    cudaError_t e_ = (expr);                   \
    if (e_ != cudaSuccess) return cuda_fail(e_, what); \
  } while (0)

template <class T>
cudaError_t dalloc(T **p, size_t count) {
  *p = nullptr;
  if (count == 0) count = 1;
  return cudaMalloc((void **)p, count * sizeof(T));
}

inline cudaStream_t S(void *stream) { return (cudaStream_t)stream; }

}  // namespace

// Error reporting for the library's other C-ABI files (gi_last_error returns it).
void gi_set_error(const char *msg) { g_err = msg; }

struct gi_ctx {
  int device;
  uint32_t sm_count;
};

// Capacity of the raster's per-tile lists: 8 tiles per triangle, at least 2^20 entries (triangles past it are walked
// by every tile instead, so the G-buffer does not depend on it)
// Entries of the voxel rebuild's chunk-to-item table (chunks past it are found by binary search)
constexpr uint32_t VOX_CITEM_CAP = 1u << 20;

static uint32_t raster_list_cap(uint32_t ntris) {
  uint64_t c = (uint64_t)ntris * 8u;
  return (uint32_t)(c < (1u << 20) ? (1u << 20) : (c > 0xffffffffull ? 0xffffffffull : c));
}

struct gi_scene {
  gi_ctx *ctx;
  float4 *pos = nullptr, *nrm = nullptr;
  uint4 *tri = nullptr;
  gi_material *mats = nullptr;
  uint32_t nverts = 0, ntris = 0, nmats = 0;
  uint32_t mat_flags = 0;    // OR of the materials' flags (4 toon, 8 object: the G-buffer raster writes style tags)
  uint64_t gen = 0;          // bumped when a buffer or a count a captured graph holds is replaced
  float2 *uv = nullptr;      // base colour textures (gi_scene_set_textures): a uv per vertex, every layer's mip chain
  float4 *tex = nullptr;
  uint32_t tex_size = 0, tex_levels = 0, tex_layers = 0, tex_layer_texels = 0;
  // G-buffer raster scratch (gbuffer.cu): two renders of one scene must not overlap on the GPU
  float4 *raster_rec = nullptr;
  uint32_t *raster_ntile = nullptr, *raster_pre = nullptr, *raster_sums = nullptr, *raster_counter = nullptr;
  uint32_t *raster_list = nullptr, *raster_over = nullptr;
  uint32_t raster_cap = 0;
  float4 *stage = nullptr;   // vertex staging for updates (nverts * 2)
  // rigid objects: a vertex range of n objects x per vertices posed on the device from a 3x4 transform per object
  float4 *rigid_rest = nullptr;   // rest positions (per * n), then rest normals (per * n)
  float *rigid_m = nullptr;       // n x 12 floats, row-major [R | t]
  uint32_t rigid_first = 0, rigid_per = 0, rigid_n = 0;
  SceneDev dev() const {
    SceneDev s;
    s.pos = pos; s.nrm = nrm; s.tri = tri; s.mats = mats; s.ntris = ntris; s.nverts = nverts; s.nmats = nmats;
    s.masked = (mat_flags & 1u) ? 1u : 0u;
    s.items = nullptr; s.lists = nullptr; s.inst = nullptr;
    s.nitems = 0; s.threads = ntris; s.key_stride = ntris; s.key_limit = ntris;
    s.uv = uv; s.tex = tex;
    s.tex_size = tex_size; s.tex_levels = tex_levels; s.tex_layers = tex_layers; s.tex_layer_texels = tex_layer_texels;
    return s;
  }
  // the scene as the rasters draw it: rows [0, ndraw) at every draw instance, triangle i * ndraw + row of instance i
  SceneDev raster_dev() const {
    SceneDev s = dev();
    s.ntris = ndraw * draw_ninst;
    if (draw_ninst > 1) { s.inst = draw_inst; s.key_stride = ndraw; }
    return s;
  }
  uint32_t ndraw = 0;          // rows the rasters draw ([0, ndraw); gi_scene_set_draw_count), all by default
  float4 *draw_inst = nullptr; // offsets of the drawn instances (gi_scene_set_draw_instances), instance 0 at the origin
  uint32_t draw_ninst = 1;
  uint32_t raster_tris = 0;    // triangles the raster scratch holds
  uint32_t static_tris = 0;    // rows the voxel rebuild reads ([0, static_tris); gi_scene_set_static_count), 0: all
};

struct gi_vox {
  gi_scene *scene;
  gi_vox_params p;
  VoxDev dev;
  bool updated = false;
  uint32_t hdr[64];
  uint64_t bytes = 0;
  // world work items (gi_vox_set_world / gi_vox_set_items): instance offsets, chunk row lists, this frame's items
  float4 *w_inst = nullptr;
  uint32_t *w_lists = nullptr;
  uint4 *w_items = nullptr;
  uint32_t w_ninst = 0, w_nlists = 0, w_items_cap = 0, w_nitems = 0, w_threads = 0, w_stride = 0;
  bool world = false;
  uint64_t items_gen = 0;   // bumped by gi_vox_set_world / gi_vox_set_items: graphs captured before are stale
  // the scene as the rebuild reads it: every row once, or this frame's work items
  SceneDev build_scene() const {
    SceneDev d = scene->dev();
    d.ntris = scene->ntris;
    if (scene->static_tris) d.threads = scene->static_tris == 0xffffffffu ? 0u : scene->static_tris;   // the dynamic tail
                                                                                                       // goes to the dynamic layer
    if (world) {
      d.items = w_items; d.lists = w_lists; d.inst = w_inst; d.nitems = w_nitems; d.threads = w_threads;
      d.key_stride = w_stride; d.key_limit = w_ninst * w_stride;
    }
    return d;
  }
};

struct gi_rc {
  gi_ctx *ctx;
  gi_rc_params p;
  uint32_t W, H;
  RcDev dev;
  float *frame = nullptr;
  float *depth = nullptr;
  uint2 *normal = nullptr;
  uint8_t *tag = nullptr;            // W*H style tags (zero at creation)
  uint32_t *tile_cnt = nullptr, *tile_fill = nullptr;   // G-buffer raster: per 16 x 16 tile (+1)
  uint32_t ntiles = 0;
  uint64_t mavg_bytes = 0;
  float4 *stage = nullptr;
  uint4 *hits = nullptr;
  void *rad_traced = nullptr;
  void *rad64 = nullptr, *irr64 = nullptr;   // FP64 reference buffers (gi_rc_merge_gather_f64), on first use
  double *sh64 = nullptr;
  bool have64 = false;
  size_t rad_elem_bytes = 0, sh_elems = 0, sh_elem_bytes = 0, irr_elem_bytes = 0;
  bool frame_set = false, gbuf_set = false, debug_hits = false;
  uint64_t bytes = 0;
  bool timing = false;
  bool timed = false;        // the last gi_solve / gi_rc_solve recorded its events
  bool timed_vox = false;    // ... and the voxel build's
  cudaEvent_t ev[7] = {};    // vox start, vox end = giBuild start, giBuild end, giTrace end, giMerge end, giGather end
  RcLaunch launch = {8u, 3u, 256u};   // gi_rc_tuning launch shapes
  cudaGraphExec_t graph = nullptr;   // one captured gi_solve (gi_rc_graph_capture)
  gi_vox *graph_vox = nullptr;
  uint64_t graph_items_gen = 0;      // the voxel world's work items the graph was captured with
  uint64_t graph_scene_gen = 0;      // its scene's gen at the capture
  float *shadow = nullptr;           // gi_rc_render_shadow: shadow_layers x shadow_size^2 depths
  uint32_t shadow_size = 0, shadow_layers = 0;
  uint32_t frame_layers = 1;         // the last frame's shadow.x (1, or 2 for a world's camera-following layers)
  uint64_t gen = 0;                  // bumped when a buffer a captured graph reads is freed or moved (shadow map,
  uint64_t graph_gen = 0;            // bounce volume, dynamic layer); graph_gen: gen at the rc graph's capture
  float4 *sm_rec = nullptr;          // its raster scratch, for up to sm_tris triangles
  uint32_t *sm_pre = nullptr, *sm_sums = nullptr, *sm_counter = nullptr;
  uint32_t sm_tris = 0;
  bool bounce = false;               // gi_rc_set_bounce: the volume, its buffers and the voxel world it is bound to
  BounceDev bn = {};
  gi_vox *bn_vox = nullptr;
  bool world = false;                // world probes (gi_rc_create_world)
  WorldDev w = {};
  struct gi_dyn *dyn = nullptr;      // gi_rc_set_dyn: the dynamic layer its traces read (gi_solve also builds it)
};

// The dynamic layer of a voxel world (dynlayer.ts createDynLayer): its device state and the scene's dynamic rows
struct gi_dyn {
  gi_vox *vox;
  DynDev dev;
  uint64_t bytes = 0;
};

static void free_scene(gi_scene *s) {
  cudaFree(s->pos); cudaFree(s->nrm); cudaFree(s->tri); cudaFree(s->mats);
  cudaFree(s->raster_rec); cudaFree(s->raster_ntile); cudaFree(s->raster_pre); cudaFree(s->raster_sums);
  cudaFree(s->raster_counter); cudaFree(s->raster_list); cudaFree(s->raster_over); cudaFree(s->stage);
  cudaFree(s->uv); cudaFree(s->tex);
  cudaFree(s->rigid_rest); cudaFree(s->rigid_m); cudaFree(s->draw_inst);
}
static void free_vox(gi_vox *v) {
  VoxDev &d = v->dev;
  cudaFree(d.hdr); cudaFree(d.ptr); cudaFree(d.occ); cudaFree(d.base); cudaFree(d.code); cudaFree(d.rep);
  cudaFree(d.big); cudaFree(d.attr); cudaFree(d.plane); cudaFree(d.sunvis);
  cudaFree(d.vpre); cudaFree(d.work); cudaFree(d.cpre); cudaFree(d.citem); cudaFree(d.look);
  cudaFree(v->w_inst); cudaFree(v->w_lists); cudaFree(v->w_items);
}
static void free_rc(gi_rc *r) {
  if (r->graph) { cudaGraphExecDestroy(r->graph); r->graph = nullptr; }
  for (cudaEvent_t &e : r->ev)
    if (e) { cudaEventDestroy(e); e = nullptr; }
  cudaFree(r->frame); cudaFree(r->depth); cudaFree(r->normal); cudaFree(r->tile_cnt); cudaFree(r->tile_fill); cudaFree(r->stage);
  cudaFree(r->tag); cudaFree(r->dev.rsteps); cudaFree(r->dev.rperm); cudaFree(r->dev.rhist);
  cudaFree(r->hits); cudaFree(r->rad_traced); cudaFree(r->rad64); cudaFree(r->sh64); cudaFree(r->irr64);
  cudaFree(r->dev.probes); cudaFree(r->dev.rad); cudaFree(r->dev.sh); cudaFree(r->dev.irr); cudaFree(r->dev.counts);
  cudaFree(r->dev.plevel); cudaFree((void *)r->dev.dirs); cudaFree(r->dev.mavg[0]); cudaFree(r->dev.mavg[1]);
  cudaFree((void *)r->dev.unorm8);
  cudaFree(r->shadow); cudaFree(r->sm_rec); cudaFree(r->sm_pre); cudaFree(r->sm_sums); cudaFree(r->sm_counter);
  cudaFree((void *)r->bn.dirs); cudaFree(r->bn.vol[0]); cudaFree(r->bn.vol[1]); cudaFree(r->bn.list); cudaFree(r->bn.inj);
  cudaFree(r->bn.ray_out);
  cudaFree(r->w.keys); cudaFree(r->w.slot_probe); cudaFree(r->w.parents); cudaFree(r->w.state); cudaFree(r->w.look);
  cudaFree(r->w.hist_tab); cudaFree(r->w.hist_grid); cudaFree(r->w.hist_sh);
  r->w = WorldDev{};
  r->bn = BounceDev{};
  r->bounce = false;
  r->dev.bn_inj = nullptr;
}

extern "C" {

int gi_version(void) { return GI_ABI_VERSION; }

const char *gi_status_string(int status) {
  switch (status) {
    case GI_OK: return "ok";
    case GI_ERR_INVALID: return "invalid argument";
    case GI_ERR_OOM: return "out of memory";
    case GI_ERR_CUDA: return "CUDA error";
    case GI_ERR_TIMEOUT: return "timeout";
    case GI_ERR_OVERFLOW: return "overflow";
    case GI_ERR_STATE: return "call out of order";
  }
  return "unknown status";
}

const char *gi_last_error(void) { return g_err.c_str(); }

int gi_ctx_create(int device, gi_ctx **out) {
  if (!out) return fail(GI_ERR_INVALID, "gi_ctx_create: out is NULL");
  *out = nullptr;
  int n = 0;
  CK(cudaGetDeviceCount(&n), "gi_ctx_create: cudaGetDeviceCount");
  if (device < 0 || device >= n) return fail(GI_ERR_INVALID, "gi_ctx_create: device %d of %d", device, n);
  CK(cudaSetDevice(device), "gi_ctx_create: cudaSetDevice");
  cudaDeviceProp prop;
  CK(cudaGetDeviceProperties(&prop, device), "gi_ctx_create: cudaGetDeviceProperties");
  if (prop.major < 10) return fail(GI_ERR_INVALID, "gi_ctx_create: device %d is sm_%d%d; this library is built for sm_100a", device, prop.major, prop.minor);
  gi_ctx *c = new (std::nothrow) gi_ctx;
  if (!c) return fail(GI_ERR_OOM, "gi_ctx_create: host allocation");
  c->device = device;
  c->sm_count = (uint32_t)prop.multiProcessorCount;
  *out = c;
  return GI_OK;
}

int gi_ctx_destroy(gi_ctx *ctx) {
  delete ctx;
  return GI_OK;
}

// ---- scene ----------------------------------------------------------------------------------------------------------
int gi_scene_upload(gi_ctx *ctx, const float *pos, const float *nrm, uint32_t nverts, const uint32_t *tri4,
                    uint32_t ntris, const gi_material *mats, uint32_t nmats, gi_scene **out) {
  if (!ctx || !out) return fail(GI_ERR_INVALID, "gi_scene_upload: NULL handle");
  *out = nullptr;
  if ((nverts && (!pos || !nrm)) || (ntris && !tri4) || (nmats && !mats))
    return fail(GI_ERR_INVALID, "gi_scene_upload: NULL array with a non-zero count");
  if (ntris && nmats == 0) return fail(GI_ERR_INVALID, "gi_scene_upload: triangles without materials");
  for (uint32_t t = 0; t < ntris; t++) {
    const uint32_t *r = tri4 + 4u * t;
    if (r[0] >= nverts || r[1] >= nverts || r[2] >= nverts)
      return fail(GI_ERR_INVALID, "gi_scene_upload: triangle %u indexes vertex %u of %u", t, r[0] >= nverts ? r[0] : (r[1] >= nverts ? r[1] : r[2]), nverts);
    if (r[3] >= nmats) return fail(GI_ERR_INVALID, "gi_scene_upload: triangle %u uses material %u of %u", t, r[3], nmats);
  }
  CK(cudaSetDevice(ctx->device), "gi_scene_upload: cudaSetDevice");
  gi_scene *s = new (std::nothrow) gi_scene;
  if (!s) return fail(GI_ERR_OOM, "gi_scene_upload: host allocation");
  s->ctx = ctx; s->nverts = nverts; s->ntris = ntris; s->nmats = nmats; s->ndraw = ntris; s->raster_tris = ntris;
  for (uint32_t m = 0; m < nmats; m++) s->mat_flags |= mats[m].flags;
  s->raster_cap = raster_list_cap(ntris);
  cudaError_t e = cudaSuccess;
  float4 *h4 = nullptr;
  do {
    if ((e = dalloc(&s->pos, nverts)) || (e = dalloc(&s->nrm, nverts)) || (e = dalloc(&s->tri, ntris)) ||
        (e = dalloc(&s->mats, nmats)) || (e = dalloc(&s->raster_rec, (size_t)3u * ntris)) ||
        (e = dalloc(&s->raster_ntile, ntris)) || (e = dalloc(&s->raster_pre, ntris)) ||
        (e = dalloc(&s->raster_sums, ntris / 256u + 1u)) || (e = dalloc(&s->raster_counter, 4)) ||
        (e = dalloc(&s->raster_list, s->raster_cap)) || (e = dalloc(&s->raster_over, ntris)) ||
        (e = dalloc(&s->stage, (size_t)nverts * 2u)))
      break;
    h4 = new (std::nothrow) float4[nverts ? nverts : 1];
    if (!h4) { free_scene(s); delete s; return fail(GI_ERR_OOM, "gi_scene_upload: host staging"); }
    for (uint32_t i = 0; i < nverts; i++) h4[i] = make_float4(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], 0.0f);
    if ((e = cudaMemcpy(s->pos, h4, nverts * sizeof(float4), cudaMemcpyHostToDevice))) break;
    for (uint32_t i = 0; i < nverts; i++) h4[i] = make_float4(nrm[3 * i], nrm[3 * i + 1], nrm[3 * i + 2], 0.0f);
    if ((e = cudaMemcpy(s->nrm, h4, nverts * sizeof(float4), cudaMemcpyHostToDevice))) break;
    if (ntris && (e = cudaMemcpy(s->tri, tri4, ntris * sizeof(uint4), cudaMemcpyHostToDevice))) break;
    if (nmats && (e = cudaMemcpy(s->mats, mats, nmats * sizeof(gi_material), cudaMemcpyHostToDevice))) break;
  } while (0);
  delete[] h4;
  if (e) { free_scene(s); delete s; return cuda_fail(e, "gi_scene_upload"); }
  *out = s;
  return GI_OK;
}

__global__ void k_pack_vertices(const float *src, float4 *dst, uint32_t n) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = make_float4(src[3 * i], src[3 * i + 1], src[3 * i + 2], 0.0f);
}

// sRGB decode of an 8-bit channel (the rgba8unorm-srgb read): c / 12.92 up to 0.04045, ((c + 0.055) / 1.055)^2.4
// above, c = k / 255, evaluated in double and rounded to f32
static void srgb_table(float lut[256]) {
  for (int k = 0; k < 256; k++) {
    const double c = (double)k / 255.0;
    lut[k] = (float)(c <= 0.04045 ? c / 12.92 : pow((c + 0.055) / 1.055, 2.4));
  }
}

int gi_scene_set_textures(gi_scene *s, const uint8_t *rgba8, uint32_t size, uint32_t layers, const float *uv) {
  if (!s || !rgba8 || !uv) return fail(GI_ERR_INVALID, "gi_scene_set_textures: NULL argument");
  if (size < 1 || size > 4096 || (size & (size - 1u)) != 0u)
    return fail(GI_ERR_INVALID, "gi_scene_set_textures: size %u (a power of two, 1 .. 4096)", size);
  if (layers < 1 || (uint64_t)layers * size * size > (1ull << 28))
    return fail(GI_ERR_INVALID, "gi_scene_set_textures: %u layers of %u^2 texels (at most 2^28 texels)", layers, size);
  CK(cudaSetDevice(s->ctx->device), "gi_scene_set_textures: cudaSetDevice");
  uint32_t levels = 0, per = 0;
  for (uint32_t n = size; n >= 1u; n >>= 1) { levels++; per += n * n; if (n == 1u) break; }
  cudaFree(s->uv); cudaFree(s->tex);
  s->uv = nullptr; s->tex = nullptr; s->tex_size = s->tex_levels = s->tex_layers = s->tex_layer_texels = 0;
  s->gen++;
  float lut[256];
  srgb_table(lut);
  uint8_t *raw = nullptr;
  float *dlut = nullptr;
  const size_t nraw = (size_t)layers * size * size * 4u;
  cudaError_t e;
  if ((e = cudaMalloc(&s->uv, (size_t)(s->nverts ? s->nverts : 1u) * sizeof(float2))) ||
      (e = cudaMalloc(&s->tex, (size_t)layers * per * sizeof(float4))) || (e = cudaMalloc(&raw, nraw)) ||
      (e = cudaMalloc(&dlut, sizeof lut)) ||
      (e = cudaMemcpy(s->uv, uv, (size_t)s->nverts * sizeof(float2), cudaMemcpyHostToDevice)) ||
      (e = cudaMemcpy(raw, rgba8, nraw, cudaMemcpyHostToDevice)) ||
      (e = cudaMemcpy(dlut, lut, sizeof lut, cudaMemcpyHostToDevice)) ||
      (e = gi_launch_tex_build(raw, dlut, s->tex, size, levels, layers, per)) || (e = cudaDeviceSynchronize())) {
    cudaFree(raw); cudaFree(dlut); cudaFree(s->uv); cudaFree(s->tex);
    s->uv = nullptr; s->tex = nullptr;
    return cuda_fail(e, "gi_scene_set_textures");
  }
  cudaFree(raw); cudaFree(dlut);
  s->tex_size = size; s->tex_levels = levels; s->tex_layers = layers; s->tex_layer_texels = per;
  s->gen++;
  return GI_OK;
}

int gi_scene_update_vertices(gi_scene *s, uint32_t first, uint32_t count, const float *pos, const float *nrm, void *stream) {
  if (!s) return fail(GI_ERR_INVALID, "gi_scene_update_vertices: NULL scene");
  if ((uint64_t)first + count > s->nverts) return fail(GI_ERR_INVALID, "gi_scene_update_vertices: [%u, %u) past %u vertices", first, first + count, s->nverts);
  if (count == 0) return GI_OK;
  if (!pos || !nrm) return fail(GI_ERR_INVALID, "gi_scene_update_vertices: NULL array");
  CK(cudaSetDevice(s->ctx->device), "gi_scene_update_vertices: cudaSetDevice");
  // the staging area holds the packed xyz triples (3 floats per vertex fit in the float4 slots)
  float *st = reinterpret_cast<float *>(s->stage);
  CK(cudaMemcpyAsync(st, pos, (size_t)count * 12u, cudaMemcpyHostToDevice, S(stream)), "gi_scene_update_vertices: positions");
  k_pack_vertices<<<(count + 255u) / 256u, 256, 0, S(stream)>>>(st, s->pos + first, count);
  CK(cudaMemcpyAsync(st + (size_t)count * 4u, nrm, (size_t)count * 12u, cudaMemcpyHostToDevice, S(stream)), "gi_scene_update_vertices: normals");
  k_pack_vertices<<<(count + 255u) / 256u, 256, 0, S(stream)>>>(st + (size_t)count * 4u, s->nrm + first, count);
  CK(cudaGetLastError(), "gi_scene_update_vertices: launch");
  return GI_OK;
}

__global__ void k_rigid_apply(float4 *pos, float4 *nrm, const float4 *rest, const float *m, uint32_t first,
                              uint32_t per, uint32_t n) {
  uint32_t total = per * n;
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  const float *M = m + 12u * (i / per);
  float4 p = rest[i], q = rest[total + i];
  pos[first + i] = make_float4(((M[0] * p.x + M[1] * p.y) + M[2] * p.z) + M[3],
                               ((M[4] * p.x + M[5] * p.y) + M[6] * p.z) + M[7],
                               ((M[8] * p.x + M[9] * p.y) + M[10] * p.z) + M[11], 0.0f);
  nrm[first + i] = make_float4((M[0] * q.x + M[1] * q.y) + M[2] * q.z, (M[4] * q.x + M[5] * q.y) + M[6] * q.z,
                               (M[8] * q.x + M[9] * q.y) + M[10] * q.z, 0.0f);
}

int gi_scene_rigid_define(gi_scene *s, uint32_t first, uint32_t verts_per_object, uint32_t n_objects) {
  if (!s) return fail(GI_ERR_INVALID, "gi_scene_rigid_define: NULL scene");
  uint64_t total = (uint64_t)verts_per_object * n_objects;
  if (total == 0 || first + total > s->nverts)
    return fail(GI_ERR_INVALID, "gi_scene_rigid_define: %u objects of %u vertices from %u do not fit %u vertices",
                n_objects, verts_per_object, first, s->nverts);
  CK(cudaSetDevice(s->ctx->device), "gi_scene_rigid_define: cudaSetDevice");
  float4 *rest = nullptr;
  float *m = nullptr;
  cudaError_t e;
  if ((e = dalloc(&rest, 2u * total)) || (e = dalloc(&m, 12u * (size_t)n_objects))) {
    cudaFree(rest);
    return cuda_fail(e, "gi_scene_rigid_define");
  }
  if ((e = cudaMemcpy(rest, s->pos + first, total * sizeof(float4), cudaMemcpyDeviceToDevice)) ||
      (e = cudaMemcpy(rest + total, s->nrm + first, total * sizeof(float4), cudaMemcpyDeviceToDevice))) {
    cudaFree(rest); cudaFree(m);
    return cuda_fail(e, "gi_scene_rigid_define: copy");
  }
  cudaFree(s->rigid_rest); cudaFree(s->rigid_m);
  s->rigid_rest = rest; s->rigid_m = m;
  s->rigid_first = first; s->rigid_per = verts_per_object; s->rigid_n = n_objects;
  s->gen++;
  return GI_OK;
}

int gi_scene_rigid_upload(gi_scene *s, const float *m34, void *stream) {
  if (!s || !m34) return fail(GI_ERR_INVALID, "gi_scene_rigid_upload: NULL argument");
  if (!s->rigid_n) return fail(GI_ERR_STATE, "gi_scene_rigid_upload: no rigid objects defined");
  CK(cudaSetDevice(s->ctx->device), "gi_scene_rigid_upload: cudaSetDevice");
  CK(cudaMemcpyAsync(s->rigid_m, m34, (size_t)s->rigid_n * 48u, cudaMemcpyHostToDevice, S(stream)),
     "gi_scene_rigid_upload: copy");
  return GI_OK;
}

int gi_scene_rigid_apply(gi_scene *s, void *stream) {
  if (!s) return fail(GI_ERR_INVALID, "gi_scene_rigid_apply: NULL scene");
  if (!s->rigid_n) return fail(GI_ERR_STATE, "gi_scene_rigid_apply: no rigid objects defined");
  CK(cudaSetDevice(s->ctx->device), "gi_scene_rigid_apply: cudaSetDevice");
  uint32_t total = s->rigid_per * s->rigid_n;
  k_rigid_apply<<<(total + 255u) / 256u, 256, 0, S(stream)>>>(s->pos, s->nrm, s->rigid_rest, s->rigid_m, s->rigid_first,
                                                                s->rigid_per, s->rigid_n);
  CK(cudaGetLastError(), "gi_scene_rigid_apply: launch");
  return GI_OK;
}

int gi_scene_destroy(gi_scene *s) {
  if (!s) return GI_OK;
  cudaSetDevice(s->ctx->device);
  free_scene(s);
  delete s;
  return GI_OK;
}

// ---- voxel world ------------------------------------------------------------------------------------------------------
int gi_vox_create(gi_scene *scene, const gi_vox_params *p, gi_vox **out) {
  if (!scene || !p || !out) return fail(GI_ERR_INVALID, "gi_vox_create: NULL argument");
  *out = nullptr;
  if (p->levels < 1 || p->levels > 8) return fail(GI_ERR_INVALID, "gi_vox_create: levels %u (1..8)", p->levels);
  if (p->G < 4 || p->G > 256 || p->G % 4) return fail(GI_ERR_INVALID, "gi_vox_create: G %u (a multiple of 4, 4..256)", p->G);
  if (!(p->v0 > 0.0)) return fail(GI_ERR_INVALID, "gi_vox_create: v0 must be > 0");
  if (p->max_bricks < 1 || p->max_voxels < 1) return fail(GI_ERR_INVALID, "gi_vox_create: empty pools");
  if ((uint64_t)p->max_bricks * 512u >= (1ull << 32) || (uint64_t)p->max_voxels >= (1ull << 31))
    return fail(GI_ERR_INVALID, "gi_vox_create: pools past 32-bit indexing");
  CK(cudaSetDevice(scene->ctx->device), "gi_vox_create: cudaSetDevice");
  gi_vox *v = new (std::nothrow) gi_vox;
  if (!v) return fail(GI_ERR_OOM, "gi_vox_create: host allocation");
  memset(&v->dev, 0, sizeof v->dev);
  v->scene = scene;
  v->p = *p;
  VoxDev &d = v->dev;
  d.v0 = (float)p->v0;
  d.levels = p->levels; d.G = p->G; d.max_bricks = p->max_bricks; d.max_voxels = p->max_voxels;
  d.big_cap = 1u << 18;   // BIG_CAP (voxel.ts:224)
  d.chunk_log2 = 7;       // default gi_vox_tuning: 128 cells per big-triangle work item, 8 blocks per SM
  d.blocks = 8;
  vox_derived(d);
  d.citem_cap = VOX_CITEM_CAP;
  uint64_t nptr = (uint64_t)p->levels * p->G * p->G * p->G;
  uint32_t scan_words = (uint32_t)((nptr + 255u) / 256u);   // blocks of the brick allocation, 256 entries each
  uint32_t vscan = (p->max_bricks + 255u) / 256u;             // and of the voxel allocation
  if (vscan > scan_words) scan_words = vscan;
  d.scan_cap = scan_words;
  cudaError_t e;
  if ((e = dalloc(&d.hdr, GI_HDR)) || (e = dalloc(&d.ptr, nptr)) || (e = dalloc(&d.occ, (size_t)p->max_bricks * 16u)) ||
      (e = dalloc(&d.base, p->max_bricks)) || (e = dalloc(&d.code, p->max_bricks)) ||
      (e = dalloc(&d.rep, (size_t)p->max_bricks * 512u)) || (e = dalloc(&d.big, (size_t)16u * d.big_cap)) ||
      (e = dalloc(&d.attr, p->max_voxels)) || (e = dalloc(&d.plane, p->max_voxels)) ||
      (e = dalloc(&d.sunvis, p->max_voxels)) ||
      (e = dalloc(&d.vpre, (size_t)p->max_bricks + 1u)) || (e = dalloc(&d.work, 4)) ||
      (e = dalloc(&d.cpre, (size_t)8u * d.big_cap)) || (e = dalloc(&d.citem, (size_t)VOX_CITEM_CAP)) ||
      (e = dalloc(&d.look, (size_t)scan_words + 1u))) {
    free_vox(v);
    delete v;
    return cuda_fail(e, "gi_vox_create");
  }
  v->bytes = (GI_HDR + nptr + (uint64_t)p->max_bricks * (16u + 2u + 512u) + (uint64_t)16u * d.big_cap +
              (uint64_t)p->max_voxels * 6u + p->max_bricks + 5u + (uint64_t)8u * d.big_cap +
              VOX_CITEM_CAP + 2u * ((uint64_t)scan_words + 1u)) * 4u;
  memset(v->hdr, 0, sizeof v->hdr);
  *out = v;
  return GI_OK;
}

int gi_vox_update(gi_vox *v, const double eye[3]) {
  if (!v || !eye) return fail(GI_ERR_INVALID, "gi_vox_update: NULL argument");
  for (int a = 0; a < 3; a++)
    if (!isfinite(eye[a])) return fail(GI_ERR_INVALID, "gi_vox_update: eye is not finite");
  memset(v->dev.origin, 0, sizeof v->dev.origin);
  for (uint32_t L = 0; L < v->p.levels; L++) {
    double bs = v->p.v0 * ldexp(1.0, (int)L) * 8.0;   // v0 * 2 ** L * 8 (voxel.ts:873)
    for (int a = 0; a < 3; a++) {
      double o = floor(eye[a] / bs) - (double)(v->p.G / 2);
      if (fabs(o) > (double)(1 << 22)) return fail(GI_ERR_INVALID, "gi_vox_update: eye too far from the origin");
      v->dev.origin[L][a] = (int32_t)o;
    }
  }
  vox_bounds(v->dev);
  v->updated = true;
  return GI_OK;
}

// The rebuild, with voxSun from a shadow map when one is given (gi_solve passes the rc's)
static int vox_build_sun(gi_vox *v, const float *frame, const float *shadow, uint32_t size, void *stream,
                         uint32_t layers = 1u) {
  if (!v) return fail(GI_ERR_INVALID, "gi_vox_build: NULL vox");
  if (!v->updated) return fail(GI_ERR_STATE, "gi_vox_build: gi_vox_update was not called");
  CK(cudaSetDevice(v->scene->ctx->device), "gi_vox_build: cudaSetDevice");
  VoxDev d = v->dev;
  d.sun_frame = frame; d.shadow = shadow; d.shadow_size = shadow ? size : 0u; d.shadow_layers = shadow ? layers : 0u;
  CK(gi_launch_vox_build(d, v->build_scene(), v->scene->ctx->sm_count, S(stream)), "gi_vox_build: launch");
  return GI_OK;
}

int gi_vox_build(gi_vox *v, void *stream) { return vox_build_sun(v, nullptr, nullptr, 0u, stream); }

// The rebuild with the rc's shadow map (voxSun) when it holds one; refused when the frame asks for more layers than
// the map was drawn with
static int rc_vox_build(gi_vox *v, gi_rc *r, void *stream);

int gi_vox_set_world(gi_vox *v, const float *instances, uint32_t ninst, const uint32_t *lists, uint32_t nlists,
                     uint32_t key_stride) {
  if (!v) return fail(GI_ERR_INVALID, "gi_vox_set_world: NULL vox");
  CK(cudaSetDevice(v->scene->ctx->device), "gi_vox_set_world: cudaSetDevice");
  cudaFree(v->w_inst); cudaFree(v->w_lists); cudaFree(v->w_items);
  v->w_inst = nullptr; v->w_lists = nullptr; v->w_items = nullptr;
  v->world = false; v->w_ninst = v->w_nlists = v->w_items_cap = v->w_nitems = v->w_threads = v->w_stride = 0;
  v->items_gen++;
  if (ninst == 0) return GI_OK;   // back to every row once
  if (!instances || (nlists && !lists)) return fail(GI_ERR_INVALID, "gi_vox_set_world: NULL argument");
  if (ninst > 1024) return fail(GI_ERR_INVALID, "gi_vox_set_world: %u instances (at most 1024, voxel.ts:742)", ninst);
  if (instances[0] != 0.0f || instances[1] != 0.0f || instances[2] != 0.0f)
    return fail(GI_ERR_INVALID, "gi_vox_set_world: instance 0 must be at the origin");
  if (key_stride != v->scene->ntris)
    return fail(GI_ERR_INVALID, "gi_vox_set_world: key stride %u, the scene has %u rows", key_stride, v->scene->ntris);
  if ((uint64_t)ninst * key_stride >= (1ull << 32)) return fail(GI_ERR_INVALID, "gi_vox_set_world: triangle keys overflow");
  for (uint32_t k = 0; k < nlists; k++)
    if (lists[k] >= key_stride) return fail(GI_ERR_INVALID, "gi_vox_set_world: list word %u names row %u", k, lists[k]);
  std::vector<float4> inst(ninst);
  for (uint32_t i = 0; i < ninst; i++) inst[i] = make_float4(instances[3 * i], instances[3 * i + 1], instances[3 * i + 2], 0.0f);
  cudaError_t e;
  if ((e = dalloc(&v->w_inst, ninst)) || (e = dalloc(&v->w_lists, nlists ? nlists : 1u)) ||
      (e = cudaMemcpy(v->w_inst, inst.data(), ninst * sizeof(float4), cudaMemcpyHostToDevice)) ||
      (nlists && (e = cudaMemcpy(v->w_lists, lists, nlists * 4u, cudaMemcpyHostToDevice))))
    return cuda_fail(e, "gi_vox_set_world");
  v->w_ninst = ninst; v->w_nlists = nlists; v->w_stride = key_stride;
  v->world = true;   // no items yet: the rebuild reads nothing until gi_vox_set_items
  return GI_OK;
}

int gi_vox_set_items(gi_vox *v, const uint32_t *items, uint32_t nitems, uint32_t threads) {
  if (!v) return fail(GI_ERR_INVALID, "gi_vox_set_items: NULL vox");
  if (!v->world) return fail(GI_ERR_STATE, "gi_vox_set_items: no world (gi_vox_set_world)");
  if (nitems && !items) return fail(GI_ERR_INVALID, "gi_vox_set_items: NULL items");
  uint32_t expect = 0;
  for (uint32_t k = 0; k < nitems; k++) {
    const uint32_t *it = items + 4u * k;
    if (it[0] != expect) return fail(GI_ERR_INVALID, "gi_vox_set_items: item %u starts at thread %u, not %u", k, it[0], expect);
    if (it[2] >= v->w_ninst) return fail(GI_ERR_INVALID, "gi_vox_set_items: item %u instance %u", k, it[2]);
    if (it[3] >= v->p.levels) return fail(GI_ERR_INVALID, "gi_vox_set_items: item %u level %u", k, it[3]);
    const uint32_t next = k + 1 < nitems ? items[4u * (k + 1)] : threads;
    if (next < it[0]) return fail(GI_ERR_INVALID, "gi_vox_set_items: item %u out of order", k);
    const uint64_t count = next - it[0];
    if (it[1] & 0x80000000u) {
      if ((uint64_t)(it[1] & 0x7fffffffu) + count > v->w_stride) return fail(GI_ERR_INVALID, "gi_vox_set_items: item %u past the rows", k);
    } else if ((uint64_t)it[1] + count > v->w_nlists) {
      return fail(GI_ERR_INVALID, "gi_vox_set_items: item %u past the lists", k);
    }
    expect = next;
  }
  CK(cudaSetDevice(v->scene->ctx->device), "gi_vox_set_items: cudaSetDevice");
  if (nitems > v->w_items_cap) {
    cudaFree(v->w_items);
    v->w_items = nullptr;
    v->w_items_cap = 0;
    cudaError_t e = dalloc(&v->w_items, nitems);
    if (e) return cuda_fail(e, "gi_vox_set_items");
    v->w_items_cap = nitems;
  }
  if (nitems) CK(cudaMemcpy(v->w_items, items, nitems * sizeof(uint4), cudaMemcpyHostToDevice), "gi_vox_set_items: copy");
  v->w_nitems = nitems;
  v->w_threads = nitems ? threads : 0u;
  v->items_gen++;
  return GI_OK;
}

// The raster scratch for n drawn triangles (grown, never shrunk)
static int ensure_raster_scratch(gi_scene *s, uint64_t n, const char *what) {
  if (n >= (1ull << 31)) return fail(GI_ERR_INVALID, "%s: %llu drawn triangles", what, (unsigned long long)n);
  if (n <= s->raster_tris) return GI_OK;
  CK(cudaSetDevice(s->ctx->device), what);
  float4 *rec = nullptr;
  uint32_t *ntile = nullptr, *pre = nullptr, *sums = nullptr, *over = nullptr, *list = nullptr;
  const uint32_t cap = raster_list_cap((uint32_t)n);
  cudaError_t e;
  if ((e = dalloc(&rec, (size_t)3u * n)) || (e = dalloc(&ntile, n)) || (e = dalloc(&pre, n)) ||
      (e = dalloc(&sums, n / 256u + 1u)) || (e = dalloc(&over, n)) ||
      (cap > s->raster_cap && (e = dalloc(&list, cap)))) {
    cudaFree(rec); cudaFree(ntile); cudaFree(pre); cudaFree(sums); cudaFree(over); cudaFree(list);
    return cuda_fail(e, what);
  }
  cudaFree(s->raster_rec); cudaFree(s->raster_ntile); cudaFree(s->raster_pre); cudaFree(s->raster_sums);
  cudaFree(s->raster_over);
  s->raster_rec = rec; s->raster_ntile = ntile; s->raster_pre = pre; s->raster_sums = sums; s->raster_over = over;
  if (list) { cudaFree(s->raster_list); s->raster_list = list; s->raster_cap = cap; }
  s->gen++;
  s->raster_tris = (uint32_t)n;
  return GI_OK;
}

int gi_scene_set_draw_count(gi_scene *s, uint32_t count) {
  if (!s) return fail(GI_ERR_INVALID, "gi_scene_set_draw_count: NULL scene");
  if (count > s->ntris) return fail(GI_ERR_INVALID, "gi_scene_set_draw_count: %u of %u rows", count, s->ntris);
  int st = ensure_raster_scratch(s, (uint64_t)count * s->draw_ninst, "gi_scene_set_draw_count");
  if (st) return st;
  s->ndraw = count;
  s->gen++;
  return GI_OK;
}

int gi_scene_set_static_count(gi_scene *s, uint32_t count) {
  if (!s) return fail(GI_ERR_INVALID, "gi_scene_set_static_count: NULL scene");
  if (count > s->ntris) return fail(GI_ERR_INVALID, "gi_scene_set_static_count: %u of %u rows", count, s->ntris);
  s->static_tris = count == s->ntris ? 0u : count;
  if (count == 0 && s->ntris) s->static_tris = 0xffffffffu;   // every row dynamic: the rebuild reads none
  s->gen++;
  return GI_OK;
}

int gi_scene_set_draw_instances(gi_scene *s, const float *offsets, uint32_t n) {
  if (!s) return fail(GI_ERR_INVALID, "gi_scene_set_draw_instances: NULL scene");
  if (n > 1024) return fail(GI_ERR_INVALID, "gi_scene_set_draw_instances: %u instances (at most 1024)", n);
  if (n > 1 && !offsets) return fail(GI_ERR_INVALID, "gi_scene_set_draw_instances: NULL offsets");
  if (n > 1 && (offsets[0] != 0.0f || offsets[1] != 0.0f || offsets[2] != 0.0f))
    return fail(GI_ERR_INVALID, "gi_scene_set_draw_instances: instance 0 must be at the origin");
  CK(cudaSetDevice(s->ctx->device), "gi_scene_set_draw_instances: cudaSetDevice");
  if (n <= 1) {
    cudaFree(s->draw_inst);
    s->draw_inst = nullptr;
    s->draw_ninst = 1;
    s->gen++;
    return GI_OK;
  }
  int st = ensure_raster_scratch(s, (uint64_t)s->ndraw * n, "gi_scene_set_draw_instances");
  if (st) return st;
  std::vector<float4> h(n);
  for (uint32_t i = 0; i < n; i++) h[i] = make_float4(offsets[3 * i], offsets[3 * i + 1], offsets[3 * i + 2], 0.0f);
  float4 *d = nullptr;
  cudaError_t e;
  if ((e = dalloc(&d, n)) || (e = cudaMemcpy(d, h.data(), n * sizeof(float4), cudaMemcpyHostToDevice))) {
    cudaFree(d);
    return cuda_fail(e, "gi_scene_set_draw_instances");
  }
  cudaFree(s->draw_inst);
  s->draw_inst = d;
  s->draw_ninst = n;
  s->gen++;
  return GI_OK;
}

static int rc_vox_build(gi_vox *v, gi_rc *r, void *stream) {
  if (!r->shadow) return vox_build_sun(v, nullptr, nullptr, 0u, stream);
  if (r->frame_layers > r->shadow_layers)
    return fail(GI_ERR_STATE, "the frame asks for %u shadow-map layers, the map was drawn with %u; draw it again "
                              "(gi_rc_render_shadow)", r->frame_layers, r->shadow_layers);
  return vox_build_sun(v, r->frame, r->shadow, r->shadow_size, stream, r->shadow_layers);
}

int gi_vox_build_sun(gi_vox *v, gi_rc *r, void *stream) {
  if (!r) return fail(GI_ERR_INVALID, "gi_vox_build_sun: NULL rc");
  if (v && v->scene->ctx->device != r->ctx->device) return fail(GI_ERR_INVALID, "gi_vox_build_sun: rc on another device");
  return rc_vox_build(v, r, stream);
}

int gi_vox_read_counters(gi_vox *v, uint32_t hdr[64], void *stream) {
  if (!v || !hdr) return fail(GI_ERR_INVALID, "gi_vox_read_counters: NULL argument");
  CK(cudaSetDevice(v->scene->ctx->device), "gi_vox_read_counters: cudaSetDevice");
  CK(cudaMemcpyAsync(v->hdr, v->dev.hdr, sizeof v->hdr, cudaMemcpyDeviceToHost, S(stream)), "gi_vox_read_counters: copy");
  CK(cudaStreamSynchronize(S(stream)), "gi_vox_read_counters: sync");
  memcpy(hdr, v->hdr, sizeof v->hdr);
  if (v->hdr[6] != 0u)
    return fail(GI_ERR_TIMEOUT, "gi_vox_read_counters: a bounded wait of the rebuild's chained scans gave up (header word 6); "
                "this rebuild's voxel state is not valid");
  return GI_OK;
}

int gi_vox_debug_hold_scan(gi_vox *v, int32_t part) {
  if (!v) return fail(GI_ERR_INVALID, "gi_vox_debug_hold_scan: NULL vox");
  v->dev.scan_hold = part < 0 ? 0u : (uint32_t)part + 1u;
  return GI_OK;
}

int gi_vox_used_bytes(gi_vox *v, uint64_t *persistent, uint64_t *build_temp) {
  if (!v) return fail(GI_ERR_INVALID, "gi_vox_used_bytes: NULL vox");
  uint64_t nb = v->hdr[0] < v->p.max_bricks ? v->hdr[0] : v->p.max_bricks;
  uint64_t nv = v->hdr[1] < v->p.max_voxels ? v->hdr[1] : v->p.max_voxels;
  uint64_t nptr = (uint64_t)v->p.levels * v->p.G * v->p.G * v->p.G;
  // voxel.ts:919-922, with this layout's per-voxel record (16 B attribute + plane + sun visibility)
  if (persistent) *persistent = (GI_HDR + nptr + nb * 18u) * 4u + nv * 24u;
  if (build_temp) *build_temp = nb * 512u * 4u;
  return GI_OK;
}

int gi_vox_read_state(gi_vox *v, uint32_t *ptr, uint32_t *occ, uint32_t *base, uint32_t *code, uint32_t *rep,
                      uint32_t *attr, float *plane, float *sunvis, void *stream) {
  if (!v) return fail(GI_ERR_INVALID, "gi_vox_read_state: NULL vox");
  CK(cudaSetDevice(v->scene->ctx->device), "gi_vox_read_state: cudaSetDevice");
  const VoxDev &d = v->dev;
  size_t nptr = (size_t)v->p.levels * v->p.G * v->p.G * v->p.G, mb = v->p.max_bricks, mv = v->p.max_voxels;
  cudaStream_t st = S(stream);
  if (ptr) CK(cudaMemcpyAsync(ptr, d.ptr, nptr * 4u, cudaMemcpyDeviceToHost, st), "gi_vox_read_state: ptr");
  if (occ) CK(cudaMemcpyAsync(occ, d.occ, mb * 64u, cudaMemcpyDeviceToHost, st), "gi_vox_read_state: occ");
  if (base) CK(cudaMemcpyAsync(base, d.base, mb * 4u, cudaMemcpyDeviceToHost, st), "gi_vox_read_state: base");
  if (code) CK(cudaMemcpyAsync(code, d.code, mb * 4u, cudaMemcpyDeviceToHost, st), "gi_vox_read_state: code");
  if (rep) CK(cudaMemcpyAsync(rep, d.rep, mb * 2048u, cudaMemcpyDeviceToHost, st), "gi_vox_read_state: rep");
  if (attr) CK(cudaMemcpyAsync(attr, d.attr, mv * 16u, cudaMemcpyDeviceToHost, st), "gi_vox_read_state: attr");
  if (plane) CK(cudaMemcpyAsync(plane, d.plane, mv * 4u, cudaMemcpyDeviceToHost, st), "gi_vox_read_state: plane");
  if (sunvis) CK(cudaMemcpyAsync(sunvis, d.sunvis, mv * 4u, cudaMemcpyDeviceToHost, st), "gi_vox_read_state: sunvis");
  CK(cudaStreamSynchronize(st), "gi_vox_read_state: sync");
  return GI_OK;
}

int gi_vox_bytes(gi_vox *v, uint64_t *bytes) {
  if (!v || !bytes) return fail(GI_ERR_INVALID, "gi_vox_bytes: NULL argument");
  *bytes = v->bytes;
  return GI_OK;
}

int gi_scene_set_raster_capacity(gi_scene *s, uint32_t entries) {
  if (!s) return fail(GI_ERR_INVALID, "gi_scene_set_raster_capacity: NULL scene");
  if (entries < 1) return fail(GI_ERR_INVALID, "gi_scene_set_raster_capacity: capacity must be >= 1");
  CK(cudaSetDevice(s->ctx->device), "gi_scene_set_raster_capacity: cudaSetDevice");
  uint32_t *list = nullptr;
  cudaError_t e = dalloc(&list, entries);
  if (e) return cuda_fail(e, "gi_scene_set_raster_capacity");
  cudaFree(s->raster_list);   // synchronises with work still using the old list
  s->raster_list = list;
  s->raster_cap = entries;
  s->gen++;
  return GI_OK;
}

int gi_scene_bytes(gi_scene *s, uint64_t *bytes) {
  if (!s || !bytes) return fail(GI_ERR_INVALID, "gi_scene_bytes: NULL argument");
  *bytes = (uint64_t)s->nverts * (16u + 16u + 32u) + (uint64_t)s->ntris * (16u + 48u + 4u + 4u + 4u) +
           (uint64_t)s->nmats * sizeof(gi_material) + 16u + (s->ntris / 256u + 1u) * 4u + (uint64_t)s->raster_cap * 4u;
  return GI_OK;
}

int gi_vox_destroy(gi_vox *v) {
  if (!v) return GI_OK;
  cudaSetDevice(v->scene->ctx->device);
  free_vox(v);
  delete v;
  return GI_OK;
}

// ---- radiance cascades --------------------------------------------------------------------------------------------------
static size_t atlas_elem_bytes(uint32_t atlas) { return atlas == GI_ATLAS_F32 ? 16u : 8u; }

// gi_rc_create and gi_rc_create_world (wp != NULL)
static int rc_create(gi_ctx *ctx, const gi_rc_params *p, const gi_world_params *wp, uint32_t W, uint32_t H, gi_rc **out) {
  if (!ctx || !p || !out) return fail(GI_ERR_INVALID, "gi_rc_create: NULL argument");
  *out = nullptr;
  if (p->cascades < 1 || p->cascades > 8) return fail(GI_ERR_INVALID, "gi_rc_create: at most 8 cascades (rc.ts:1022), got %u", p->cascades);
  if (W < 1 || H < 1 || W > 16384 || H > 16384) return fail(GI_ERR_INVALID, "gi_rc_create: size %ux%u", W, H);
  if (p->P < 1 || p->P > 1024) return fail(GI_ERR_INVALID, "gi_rc_create: P %u", p->P);
  if (p->atlas > GI_ATLAS_BF16) return fail(GI_ERR_INVALID, "gi_rc_create: atlas %u", p->atlas);
  if (p->dda_cap < 1) return fail(GI_ERR_INVALID, "gi_rc_create: dda_cap must be >= 1");
  if (!(p->k_interval > 0.0f)) return fail(GI_ERR_INVALID, "gi_rc_create: k_interval must be > 0");
  if (wp) {
    if (wp->relocate > GI_RELOCATE_VOXEL) return fail(GI_ERR_INVALID, "gi_rc_create_world: relocate %u", wp->relocate);
    for (uint32_t i = 0; i < p->cascades; i++)
      if (wp->caps[i] < 1u || wp->caps[i] > (1u << 24))
        return fail(GI_ERR_INVALID, "gi_rc_create_world: cascade %u capacity %u (1 .. 2^24)", i, wp->caps[i]);
  }
  CK(cudaSetDevice(ctx->device), "gi_rc_create: cudaSetDevice");
  gi_rc *r = new (std::nothrow) gi_rc;
  if (!r) return fail(GI_ERR_OOM, "gi_rc_create: host allocation");
  memset(&r->dev, 0, sizeof r->dev);
  r->ctx = ctx; r->p = *p; r->W = W; r->H = H;
  RcDev &d = r->dev;
  d.cascades = p->cascades; d.width = W; d.height = H; d.atlas = p->atlas;
  d.vox_scale = p->vox_scale; d.vox_offset = p->vox_offset; d.level_map = p->level_map; d.vox_skip = p->vox_skip;
  d.dda_cap = p->dda_cap; d.stats = p->stats;
  d.trace_order = 0; d.trace_rays = 1;
  d.f32_out = p->f32_out ? 1u : 0u;
  d.irr_f16 = p->irr_f16 ? 1u : 0u;
  // cascade layout (rc.ts:1027-1035)
  uint64_t probe_total = 0, ray_total = 0, dir_total = 0;
  for (uint32_t i = 0; i < p->cascades; i++) {
    CascDev &c = d.c[i];
    uint32_t rc_ = i < p->res_cap ? i : p->res_cap;
    if (rc_ > 10) return delete r, fail(GI_ERR_INVALID, "gi_rc_create: directions per cascade past 4096^2");
    c.res = 4u << rc_;
    uint64_t ts = (uint64_t)p->P << i;
    if (ts > (1u << 20)) return delete r, fail(GI_ERR_INVALID, "gi_rc_create: tile size overflow");
    if (wp) {   // world probes: no screen tiles; probes and atlas entries by capacity (rc.ts:1029)
      c.tile_size = 0; c.tiles_x = wp->caps[i]; c.tiles_y = 1;
    } else {
      c.tile_size = (uint32_t)ts;
      c.tiles_x = (uint32_t)((W + ts - 1) / ts);
      c.tiles_y = (uint32_t)((H + ts - 1) / ts);
    }
    c.probe_off = (uint32_t)probe_total;
    c.rad_off = (uint32_t)ray_total;
    c.ray_off = (uint32_t)ray_total;
    c.dir_off = (uint32_t)dir_total;
    dir_total += (uint64_t)c.res * c.res;
    double b0 = (double)p->k_interval * (pow(4.0, (double)i) - 1.0) / 3.0;
    double b1 = (double)p->k_interval * (pow(4.0, (double)(i + 1)) - 1.0) / 3.0;
    c.b0 = (float)b0; c.b1 = (float)b1;
    c.dirs_log2 = 2u * (2u + rc_);
    c.np = c.tiles_x * c.tiles_y;
    c.inv_tile = c.tile_size && (c.tile_size & (c.tile_size - 1u)) == 0u ? 1.0f / (float)c.tile_size : 0.0f;
    probe_total += (uint64_t)c.tiles_x * c.tiles_y;
    ray_total += (uint64_t)c.tiles_x * c.tiles_y * c.res * c.res;
  }
  if (ray_total >= (1ull << 31)) return delete r, fail(GI_ERR_INVALID, "gi_rc_create: %llu rays past 2^31", (unsigned long long)ray_total);
  d.probes_total = (uint32_t)probe_total;
  d.rays_total = (uint32_t)ray_total;
  r->rad_elem_bytes = atlas_elem_bytes(p->atlas);
  r->sh_elem_bytes = p->f32_out ? 16u : r->rad_elem_bytes;
  r->irr_elem_bytes = p->irr_f16 ? 8u : p->f32_out ? 16u : atlas_elem_bytes(p->atlas);
  r->sh_elems = (size_t)d.c[0].tiles_x * d.c[0].tiles_y * 8u;
  size_t npx = (size_t)W * H;
  r->ntiles = gi_raster_tiles(W, H);
  cudaError_t e;
  ProbeDev *probes = nullptr;
  void *rad = nullptr, *sh = nullptr, *irr = nullptr;
  uint32_t *counts = nullptr, *plevel = nullptr;
  float4 *dirs = nullptr;
  if ((e = dalloc(&r->frame, 160)) || (e = dalloc(&r->depth, npx)) || (e = dalloc(&r->normal, npx)) ||
      (e = cudaMalloc(&r->tag, npx)) || (e = cudaMemset(r->tag, 0, npx)) ||
      (e = dalloc(&r->tile_cnt, (size_t)r->ntiles + 1u)) || (e = dalloc(&r->tile_fill, r->ntiles)) ||
      (e = dalloc(&r->stage, npx)) || (e = dalloc(&probes, probe_total)) ||
      (e = cudaMalloc(&rad, ray_total * r->rad_elem_bytes)) || (e = cudaMalloc(&sh, r->sh_elems * r->sh_elem_bytes)) ||
      (e = cudaMalloc(&irr, npx * r->irr_elem_bytes)) || (e = dalloc(&counts, 96)) ||
      (e = dalloc(&plevel, probe_total)) || (e = dalloc(&dirs, 2u * dir_total))) {
    d.probes = probes; d.rad = rad; d.sh = sh; d.irr = irr; d.counts = counts; d.plevel = plevel; d.dirs = dirs;
    free_rc(r);
    delete r;
    return cuda_fail(e, "gi_rc_create");
  }
  d.probes = probes; d.rad = rad; d.sh = sh; d.irr = irr; d.counts = counts; d.plevel = plevel; d.dirs = dirs;
  d.idirs = dirs + dir_total;
  d.frame = r->frame; d.depth = r->depth; d.normal = r->normal; d.tag = r->tag;
  // the merge's quad averages of a cascade whose resolution is twice the one below
  size_t avg_elems = 1;
  for (uint32_t i = 1; i < p->cascades && !wp; i++)
    if (d.c[i].res == 2u * d.c[i - 1].res) {
      size_t n = (size_t)d.c[i].np * d.c[i].res * d.c[i].res / 4u;
      if (n > avg_elems) avg_elems = n;
    }
  d.mavg[0] = d.mavg[1] = nullptr;
  {
    // k / 255 and (k / 255) / pi for k = 0..255, IEEE f32 quotients
    float tab[512];
    for (int k = 0; k < 256; k++) {
      volatile float a = (float)k / 255.0f;
      volatile float ap = a / 3.14159265f;
      tab[k] = a;
      tab[256 + k] = ap;
    }
    float *u8 = nullptr;
    if ((e = dalloc(&u8, 512)) || (e = cudaMemcpy(u8, tab, sizeof tab, cudaMemcpyHostToDevice))) {
      cudaFree(u8);
      free_rc(r);
      delete r;
      return cuda_fail(e, "gi_rc_create: tables");
    }
    d.unorm8 = u8;
  }
  if ((e = dalloc(&d.mavg[0], avg_elems)) || (e = dalloc(&d.mavg[1], avg_elems))) {
    free_rc(r);
    delete r;
    return cuda_fail(e, "gi_rc_create: merge averages");
  }
  r->mavg_bytes = 2u * avg_elems * sizeof(float4);
  cudaMemset(counts, 0, 96 * 4);
  if ((e = gi_launch_init_dirs(d, dirs, (uint32_t)dir_total, 0)) || (e = cudaDeviceSynchronize())) {
    free_rc(r);
    delete r;
    return cuda_fail(e, "gi_rc_create: direction table");
  }
  r->bytes = r->mavg_bytes + 160 * 4 + npx * (4 + 8 + 16) + (uint64_t)r->ntiles * 8u + 4u + probe_total * 52 + dir_total * 32 + ray_total * r->rad_elem_bytes +
             r->sh_elems * r->sh_elem_bytes + npx * r->irr_elem_bytes + 96 * 4;
  if (wp) {
    WorldDev &w = r->w;
    uint64_t hash_total = 0, look_total = 0;
    for (uint32_t i = 0; i < p->cascades; i++) {
      uint32_t hs = 1;
      while (hs < 2u * wp->caps[i]) hs <<= 1;   // nextPow2(2 cap) (rc.ts:978, :1030)
      w.hash_off[i] = (uint32_t)hash_total; w.hash_mask[i] = hs - 1u; w.cap[i] = wp->caps[i];
      w.look_off[i] = (uint32_t)look_total;
      hash_total += hs;
      look_total += (hs + 2047u) / 2048u + 1u;   // compact's blocks of 2048 slots, + the ticket word
    }
    w.hash_total = (uint32_t)hash_total; w.look_total = (uint32_t)look_total;
    w.relocate = wp->relocate; w.hist_h = w.hash_mask[0] + 1u;
    const size_t cap0 = wp->caps[0];
    if ((e = dalloc(&w.keys, hash_total)) || (e = dalloc(&w.slot_probe, hash_total)) ||
        (e = dalloc(&w.parents, probe_total * 8u)) || (e = dalloc(&w.state, 64)) || (e = dalloc(&w.look, look_total)) ||
        (e = dalloc(&w.hist_tab, 2u * (size_t)w.hist_h)) || (e = dalloc(&w.hist_grid, 2u * cap0)) ||
        (e = dalloc(&w.hist_sh, 16u * cap0)) || (e = cudaMemset(w.state, 0, 64 * 4)) ||
        (e = cudaMemset(w.hist_tab, 0, 2u * (size_t)w.hist_h * 4u)) || (e = cudaMemset(w.parents, 0xff, probe_total * 32u)) ||
        (e = gi_world_tables())) {
      free_rc(r);
      delete r;
      return cuda_fail(e, "gi_rc_create_world");
    }
    r->world = true;
    r->bytes += hash_total * 8u + probe_total * 32u + 64 * 4 + look_total * 8u + 2u * (uint64_t)w.hist_h * 4u +
                cap0 * (2u * 16u + 16u * 16u);
  }
  *out = r;
  return GI_OK;
}

int gi_rc_create(gi_ctx *ctx, const gi_rc_params *p, uint32_t W, uint32_t H, gi_rc **out) {
  return rc_create(ctx, p, nullptr, W, H, out);
}

int gi_rc_create_world(gi_ctx *ctx, const gi_rc_params *p, const gi_world_params *world, uint32_t W, uint32_t H,
                       gi_rc **out) {
  if (!world) return fail(GI_ERR_INVALID, "gi_rc_create_world: NULL world parameters");
  return rc_create(ctx, p, world, W, H, out);
}

int gi_rc_set_frame(gi_rc *r, const void *frame640, void *stream) {
  if (!r || !frame640) return fail(GI_ERR_INVALID, "gi_rc_set_frame: NULL argument");
  const float *f = (const float *)frame640;
  if (f[100] != (float)r->W || f[101] != (float)r->H)
    return fail(GI_ERR_INVALID, "gi_rc_set_frame: frame size %gx%g, cascades made for %ux%u", f[100], f[101], r->W, r->H);
  if (!(f[83] > 0.0f)) return fail(GI_ERR_INVALID, "gi_rc_set_frame: near plane must be > 0");
  CK(cudaSetDevice(r->ctx->device), "gi_rc_set_frame: cudaSetDevice");
  CK(cudaMemcpyAsync(r->frame, frame640, 640, cudaMemcpyHostToDevice, S(stream)), "gi_rc_set_frame: copy");
  r->frame_set = true;
  r->frame_layers = f[156] >= 1.5f ? 2u : 1u;   // shadow.x: the shadow map's layers (frame.ts:20)
  return GI_OK;
}

int gi_rc_set_gbuffer(gi_rc *r, const float *depth, const float *normal4, void *stream) {
  if (!r || !depth || !normal4) return fail(GI_ERR_INVALID, "gi_rc_set_gbuffer: NULL argument");
  CK(cudaSetDevice(r->ctx->device), "gi_rc_set_gbuffer: cudaSetDevice");
  size_t npx = (size_t)r->W * r->H;
  CK(cudaMemcpyAsync(r->depth, depth, npx * 4u, cudaMemcpyHostToDevice, S(stream)), "gi_rc_set_gbuffer: depth");
  CK(cudaMemcpyAsync(r->stage, normal4, npx * 16u, cudaMemcpyHostToDevice, S(stream)), "gi_rc_set_gbuffer: normal");
  CK(gi_launch_normal_f32_to_f16(r->stage, r->normal, (uint32_t)npx, S(stream)), "gi_rc_set_gbuffer: convert");
  r->gbuf_set = true;
  return GI_OK;
}

int gi_rc_set_gbuffer_f16(gi_rc *r, const float *depth, const uint16_t *normal, void *stream) {
  if (!r || !depth || !normal) return fail(GI_ERR_INVALID, "gi_rc_set_gbuffer_f16: NULL argument");
  CK(cudaSetDevice(r->ctx->device), "gi_rc_set_gbuffer_f16: cudaSetDevice");
  size_t npx = (size_t)r->W * r->H;
  CK(cudaMemcpyAsync(r->depth, depth, npx * 4u, cudaMemcpyHostToDevice, S(stream)), "gi_rc_set_gbuffer_f16: depth");
  CK(cudaMemcpyAsync(r->normal, normal, npx * 8u, cudaMemcpyHostToDevice, S(stream)), "gi_rc_set_gbuffer_f16: normal");
  r->gbuf_set = true;
  return GI_OK;
}

int gi_rc_set_gbuffer_rgb16f(gi_rc *r, const float *depth, const uint16_t *normal, void *stream) {
  if (!r || !depth || !normal) return fail(GI_ERR_INVALID, "gi_rc_set_gbuffer_rgb16f: NULL argument");
  CK(cudaSetDevice(r->ctx->device), "gi_rc_set_gbuffer_rgb16f: cudaSetDevice");
  size_t npx = (size_t)r->W * r->H;
  CK(cudaMemcpyAsync(r->depth, depth, npx * 4u, cudaMemcpyHostToDevice, S(stream)), "gi_rc_set_gbuffer_rgb16f: depth");
  CK(cudaMemcpyAsync(r->stage, normal, npx * 6u, cudaMemcpyHostToDevice, S(stream)), "gi_rc_set_gbuffer_rgb16f: normal");
  CK(gi_launch_normal_rgb_to_rgba(reinterpret_cast<const uint16_t *>(r->stage), r->normal, (uint32_t)npx, S(stream)),
     "gi_rc_set_gbuffer_rgb16f: expand");
  r->gbuf_set = true;
  return GI_OK;
}

// From the first tagged G-buffer on, the world gather reads the tags (a kernel variant; graphs captured before are
// refused, as their launches hold the variant without)
static void use_tags(gi_rc *r) {
  if (r->dev.tag_any) return;
  r->dev.tag_any = 1u;
  r->gen++;
}

int gi_rc_set_gbuffer_tag(gi_rc *r, const uint8_t *tag, void *stream) {
  if (!r || !tag) return fail(GI_ERR_INVALID, "gi_rc_set_gbuffer_tag: NULL argument");
  CK(cudaSetDevice(r->ctx->device), "gi_rc_set_gbuffer_tag: cudaSetDevice");
  CK(cudaMemcpyAsync(r->tag, tag, (size_t)r->W * r->H, cudaMemcpyHostToDevice, S(stream)), "gi_rc_set_gbuffer_tag: copy");
  use_tags(r);
  return GI_OK;
}

int gi_rc_render_gbuffer(gi_rc *r, gi_scene *s, void *stream) {
  if (!r || !s) return fail(GI_ERR_INVALID, "gi_rc_render_gbuffer: NULL argument");
  if (!r->frame_set) return fail(GI_ERR_STATE, "gi_rc_render_gbuffer: no frame set");
  if (s->ctx->device != r->ctx->device) return fail(GI_ERR_INVALID, "gi_rc_render_gbuffer: scene on another device");
  CK(cudaSetDevice(r->ctx->device), "gi_rc_render_gbuffer: cudaSetDevice");
  RasterDev rd;
  rd.rec = s->raster_rec; rd.ntile = s->raster_ntile; rd.pre = s->raster_pre; rd.sums = s->raster_sums;
  rd.counter = s->raster_counter; rd.list = s->raster_list; rd.over = s->raster_over;
  rd.tile_cnt = r->tile_cnt; rd.tile_fill = r->tile_fill; rd.list_cap = s->raster_cap; rd.ntiles = r->ntiles;
  CK(gi_launch_gbuffer(s->raster_dev(), r->frame, r->W, r->H, r->depth, r->normal, r->tag, rd, r->ctx->sm_count, S(stream)),
     "gi_rc_render_gbuffer: launch");
  if (s->mat_flags & 12u) use_tags(r);   // toon or object materials: the tags matter
  r->gbuf_set = true;
  return GI_OK;
}

int gi_rc_render_shadow(gi_rc *r, gi_scene *s, uint32_t size, void *stream) {
  if (!r || !s) return fail(GI_ERR_INVALID, "gi_rc_render_shadow: NULL argument");
  if (size > 16384u) return fail(GI_ERR_INVALID, "gi_rc_render_shadow: size %u (at most 16384)", size);
  if (s->ctx->device != r->ctx->device) return fail(GI_ERR_INVALID, "gi_rc_render_shadow: scene on another device");
  CK(cudaSetDevice(r->ctx->device), "gi_rc_render_shadow: cudaSetDevice");
  if (size == 0) {
    cudaFree(r->shadow);
    r->shadow = nullptr;
    r->shadow_size = r->shadow_layers = 0;
    r->gen++;
    return GI_OK;
  }
  if (!r->frame_set) return fail(GI_ERR_STATE, "gi_rc_render_shadow: no frame set");
  cudaError_t e;
  const uint32_t layers = r->frame_layers;
  if (size != r->shadow_size || layers != r->shadow_layers) {
    cudaFree(r->shadow);
    r->shadow = nullptr;
    r->shadow_size = r->shadow_layers = 0;
    r->gen++;
    if ((e = dalloc(&r->shadow, (size_t)size * size * layers))) return cuda_fail(e, "gi_rc_render_shadow");
    r->shadow_size = size;
    r->shadow_layers = layers;
  }
  uint32_t nt = s->ndraw * s->draw_ninst;   // the drawn triangles (ensure_raster_scratch bounds the product)
  if (nt > r->sm_tris || !r->sm_counter) {
    cudaFree(r->sm_rec); cudaFree(r->sm_pre); cudaFree(r->sm_sums); cudaFree(r->sm_counter);
    r->sm_rec = nullptr; r->sm_pre = r->sm_sums = r->sm_counter = nullptr; r->sm_tris = 0;
    size_t cap = nt ? nt : 1u;
    if ((e = dalloc(&r->sm_rec, 4u * cap)) || (e = dalloc(&r->sm_pre, cap)) || (e = dalloc(&r->sm_sums, (cap + 255u) / 256u)) ||
        (e = dalloc(&r->sm_counter, 4)))
      return cuda_fail(e, "gi_rc_render_shadow");
    r->sm_tris = (uint32_t)cap;
  }
  ShadowRaster sr;
  sr.map = r->shadow; sr.rec = r->sm_rec; sr.pre = r->sm_pre; sr.sums = r->sm_sums; sr.counter = r->sm_counter;
  for (uint32_t l = 0; l < layers; l++) {   // layer 0: lightViewProj (frame word 64), layer 1: lightViewProjFar (140)
    sr.map = r->shadow + (size_t)l * size * size;
    CK(gi_launch_shadow(s->raster_dev(), r->frame + (l ? 140 : 64), size, sr, r->ctx->sm_count, S(stream)),
       "gi_rc_render_shadow: launch");
  }
  return GI_OK;
}

// sfDir (bounce.ts:147-152): z = 1 - (2i + 1) / n, r = sqrt(max(0, 1 - z^2)), phi = 2 pi fract(i 0.618033988749), the
// f32 steps as the shader does them and cos / sin of the f32 phi in double precision (the shader's are
// implementation-defined)
static void bounce_dirs(uint32_t n, float4 *out) {
  for (uint32_t i = 0; i < n; i++) {
    volatile float fi = (float)i, fn = (float)n;
    volatile float z = 1.0f - (2.0f * fi + 1.0f) / fn;
    volatile float zz = 1.0f - z * z;
    float r = sqrtf(zz > 0.0f ? zz : 0.0f);
    volatile float xi = fi * 0.618033988749f;
    volatile float fr = xi - floorf(xi);
    volatile float phi = 2.0f * 3.14159265f * fr;
    volatile float cx = (float)cos((double)phi), sy = (float)sin((double)phi);
    volatile float x = r * cx, y = r * sy;
    out[i] = make_float4(x, y, z, 0.0f);
  }
}

int gi_rc_set_bounce(gi_rc *r, gi_vox *v, const gi_bounce_params *p) {
  if (!r) return fail(GI_ERR_INVALID, "gi_rc_set_bounce: NULL rc");
  CK(cudaSetDevice(r->ctx->device), "gi_rc_set_bounce: cudaSetDevice");
  cudaFree((void *)r->bn.dirs); cudaFree(r->bn.vol[0]); cudaFree(r->bn.vol[1]); cudaFree(r->bn.list); cudaFree(r->bn.inj);
  cudaFree(r->bn.ray_out);
  r->bn = BounceDev{};
  r->bounce = false;
  r->gen++;
  r->bn_vox = nullptr;
  r->dev.bn_inj = nullptr;
  if (!p) return GI_OK;
  if (!v) return fail(GI_ERR_INVALID, "gi_rc_set_bounce: NULL voxel world");
  if (v->scene->ctx->device != r->ctx->device) return fail(GI_ERR_INVALID, "gi_rc_set_bounce: voxel world on another device");
  if (!(p->cell > 0.0f) || p->dx < 1 || p->dy < 1 || p->dz < 1 || p->dx > 1024 || p->dy > 1024 || p->dz > 1024 ||
      (uint64_t)p->dx * p->dy * p->dz > (1u << 24) || p->rays < 1 || p->rays > 26 || p->div < 1)
    return fail(GI_ERR_INVALID, "gi_rc_set_bounce: cell > 0, dims 1..1024 (at most 2^24 probes), rays 1..26, div >= 1");
  BounceDev &b = r->bn;
  b.cell = p->cell; b.v0 = v->dev.vs[0];
  b.dx = p->dx; b.dy = p->dy; b.dz = p->dz; b.rays = p->rays; b.div = p->div; b.n = p->dx * p->dy * p->dz;
  b.levels = v->dev.levels;
  size_t texels = (size_t)b.dx * b.dy * (6u * b.dz + 1u);
  float4 hdirs[32];
  bounce_dirs(b.rays, hdirs);
  float4 *dirs = nullptr;
  cudaError_t e;
  if ((e = dalloc(&dirs, b.rays)) || (e = dalloc(&b.vol[0], texels)) || (e = dalloc(&b.vol[1], texels)) ||
      (e = dalloc(&b.list, 4u + (size_t)b.n)) || (e = dalloc(&b.inj, (size_t)v->p.max_voxels)) ||
      (e = dalloc(&b.ray_out, (size_t)b.n * (b.rays + 6u)))) {
    cudaFree(dirs); b.dirs = nullptr;
    cudaFree(b.vol[0]); cudaFree(b.vol[1]); cudaFree(b.list); cudaFree(b.inj); cudaFree(b.ray_out);
    r->bn = BounceDev{};
    return cuda_fail(e, "gi_rc_set_bounce");
  }
  b.dirs = dirs;
  CK(cudaMemcpy(dirs, hdirs, b.rays * sizeof(float4), cudaMemcpyHostToDevice), "gi_rc_set_bounce: copy");
  CK(cudaMemset(b.vol[0], 0, texels * sizeof(uint2)), "gi_rc_set_bounce: clear");
  CK(cudaMemset(b.vol[1], 0, texels * sizeof(uint2)), "gi_rc_set_bounce: clear");
  CK(cudaMemset(b.list, 0, (4u + (size_t)b.n) * 4u), "gi_rc_set_bounce: clear");
  CK(cudaMemset(b.inj, 0, (size_t)v->p.max_voxels * sizeof(uint4)), "gi_rc_set_bounce: clear");
  r->bounce = true;
  r->bn_vox = v;
  r->dev.bn_inj = b.inj;
  return GI_OK;
}

int gi_rc_solve(gi_rc *r, gi_vox *v, void *stream) {
  if (!r || !v) return fail(GI_ERR_INVALID, "gi_rc_solve: NULL argument");
  if (r->bounce && v != r->bn_vox) return fail(GI_ERR_INVALID, "gi_rc_solve: multi-bounce is bound to another voxel world");
  if (!r->frame_set) return fail(GI_ERR_STATE, "gi_rc_solve: no frame set");
  if (!r->gbuf_set) return fail(GI_ERR_STATE, "gi_rc_solve: no G-buffer set");
  if (!v->updated) return fail(GI_ERR_STATE, "gi_rc_solve: the voxel world was never updated");
  if (v->scene->ctx->device != r->ctx->device) return fail(GI_ERR_INVALID, "gi_rc_solve: voxel world on another device");
  CK(cudaSetDevice(r->ctx->device), "gi_rc_solve: cudaSetDevice");
  if (r->world && !r->w.keys) return fail(GI_ERR_STATE, "gi_rc_solve: the world-probe buffers are missing");
  r->dev.hits = r->debug_hits ? r->hits : nullptr;
  r->dev.rad_traced = r->debug_hits ? r->rad_traced : nullptr;
  CK(gi_launch_rc_solve(r->dev, v->dev, r->ctx->sm_count, S(stream), r->timing ? r->ev + 1 : nullptr, &r->launch,
                        r->bounce ? &r->bn : nullptr, r->world ? &r->w : nullptr),
     "gi_rc_solve: launch");
  r->timed = r->timing;
  r->timed_vox = false;
  return GI_OK;
}

int gi_solve(gi_rc *r, gi_vox *v, void *stream) {
  if (!r || !v) return fail(GI_ERR_INVALID, "gi_solve: NULL argument");
  if (r->timing) {
    CK(cudaSetDevice(r->ctx->device), "gi_solve: cudaSetDevice");
    CK(cudaEventRecord(r->ev[0], S(stream)), "gi_solve: event");
  }
  int st = rc_vox_build(v, r, stream);
  if (st != GI_OK) return st;
  if (r->dyn) {   // the dynamic layer after the static rebuild (rcrun.ts encodeFrame: one 'vox' pass holds both)
    if (r->dyn->vox != v) return fail(GI_ERR_INVALID, "gi_solve: the rc's dynamic layer belongs to another voxel world");
    CK(gi_launch_dyn_build(r->dyn->dev, v->dev, v->scene->dev(), r->frame, r->shadow,
                           r->shadow ? r->shadow_size : 0u, r->shadow_layers,
                           r->ctx->sm_count, S(stream)), "gi_solve: dynamic layer");
  }
  st = gi_rc_solve(r, v, stream);
  r->timed_vox = st == GI_OK && r->timing;
  return st;
}

int gi_rc_graph_capture(gi_rc *r, gi_vox *v, void *stream) {
  if (!r || !v) return fail(GI_ERR_INVALID, "gi_rc_graph_capture: NULL argument");
  if (!stream) return fail(GI_ERR_INVALID, "gi_rc_graph_capture: the legacy default stream cannot be captured; pass a stream");
  if (!r->frame_set || !r->gbuf_set || !v->updated) return fail(GI_ERR_STATE, "gi_rc_graph_capture: frame, G-buffer and voxel window must be set first");
  CK(cudaSetDevice(r->ctx->device), "gi_rc_graph_capture: cudaSetDevice");
  if (r->graph) { cudaGraphExecDestroy(r->graph); r->graph = nullptr; r->graph_vox = nullptr; }
  bool timing = r->timing;
  r->timing = false;   // no event records inside the graph
  CK(cudaStreamBeginCapture(S(stream), cudaStreamCaptureModeThreadLocal), "gi_rc_graph_capture: begin");
  int st = gi_solve(r, v, stream);
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(S(stream), &g);
  r->timing = timing;
  if (st != GI_OK) { if (g) cudaGraphDestroy(g); return st; }
  if (e != cudaSuccess) return cuda_fail(e, "gi_rc_graph_capture: end");
  e = cudaGraphInstantiate(&r->graph, g, 0);
  r->graph_gen = r->gen;
  cudaGraphDestroy(g);
  if (e != cudaSuccess) { r->graph = nullptr; return cuda_fail(e, "gi_rc_graph_capture: instantiate"); }
  r->graph_vox = v;
  r->graph_items_gen = v->items_gen;
  r->graph_scene_gen = v->scene->gen;
  return GI_OK;
}

int gi_rc_graph_capture_frame(gi_rc *r, gi_vox *v, gi_scene *sc, void *irr_out, void *stream) {
  if (!r || !v || !sc) return fail(GI_ERR_INVALID, "gi_rc_graph_capture_frame: NULL argument");
  if (!stream) return fail(GI_ERR_INVALID, "gi_rc_graph_capture_frame: the legacy default stream cannot be captured; pass a stream");
  if (!r->frame_set || !v->updated) return fail(GI_ERR_STATE, "gi_rc_graph_capture_frame: frame and voxel window must be set first");
  if (v->scene != sc) return fail(GI_ERR_INVALID, "gi_rc_graph_capture_frame: the voxel world is built from another scene");
  CK(cudaSetDevice(r->ctx->device), "gi_rc_graph_capture_frame: cudaSetDevice");
  if (r->graph) { cudaGraphExecDestroy(r->graph); r->graph = nullptr; r->graph_vox = nullptr; }
  bool timing = r->timing;
  r->timing = false;
  CK(cudaStreamBeginCapture(S(stream), cudaStreamCaptureModeThreadLocal), "gi_rc_graph_capture_frame: begin");
  int st = sc->rigid_n ? gi_scene_rigid_apply(sc, stream) : GI_OK;
  if (st == GI_OK) st = gi_rc_render_gbuffer(r, sc, stream);
  if (st == GI_OK) st = gi_solve(r, v, stream);
  if (st == GI_OK && irr_out) {
    cudaError_t ce = cudaMemcpyAsync(irr_out, r->dev.irr, (size_t)r->W * r->H * r->irr_elem_bytes,
                                     cudaMemcpyDefault, S(stream));
    if (ce != cudaSuccess) st = cuda_fail(ce, "gi_rc_graph_capture_frame: readback");
  }
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(S(stream), &g);
  r->timing = timing;
  if (st != GI_OK) { if (g) cudaGraphDestroy(g); return st; }
  if (e != cudaSuccess) return cuda_fail(e, "gi_rc_graph_capture_frame: end");
  e = cudaGraphInstantiate(&r->graph, g, 0);
  r->graph_gen = r->gen;
  cudaGraphDestroy(g);
  if (e != cudaSuccess) { r->graph = nullptr; return cuda_fail(e, "gi_rc_graph_capture_frame: instantiate"); }
  r->graph_vox = v;
  r->graph_items_gen = v->items_gen;
  r->graph_scene_gen = v->scene->gen;
  return GI_OK;
}

int gi_rc_graph_launch(gi_rc *r, void *stream) {
  if (!r) return fail(GI_ERR_INVALID, "gi_rc_graph_launch: NULL rc");
  if (!r->graph) return fail(GI_ERR_STATE, "gi_rc_graph_launch: no graph captured");
  if (r->graph_vox && r->graph_vox->items_gen != r->graph_items_gen)
    return fail(GI_ERR_STATE, "gi_rc_graph_launch: the voxel world's work items changed since the capture; capture again");
  if (r->graph_vox && r->graph_vox->scene->gen != r->graph_scene_gen)
    return fail(GI_ERR_STATE, "gi_rc_graph_launch: the scene's textures, rigid objects, draw counts or raster buffers "
                              "changed since the capture; capture again");
  if (r->gen != r->graph_gen)
    return fail(GI_ERR_STATE, "gi_rc_graph_launch: the shadow map, bounce volume or dynamic layer changed since the "
                              "capture; capture again");
  if (r->shadow && r->frame_layers > r->shadow_layers)
    return fail(GI_ERR_STATE, "gi_rc_graph_launch: the frame asks for %u shadow layers, the map has %u; draw it again",
                r->frame_layers, r->shadow_layers);
  CK(cudaSetDevice(r->ctx->device), "gi_rc_graph_launch: cudaSetDevice");
  CK(cudaGraphLaunch(r->graph, S(stream)), "gi_rc_graph_launch");
  r->timed = false;
  return GI_OK;
}

// ---- batches of solves --------------------------------------------------------------------------------------------------
struct gi_batch {
  gi_ctx *ctx;
  uint32_t n = 0;
  gi_rc **rcs = nullptr;
  gi_vox **voxes = nullptr;
  cudaStream_t *streams = nullptr;
  cudaEvent_t *done = nullptr;
  cudaEvent_t start = nullptr;
  cudaGraphExec_t graph = nullptr;
  // gi_batch_capture_passes: the solves' descriptors and work prefixes on the device
  RcDev *d_rc = nullptr;
  VoxDev *d_vox = nullptr;
  uint32_t *d_pre = nullptr;
  uint64_t *gens = nullptr;   // each rc's gen at the capture
  uint64_t *sgens = nullptr;  // each voxel world's scene gen at the capture
};

static void free_batch(gi_batch *b) {
  if (b->graph) cudaGraphExecDestroy(b->graph);
  for (uint32_t i = 0; i < b->n; i++) {
    if (b->streams && b->streams[i]) cudaStreamDestroy(b->streams[i]);
    if (b->done && b->done[i]) cudaEventDestroy(b->done[i]);
  }
  if (b->start) cudaEventDestroy(b->start);
  cudaFree(b->d_rc); cudaFree(b->d_vox); cudaFree(b->d_pre);
  delete[] b->rcs; delete[] b->voxes; delete[] b->streams; delete[] b->done; delete[] b->gens; delete[] b->sgens;
}

int gi_batch_create(gi_ctx *ctx, gi_rc *const *rcs, gi_vox *const *voxes, uint32_t n, gi_batch **out) {
  if (!ctx || !rcs || !voxes || !out) return fail(GI_ERR_INVALID, "gi_batch_create: NULL argument");
  *out = nullptr;
  if (n < 1 || n > 4096) return fail(GI_ERR_INVALID, "gi_batch_create: %u solves (1..4096)", n);
  for (uint32_t i = 0; i < n; i++) {
    if (!rcs[i] || !voxes[i]) return fail(GI_ERR_INVALID, "gi_batch_create: solve %u has a NULL handle", i);
    if (rcs[i]->ctx->device != ctx->device || voxes[i]->scene->ctx->device != ctx->device)
      return fail(GI_ERR_INVALID, "gi_batch_create: solve %u lives on another device", i);
    for (uint32_t j = 0; j < i; j++)
      if (rcs[j] == rcs[i] || voxes[j] == voxes[i])
        return fail(GI_ERR_INVALID, "gi_batch_create: solves %u and %u share a handle (their work would race)", j, i);
  }
  CK(cudaSetDevice(ctx->device), "gi_batch_create: cudaSetDevice");
  gi_batch *b = new (std::nothrow) gi_batch;
  if (!b) return fail(GI_ERR_OOM, "gi_batch_create: host allocation");
  b->ctx = ctx;
  b->rcs = new (std::nothrow) gi_rc *[n];
  b->voxes = new (std::nothrow) gi_vox *[n];
  b->streams = new (std::nothrow) cudaStream_t[n]();
  b->done = new (std::nothrow) cudaEvent_t[n]();
  b->gens = new (std::nothrow) uint64_t[n]();
  b->sgens = new (std::nothrow) uint64_t[n]();
  if (!b->rcs || !b->voxes || !b->streams || !b->done || !b->gens || !b->sgens) { free_batch(b); delete b; return fail(GI_ERR_OOM, "gi_batch_create: host allocation"); }
  b->n = n;
  cudaError_t e = cudaEventCreateWithFlags(&b->start, cudaEventDisableTiming);
  for (uint32_t i = 0; i < n && e == cudaSuccess; i++) {
    b->rcs[i] = rcs[i];
    b->voxes[i] = voxes[i];
    e = cudaStreamCreateWithFlags(&b->streams[i], cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->done[i], cudaEventDisableTiming);
  }
  if (e != cudaSuccess) { free_batch(b); delete b; return cuda_fail(e, "gi_batch_create"); }
  *out = b;
  return GI_OK;
}

int gi_batch_capture(gi_batch *b, void *stream) {
  if (!b) return fail(GI_ERR_INVALID, "gi_batch_capture: NULL batch");
  if (!stream) return fail(GI_ERR_INVALID, "gi_batch_capture: the legacy default stream cannot be captured; pass a stream");
  for (uint32_t i = 0; i < b->n; i++)
    if (!b->rcs[i]->frame_set || !b->rcs[i]->gbuf_set || !b->voxes[i]->updated)
      return fail(GI_ERR_STATE, "gi_batch_capture: solve %u lacks its frame, G-buffer or voxel window", i);
  CK(cudaSetDevice(b->ctx->device), "gi_batch_capture: cudaSetDevice");
  if (b->graph) { cudaGraphExecDestroy(b->graph); b->graph = nullptr; }
  cudaStream_t st = S(stream);
  CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "gi_batch_capture: begin");
  int status = GI_OK;
  cudaError_t e = cudaEventRecord(b->start, st);
  for (uint32_t i = 0; i < b->n && e == cudaSuccess && status == GI_OK; i++) {
    e = cudaStreamWaitEvent(b->streams[i], b->start, 0);   // fork: every solve's chain starts from the batch start
    if (e != cudaSuccess) break;
    bool timing = b->rcs[i]->timing;
    b->rcs[i]->timing = false;
    status = gi_solve(b->rcs[i], b->voxes[i], b->streams[i]);
    b->rcs[i]->timing = timing;
    if (status == GI_OK) e = cudaEventRecord(b->done[i], b->streams[i]);
    if (e == cudaSuccess && status == GI_OK) e = cudaStreamWaitEvent(st, b->done[i], 0);   // join
  }
  cudaGraph_t g = nullptr;
  cudaError_t e2 = cudaStreamEndCapture(st, &g);
  if (status != GI_OK) { if (g) cudaGraphDestroy(g); return status; }
  if (e != cudaSuccess) { if (g) cudaGraphDestroy(g); return cuda_fail(e, "gi_batch_capture"); }
  if (e2 != cudaSuccess) return cuda_fail(e2, "gi_batch_capture: end");
  e = cudaGraphInstantiate(&b->graph, g, 0);
  for (uint32_t i = 0; i < b->n; i++) { b->gens[i] = b->rcs[i]->gen; b->sgens[i] = b->voxes[i]->scene->gen; }
  cudaGraphDestroy(g);
  if (e != cudaSuccess) { b->graph = nullptr; return cuda_fail(e, "gi_batch_capture: instantiate"); }
  return GI_OK;
}

int gi_batch_capture_passes(gi_batch *b, void *stream) {
  if (!b) return fail(GI_ERR_INVALID, "gi_batch_capture_passes: NULL batch");
  if (!stream) return fail(GI_ERR_INVALID, "gi_batch_capture_passes: the legacy default stream cannot be captured; pass a stream");
  const uint32_t n = b->n;
  const RcDev &r0 = b->rcs[0]->dev;
  for (uint32_t i = 0; i < n; i++) {
    gi_rc *r = b->rcs[i];
    if (!r->frame_set || !r->gbuf_set || !b->voxes[i]->updated)
      return fail(GI_ERR_STATE, "gi_batch_capture_passes: solve %u lacks its frame, G-buffer or voxel window", i);
    if (r->dev.atlas != r0.atlas || r->dev.c[0].tile_size != r0.c[0].tile_size)
      return fail(GI_ERR_INVALID, "gi_batch_capture_passes: solve %u has another atlas format or probe spacing than solve 0", i);
    if (r->bounce) return fail(GI_ERR_INVALID, "gi_batch_capture_passes: solve %u has multi-bounce on (capture its chain with gi_batch_capture)", i);
    if (r->world) return fail(GI_ERR_INVALID, "gi_batch_capture_passes: solve %u has world probes (capture its chain with gi_batch_capture)", i);
    if (r->dyn) return fail(GI_ERR_INVALID, "gi_batch_capture_passes: solve %u reads a dynamic layer (capture its chain with gi_batch_capture)", i);
  }
  const uint32_t P0 = r0.c[0].tile_size;
  if (P0 != 8u && P0 != 16u && P0 != 32u)
    return fail(GI_ERR_INVALID, "gi_batch_capture_passes: probe spacing %u (8, 16 or 32)", P0);
  CK(cudaSetDevice(b->ctx->device), "gi_batch_capture_passes: cudaSetDevice");
  // descriptors and prefixes, built on the host
  std::vector<RcDev> hrc(n);
  std::vector<VoxDev> hvox(n);
  uint32_t max_casc = 0;
  for (uint32_t i = 0; i < n; i++) max_casc = std::max(max_casc, b->rcs[i]->dev.cascades);
  const size_t stride = n + 1u;
  std::vector<uint32_t> pre((3u + max_casc) * stride, 0u);   // setup, rays, gather, then merge steps
  uint32_t *setup = pre.data(), *rays = setup + stride, *gath = rays + stride, *merge = gath + stride;
  BatchSizes z = {};
  z.atlas = r0.atlas;
  z.P0 = P0;
  for (uint32_t i = 0; i < n; i++) {
    gi_rc *r = b->rcs[i];
    r->dev.hits = r->debug_hits ? r->hits : nullptr;
    r->dev.rad_traced = r->debug_hits ? r->rad_traced : nullptr;
    hrc[i] = r->dev;
    hvox[i] = b->voxes[i]->dev;
    const RcDev &d = r->dev;
    setup[i + 1] = setup[i] + (d.probes_total + 255u) / 256u;
    rays[i + 1] = rays[i] + (d.rays_total + 31u) / 32u * 32u;
    const uint32_t th = 32u / P0, ntx = (r->W + P0 / 2u + P0 - 1u) / P0, nty = (r->H + P0 / 2u + th - 1u) / th;
    gath[i + 1] = gath[i] + ((ntx + 1u) / 2u) * ((nty + 3u) / 4u);
    for (uint32_t k = 0; k < max_casc; k++) {
      uint32_t blocks = 0;
      if (k < d.cascades) {
        const CascDev &L = d.c[d.cascades - 1u - k];
        blocks = (L.np * (L.res * L.res / 4u) + 255u) / 256u;
      }
      merge[k * stride + i + 1] = merge[k * stride + i] + blocks;
    }
  }
  z.setup_blocks = setup[n];
  z.gather_blocks = gath[n];
  for (uint32_t k = 0; k < max_casc; k++) z.merge_blocks[k] = merge[k * stride + n];
  cudaFree(b->d_rc); cudaFree(b->d_vox); cudaFree(b->d_pre);
  b->d_rc = nullptr; b->d_vox = nullptr; b->d_pre = nullptr;
  cudaError_t e;
  if ((e = dalloc(&b->d_rc, n)) || (e = dalloc(&b->d_vox, n)) || (e = dalloc(&b->d_pre, pre.size() + 1u)))
    return cuda_fail(e, "gi_batch_capture_passes");
  CK(cudaMemcpy(b->d_rc, hrc.data(), n * sizeof(RcDev), cudaMemcpyHostToDevice), "gi_batch_capture_passes: copy");
  CK(cudaMemcpy(b->d_vox, hvox.data(), n * sizeof(VoxDev), cudaMemcpyHostToDevice), "gi_batch_capture_passes: copy");
  CK(cudaMemcpy(b->d_pre, pre.data(), pre.size() * 4u, cudaMemcpyHostToDevice), "gi_batch_capture_passes: copy");
  BatchDev B;
  B.rc = b->d_rc; B.vox = b->d_vox; B.n = n; B.max_casc = max_casc;
  B.setup_blk = b->d_pre; B.ray_pre = b->d_pre + stride; B.gather_blk = b->d_pre + 2u * stride;
  B.merge_blk = b->d_pre + 3u * stride; B.counter = b->d_pre + pre.size();
  if (b->graph) { cudaGraphExecDestroy(b->graph); b->graph = nullptr; }
  cudaStream_t st = S(stream);
  CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "gi_batch_capture_passes: begin");
  int status = GI_OK;
  e = cudaEventRecord(b->start, st);
  // the rebuilds, each on its own stream from the batch start
  for (uint32_t i = 0; i < n && e == cudaSuccess && status == GI_OK; i++) {
    gi_rc *r = b->rcs[i];
    e = cudaStreamWaitEvent(b->streams[i], b->start, 0);
    if (e != cudaSuccess) break;
    status = rc_vox_build(b->voxes[i], r, b->streams[i]);
    if (status == GI_OK) e = cudaEventRecord(b->done[i], b->streams[i]);
    if (e == cudaSuccess && status == GI_OK) e = cudaStreamWaitEvent(st, b->done[i], 0);
  }
  // then one launch per pass over every solve
  if (e == cudaSuccess && status == GI_OK) e = gi_launch_batch_passes(B, z, b->ctx->sm_count, st);
  cudaGraph_t g = nullptr;
  cudaError_t e2 = cudaStreamEndCapture(st, &g);
  if (status != GI_OK) { if (g) cudaGraphDestroy(g); return status; }
  if (e != cudaSuccess) { if (g) cudaGraphDestroy(g); return cuda_fail(e, "gi_batch_capture_passes"); }
  if (e2 != cudaSuccess) return cuda_fail(e2, "gi_batch_capture_passes: end");
  e = cudaGraphInstantiate(&b->graph, g, 0);
  for (uint32_t i = 0; i < b->n; i++) { b->gens[i] = b->rcs[i]->gen; b->sgens[i] = b->voxes[i]->scene->gen; }
  cudaGraphDestroy(g);
  if (e != cudaSuccess) { b->graph = nullptr; return cuda_fail(e, "gi_batch_capture_passes: instantiate"); }
  return GI_OK;
}

int gi_batch_launch(gi_batch *b, void *stream) {
  if (!b) return fail(GI_ERR_INVALID, "gi_batch_launch: NULL batch");
  if (!b->graph) return fail(GI_ERR_STATE, "gi_batch_launch: no graph captured");
  for (uint32_t i = 0; i < b->n; i++) {
    if (b->voxes[i]->scene->gen != b->sgens[i])
      return fail(GI_ERR_STATE, "gi_batch_launch: solve %u's scene changed its buffers since the capture; capture again", i);
    if (b->rcs[i]->gen != b->gens[i])
      return fail(GI_ERR_STATE, "gi_batch_launch: solve %u's shadow map, bounce volume or dynamic layer changed since "
                                "the capture; capture again", i);
    if (b->rcs[i]->shadow && b->rcs[i]->frame_layers > b->rcs[i]->shadow_layers)
      return fail(GI_ERR_STATE, "gi_batch_launch: solve %u's frame asks for more shadow layers than its map has", i);
  }
  CK(cudaSetDevice(b->ctx->device), "gi_batch_launch: cudaSetDevice");
  CK(cudaGraphLaunch(b->graph, S(stream)), "gi_batch_launch");
  return GI_OK;
}

int gi_batch_destroy(gi_batch *b) {
  if (!b) return GI_OK;
  cudaSetDevice(b->ctx->device);
  free_batch(b);
  delete b;
  return GI_OK;
}

int gi_rc_set_timing(gi_rc *r, int on) {
  if (!r) return fail(GI_ERR_INVALID, "gi_rc_set_timing: NULL rc");
  CK(cudaSetDevice(r->ctx->device), "gi_rc_set_timing: cudaSetDevice");
  if (on && !r->ev[0])
    for (cudaEvent_t &e : r->ev) CK(cudaEventCreate(&e), "gi_rc_set_timing: cudaEventCreate");
  r->timing = on != 0;
  return GI_OK;
}

int gi_rc_pass_times(gi_rc *r, float ms[5]) {
  if (!r || !ms) return fail(GI_ERR_INVALID, "gi_rc_pass_times: NULL argument");
  if (!r->timed) return fail(GI_ERR_STATE, "gi_rc_pass_times: the last solve was not timed (gi_rc_set_timing)");
  CK(cudaSetDevice(r->ctx->device), "gi_rc_pass_times: cudaSetDevice");
  CK(cudaEventSynchronize(r->ev[5]), "gi_rc_pass_times: sync");
  ms[0] = 0.0f;
  if (r->timed_vox) CK(cudaEventElapsedTime(&ms[0], r->ev[0], r->ev[1]), "gi_rc_pass_times: vox");
  for (int i = 0; i < 4; i++) CK(cudaEventElapsedTime(&ms[i + 1], r->ev[i + 1], r->ev[i + 2]), "gi_rc_pass_times: pass");
  return GI_OK;
}

int gi_rc_read_irradiance(gi_rc *r, float *rgba, void *stream) {
  if (!r || !rgba) return fail(GI_ERR_INVALID, "gi_rc_read_irradiance: NULL argument");
  CK(cudaSetDevice(r->ctx->device), "gi_rc_read_irradiance: cudaSetDevice");
  size_t npx = (size_t)r->W * r->H;
  CK(gi_launch_irr_to_f32(r->dev, r->stage, S(stream)), "gi_rc_read_irradiance: convert");
  CK(cudaMemcpyAsync(rgba, r->stage, npx * 16u, cudaMemcpyDeviceToHost, S(stream)), "gi_rc_read_irradiance: copy");
  CK(cudaStreamSynchronize(S(stream)), "gi_rc_read_irradiance: sync");
  return GI_OK;
}

int gi_rc_read_irradiance_raw(gi_rc *r, void *out, size_t bytes, void *stream) {
  if (!r || !out) return fail(GI_ERR_INVALID, "gi_rc_read_irradiance_raw: NULL argument");
  size_t need = (size_t)r->W * r->H * r->irr_elem_bytes;
  if (bytes < need) return fail(GI_ERR_INVALID, "gi_rc_read_irradiance_raw: %zu bytes, need %zu", bytes, need);
  CK(cudaSetDevice(r->ctx->device), "gi_rc_read_irradiance_raw: cudaSetDevice");
  CK(cudaMemcpyAsync(out, r->dev.irr, need, cudaMemcpyDeviceToHost, S(stream)), "gi_rc_read_irradiance_raw: copy");
  CK(cudaStreamSynchronize(S(stream)), "gi_rc_read_irradiance_raw: sync");
  return GI_OK;
}

int gi_rc_read_irradiance_async(gi_rc *r, void *out, size_t bytes, void *stream) {
  if (!r || !out) return fail(GI_ERR_INVALID, "gi_rc_read_irradiance_async: NULL argument");
  size_t need = (size_t)r->W * r->H * r->irr_elem_bytes;
  if (bytes < need) return fail(GI_ERR_INVALID, "gi_rc_read_irradiance_async: %zu bytes, need %zu", bytes, need);
  CK(cudaSetDevice(r->ctx->device), "gi_rc_read_irradiance_async: cudaSetDevice");
  CK(cudaMemcpyAsync(out, r->dev.irr, need, cudaMemcpyDefault, S(stream)), "gi_rc_read_irradiance_async: copy");
  return GI_OK;
}

int gi_rc_read_counts(gi_rc *r, uint32_t counts[80], void *stream) {
  if (!r || !counts) return fail(GI_ERR_INVALID, "gi_rc_read_counts: NULL argument");
  CK(cudaSetDevice(r->ctx->device), "gi_rc_read_counts: cudaSetDevice");
  CK(cudaMemcpyAsync(counts, r->dev.counts, 80 * 4, cudaMemcpyDeviceToHost, S(stream)), "gi_rc_read_counts: copy");
  uint32_t gave_up = 0;
  if (r->world) CK(cudaMemcpyAsync(&gave_up, r->w.state + 7, 4, cudaMemcpyDeviceToHost, S(stream)), "gi_rc_read_counts: copy");
  CK(cudaStreamSynchronize(S(stream)), "gi_rc_read_counts: sync");
  if (gave_up)
    return fail(GI_ERR_TIMEOUT, "gi_rc_read_counts: a bounded wait of the world probes' compaction gave up; this solve's "
                "probes are not valid");
  return GI_OK;
}

int gi_rc_set_stats(gi_rc *r, uint32_t level) {
  if (!r) return fail(GI_ERR_INVALID, "gi_rc_set_stats: NULL rc");
  if (level > 1) return fail(GI_ERR_INVALID, "gi_rc_set_stats: level %u (0 off, 1 DDA steps; the triangle comparison is not built)", level);
  r->p.stats = level;
  r->dev.stats = level;
  return GI_OK;
}

// The walk-length order's buffers (trace_order 2): a key per ray (zero: the first solve's order is the keys' initial
// one), the order (the identity until the first scatter), the key counts and cursors
static cudaError_t alloc_walk_order(gi_rc *r) {
  const size_t n = r->dev.rays_total;
  uint8_t *steps = nullptr;
  uint32_t *perm = nullptr, *hist = nullptr;
  cudaError_t e;
  if ((e = cudaMalloc(&steps, n ? n : 1u)) || (e = cudaMemset(steps, 0, n ? n : 1u)) ||
      (e = cudaMalloc(&perm, (n ? n : 1u) * 4u)) || (e = cudaMalloc(&hist, 256u * 4u)) ||
      (e = cudaMemset(hist, 0, 256u * 4u)) || (e = gi_launch_iota(perm, (uint32_t)n, nullptr)) ||
      (e = cudaDeviceSynchronize())) {
    cudaFree(steps); cudaFree(perm); cudaFree(hist);
    return e;
  }
  r->dev.rsteps = steps; r->dev.rperm = perm; r->dev.rhist = hist;
  return cudaSuccess;
}

int gi_rc_set_tuning(gi_rc *r, const gi_rc_tuning *t) {
  if (!r || !t) return fail(GI_ERR_INVALID, "gi_rc_set_tuning: NULL argument");
  if (t->trace_order > 2) return fail(GI_ERR_INVALID, "gi_rc_set_tuning: trace_order %u", t->trace_order);
  if (t->trace_order == 2 && r->world)
    return fail(GI_ERR_INVALID, "gi_rc_set_tuning: trace_order 2 (walk-length order) is for screen probes");
  if (t->trace_rays != 1 && t->trace_rays != 2 && t->trace_rays != 4)
    return fail(GI_ERR_INVALID, "gi_rc_set_tuning: trace_rays %u (1, 2 or 4)", t->trace_rays);
  if (t->trace_blocks < 1 || t->trace_blocks > 16) return fail(GI_ERR_INVALID, "gi_rc_set_tuning: trace_blocks %u", t->trace_blocks);
  if (t->gather_shape > 3) return fail(GI_ERR_INVALID, "gi_rc_set_tuning: gather_shape %u", t->gather_shape);
  if (t->merge_threads != 64 && t->merge_threads != 128 && t->merge_threads != 256 && t->merge_threads != 512)
    return fail(GI_ERR_INVALID, "gi_rc_set_tuning: merge_threads %u", t->merge_threads);
  if (t->trace_order == 2 && !r->dev.rperm) {   // the walk-length order's buffers, on first use
    CK(cudaSetDevice(r->ctx->device), "gi_rc_set_tuning: cudaSetDevice");
    CK(alloc_walk_order(r), "gi_rc_set_tuning: walk-length order buffers");
    r->bytes += 5u * (uint64_t)r->dev.rays_total + 1024u;
    r->gen++;   // graphs captured before launch the other trace
  }
  if ((t->trace_order == 2) != (r->dev.trace_order == 2)) r->gen++;
  r->dev.trace_order = t->trace_order;
  r->dev.trace_rays = t->trace_rays;
  r->launch.trace_blocks = t->trace_blocks;
  r->launch.gather_shape = t->gather_shape;
  r->launch.merge_threads = t->merge_threads;
  return GI_OK;
}

int gi_rc_get_tuning(gi_rc *r, gi_rc_tuning *t) {
  if (!r || !t) return fail(GI_ERR_INVALID, "gi_rc_get_tuning: NULL argument");
  *t = gi_rc_tuning{};
  t->trace_order = r->dev.trace_order; t->trace_rays = r->dev.trace_rays; t->trace_blocks = r->launch.trace_blocks;
  t->gather_shape = r->launch.gather_shape; t->merge_threads = r->launch.merge_threads;
  return GI_OK;
}

int gi_vox_set_tuning(gi_vox *v, const gi_vox_tuning *t) {
  if (!v || !t) return fail(GI_ERR_INVALID, "gi_vox_set_tuning: NULL argument");
  uint32_t c = t->chunk_cells, lg = 0;
  while ((1u << lg) < c && lg < 31) lg++;
  if (c < 32 || c > 1024 || (1u << lg) != c)
    return fail(GI_ERR_INVALID, "gi_vox_set_tuning: chunk_cells %u (a power of two, 32..1024)", c);
  if (t->blocks < 1 || t->blocks > 16) return fail(GI_ERR_INVALID, "gi_vox_set_tuning: blocks %u", t->blocks);
  v->dev.chunk_log2 = lg;
  v->dev.blocks = t->blocks;
  return GI_OK;
}

int gi_vox_get_tuning(gi_vox *v, gi_vox_tuning *t) {
  if (!v || !t) return fail(GI_ERR_INVALID, "gi_vox_get_tuning: NULL argument");
  *t = gi_vox_tuning{};
  t->chunk_cells = 1u << v->dev.chunk_log2;
  t->blocks = v->dev.blocks;
  return GI_OK;
}

int gi_rc_bytes(gi_rc *r, uint64_t *bytes) {
  if (!r || !bytes) return fail(GI_ERR_INVALID, "gi_rc_bytes: NULL argument");
  *bytes = r->bytes;
  return GI_OK;
}

int gi_rc_set_debug_hits(gi_rc *r, int on) {
  if (!r) return fail(GI_ERR_INVALID, "gi_rc_set_debug_hits: NULL rc");
  CK(cudaSetDevice(r->ctx->device), "gi_rc_set_debug_hits: cudaSetDevice");
  if (on && !r->hits) {
    cudaError_t e;
    if ((e = dalloc(&r->hits, r->dev.rays_total)) || (e = cudaMalloc(&r->rad_traced, (size_t)r->dev.rays_total * r->rad_elem_bytes)))
      return cuda_fail(e, "gi_rc_set_debug_hits");
  }
  r->debug_hits = on != 0;
  return GI_OK;
}

int gi_rc_buffer_bytes(gi_rc *r, int what, size_t *bytes) {
  if (!r || !bytes) return fail(GI_ERR_INVALID, "gi_rc_buffer_bytes: NULL argument");
  size_t npx = (size_t)r->W * r->H;
  switch (what) {
    case GI_RC_PROBES: *bytes = (size_t)r->dev.probes_total * 48u; break;
    case GI_RC_RAD: case GI_RC_RAD_TRACED: *bytes = (size_t)r->dev.rays_total * r->rad_elem_bytes; break;
    case GI_RC_SH: *bytes = r->sh_elems * r->sh_elem_bytes; break;
    case GI_RC_DEPTH: *bytes = npx * 4u; break;
    case GI_RC_NORMAL: *bytes = npx * 8u; break;
    case GI_RC_TAG: *bytes = npx; break;
    case GI_RC_HITS: *bytes = (size_t)r->dev.rays_total * 16u; break;
    case GI_RC_SHADOW: *bytes = (size_t)r->shadow_size * r->shadow_size * 4u * r->shadow_layers; break;
    case GI_RC_BOUNCE_VOL: *bytes = r->bounce ? 2u * (size_t)r->bn.dx * r->bn.dy * (6u * r->bn.dz + 1u) * 8u : 0u; break;
    case GI_RC_BOUNCE_INJ: *bytes = r->bounce ? (size_t)r->bn_vox->p.max_voxels * 16u : 0u; break;
    case GI_RC_BOUNCE_LIST: *bytes = r->bounce ? (4u + (size_t)r->bn.n) * 4u : 0u; break;
    case GI_RC_WORLD_KEYS: case GI_RC_WORLD_SLOTS: *bytes = r->world ? (size_t)r->w.hash_total * 4u : 0u; break;
    case GI_RC_WORLD_PARENTS: *bytes = r->world ? (size_t)r->dev.probes_total * 32u : 0u; break;
    case GI_RC_WORLD_STATE: *bytes = r->world ? 64u * 4u : 0u; break;
    default: return fail(GI_ERR_INVALID, "gi_rc_buffer_bytes: unknown buffer %d", what);
  }
  return GI_OK;
}

int gi_rc_read_buffer(gi_rc *r, int what, void *out, size_t bytes, void *stream) {
  if (!r || !out) return fail(GI_ERR_INVALID, "gi_rc_read_buffer: NULL argument");
  size_t need = 0;
  int st = gi_rc_buffer_bytes(r, what, &need);
  if (st) return st;
  if (bytes < need) return fail(GI_ERR_INVALID, "gi_rc_read_buffer: %zu bytes, need %zu", bytes, need);
  const void *src = nullptr;
  switch (what) {
    case GI_RC_PROBES: src = r->dev.probes; break;
    case GI_RC_RAD: src = r->dev.rad; break;
    case GI_RC_SH: src = r->dev.sh; break;
    case GI_RC_DEPTH: src = r->depth; break;
    case GI_RC_NORMAL: src = r->normal; break;
    case GI_RC_TAG: src = r->tag; break;
    case GI_RC_HITS: src = r->hits; break;
    case GI_RC_RAD_TRACED: src = r->rad_traced; break;
    case GI_RC_SHADOW: src = r->shadow; break;
    case GI_RC_BOUNCE_INJ: src = r->bn.inj; break;
    case GI_RC_BOUNCE_LIST: src = r->bn.list; break;
    case GI_RC_WORLD_KEYS: src = r->w.keys; break;
    case GI_RC_WORLD_SLOTS: src = r->w.slot_probe; break;
    case GI_RC_WORLD_PARENTS: src = r->w.parents; break;
    case GI_RC_WORLD_STATE: src = r->w.state; break;
    case GI_RC_BOUNCE_VOL:
      if (r->bounce) {   // two allocations: copy them one after the other
        size_t half = need / 2u;
        CK(cudaSetDevice(r->ctx->device), "gi_rc_read_buffer: cudaSetDevice");
        CK(cudaMemcpyAsync(out, r->bn.vol[0], half, cudaMemcpyDeviceToHost, S(stream)), "gi_rc_read_buffer: copy");
        CK(cudaMemcpyAsync((char *)out + half, r->bn.vol[1], half, cudaMemcpyDeviceToHost, S(stream)), "gi_rc_read_buffer: copy");
        CK(cudaStreamSynchronize(S(stream)), "gi_rc_read_buffer: sync");
        return GI_OK;
      }
      break;
  }
  if (!src) return fail(GI_ERR_STATE, "gi_rc_read_buffer: buffer %d not kept (debug hits off, or no shadow map)", what);
  CK(cudaSetDevice(r->ctx->device), "gi_rc_read_buffer: cudaSetDevice");
  CK(cudaMemcpyAsync(out, src, need, cudaMemcpyDeviceToHost, S(stream)), "gi_rc_read_buffer: copy");
  CK(cudaStreamSynchronize(S(stream)), "gi_rc_read_buffer: sync");
  return GI_OK;
}

int gi_rc_merge_gather_f64(gi_rc *r, void *stream) { return gi_rc_merge_gather_f64_rounded(r, 0u, stream); }

int gi_rc_merge_gather_f64_rounded(gi_rc *r, uint32_t f16_cascades, void *stream) {
  if (!r) return fail(GI_ERR_INVALID, "gi_rc_merge_gather_f64: NULL rc");
  if (r->world) return fail(GI_ERR_STATE, "gi_rc_merge_gather_f64: screen probes only");
  if (r->p.atlas != GI_ATLAS_F32) return fail(GI_ERR_STATE, "gi_rc_merge_gather_f64: needs an F32 atlas");
  if (!r->debug_hits || !r->rad_traced)
    return fail(GI_ERR_STATE, "gi_rc_merge_gather_f64: the traced intervals are not kept (gi_rc_set_debug_hits)");
  CK(cudaSetDevice(r->ctx->device), "gi_rc_merge_gather_f64: cudaSetDevice");
  size_t npx = (size_t)r->W * r->H, np0 = (size_t)r->dev.c[0].tiles_x * r->dev.c[0].tiles_y;
  if (!r->rad64) {
    cudaError_t e;
    if ((e = cudaMalloc(&r->rad64, (size_t)r->dev.rays_total * 32u)) || (e = cudaMalloc(&r->sh64, np0 * 27u * 8u)) ||
        (e = cudaMalloc(&r->irr64, npx * 32u))) {
      cudaFree(r->rad64); cudaFree(r->sh64); cudaFree(r->irr64);
      r->rad64 = r->irr64 = nullptr; r->sh64 = nullptr;
      return cuda_fail(e, "gi_rc_merge_gather_f64: allocate");
    }
  }
  CK(gi_launch_merge_gather_f64(r->dev, reinterpret_cast<const float4 *>(r->rad_traced), r->rad64, r->sh64, r->irr64,
                                f16_cascades, S(stream)), "gi_rc_merge_gather_f64: launch");
  r->have64 = true;
  return GI_OK;
}

int gi_rc_read_irradiance_f64(gi_rc *r, double *rgba, void *stream) {
  if (!r || !rgba) return fail(GI_ERR_INVALID, "gi_rc_read_irradiance_f64: NULL argument");
  if (!r->have64) return fail(GI_ERR_STATE, "gi_rc_read_irradiance_f64: no gi_rc_merge_gather_f64 ran");
  CK(cudaSetDevice(r->ctx->device), "gi_rc_read_irradiance_f64: cudaSetDevice");
  CK(cudaMemcpyAsync(rgba, r->irr64, (size_t)r->W * r->H * 32u, cudaMemcpyDefault, S(stream)),
     "gi_rc_read_irradiance_f64: copy");
  CK(cudaStreamSynchronize(S(stream)), "gi_rc_read_irradiance_f64: sync");
  return GI_OK;
}

// ---- the dynamic layer (dynlayer.ts) ----------------------------------------------------------------------------------
int gi_dyn_create(gi_vox *v, uint32_t bricks, uint32_t first_dynamic, uint32_t albedo, gi_dyn **out) {
  if (!v || !out) return fail(GI_ERR_INVALID, "gi_dyn_create: NULL argument");
  *out = nullptr;
  const uint32_t G = v->p.G, G3 = G * G * G, levels = v->p.levels;
  if (G3 % 32u) return fail(GI_ERR_INVALID, "gi_dyn_create: G^3 must be a multiple of 32 (dynlayer.ts:687)");
  if (bricks < 1 || bricks > (1u << 20)) return fail(GI_ERR_INVALID, "gi_dyn_create: %u bricks (1 .. 2^20)", bricks);
  if (first_dynamic > v->scene->ntris)
    return fail(GI_ERR_INVALID, "gi_dyn_create: first dynamic row %u of %u", first_dynamic, v->scene->ntris);
  CK(cudaSetDevice(v->scene->ctx->device), "gi_dyn_create: cudaSetDevice");
  gi_dyn *d = new (std::nothrow) gi_dyn;
  if (!d) return fail(GI_ERR_OOM, "gi_dyn_create: host allocation");
  d->vox = v;
  DynDev &q = d->dev;
  memset(&q, 0, sizeof q);
  q.nb = bricks; q.albedo = albedo ? 1u : 0u; q.first = first_dynamic; q.end = v->scene->ntris;
  const size_t np = (size_t)levels * G3, nw = np / 32u;
  q.look_cap = (uint32_t)((nw + 255u) / 256u);
  cudaError_t e;
  if ((e = dalloc(&q.hdr, 64)) || (e = dalloc(&q.ptr, np)) || (e = dalloc(&q.bits, 2u * nw)) || (e = dalloc(&q.meta, bricks)) ||
      (e = dalloc(&q.mask, (size_t)bricks * 16u)) || (e = dalloc(&q.data, (size_t)bricks * 512u * DYN_W)) ||
      (e = dalloc(&q.look, (size_t)q.look_cap + 1u))) {
    cudaFree(q.hdr); cudaFree(q.ptr); cudaFree(q.bits); cudaFree(q.meta); cudaFree(q.mask); cudaFree(q.data); cudaFree(q.look);
    delete d;
    return cuda_fail(e, "gi_dyn_create");
  }
  // createDynLayer's initial state (dynlayer.ts:690-694): empty pointers, bounds reset, zero bitsets
  uint32_t h[64] = {};
  h[32] = h[33] = h[34] = 0xffffffffu;
  if ((e = cudaMemcpy(q.hdr, h, sizeof h, cudaMemcpyHostToDevice)) || (e = cudaMemset(q.ptr, 0xff, np * 4u)) ||
      (e = cudaMemset(q.bits, 0, 2u * nw * 4u)) || (e = cudaMemset(q.meta, 0, (size_t)bricks * 4u)) ||
      (e = cudaMemset(q.mask, 0, (size_t)bricks * 64u)) || (e = cudaMemset(q.data, 0, (size_t)bricks * 512u * DYN_W * 4u))) {
    cudaFree(q.hdr); cudaFree(q.ptr); cudaFree(q.bits); cudaFree(q.meta); cudaFree(q.mask); cudaFree(q.data); cudaFree(q.look);
    delete d;
    return cuda_fail(e, "gi_dyn_create: init");
  }
  d->bytes = (64u + np + 2u * nw + (uint64_t)bricks * (1u + 16u + 512u * DYN_W) + q.look_cap + 1u) * 4u;
  *out = d;
  return GI_OK;
}

int gi_dyn_build(gi_dyn *d, gi_rc *r, void *stream) {
  if (!d || !r) return fail(GI_ERR_INVALID, "gi_dyn_build: NULL argument");
  if (!r->frame_set) return fail(GI_ERR_STATE, "gi_dyn_build: the rc has no frame");
  if (!d->vox->updated) return fail(GI_ERR_STATE, "gi_dyn_build: gi_vox_update was not called");
  if (r->shadow && r->frame_layers > r->shadow_layers)
    return fail(GI_ERR_STATE, "gi_dyn_build: the frame asks for more shadow-map layers than the map was drawn with");
  CK(cudaSetDevice(d->vox->scene->ctx->device), "gi_dyn_build: cudaSetDevice");
  CK(gi_launch_dyn_build(d->dev, d->vox->dev, d->vox->scene->dev(), r->frame, r->shadow,
                         r->shadow ? r->shadow_size : 0u, r->shadow_layers,
                         d->vox->scene->ctx->sm_count, S(stream)), "gi_dyn_build: launch");
  return GI_OK;
}

int gi_dyn_read_counters(gi_dyn *d, uint32_t hdr[64], void *stream) {
  if (!d || !hdr) return fail(GI_ERR_INVALID, "gi_dyn_read_counters: NULL argument");
  CK(cudaSetDevice(d->vox->scene->ctx->device), "gi_dyn_read_counters: cudaSetDevice");
  CK(cudaMemcpyAsync(hdr, d->dev.hdr, 64 * 4, cudaMemcpyDeviceToHost, S(stream)), "gi_dyn_read_counters: copy");
  CK(cudaStreamSynchronize(S(stream)), "gi_dyn_read_counters: sync");
  if (hdr[12] != 0u)
    return fail(GI_ERR_TIMEOUT, "gi_dyn_read_counters: a bounded wait of the allocation scan gave up (header word 12)");
  return GI_OK;
}

int gi_dyn_read_state(gi_dyn *d, uint32_t *ptr, uint32_t *bits, uint32_t *meta, uint32_t *mask, uint32_t *data, void *stream) {
  if (!d) return fail(GI_ERR_INVALID, "gi_dyn_read_state: NULL dynamic layer");
  CK(cudaSetDevice(d->vox->scene->ctx->device), "gi_dyn_read_state: cudaSetDevice");
  const DynDev &q = d->dev;
  const size_t np = (size_t)d->vox->p.levels * d->vox->p.G * d->vox->p.G * d->vox->p.G;
  struct { void *dst; const void *src; size_t bytes; } c[5] = {
      {ptr, q.ptr, np * 4u}, {bits, q.bits, np / 32u * 2u * 4u}, {meta, q.meta, (size_t)q.nb * 4u},
      {mask, q.mask, (size_t)q.nb * 64u}, {data, q.data, (size_t)q.nb * 512u * DYN_W * 4u}};
  for (auto &x : c)
    if (x.dst) CK(cudaMemcpyAsync(x.dst, x.src, x.bytes, cudaMemcpyDeviceToHost, S(stream)), "gi_dyn_read_state: copy");
  CK(cudaStreamSynchronize(S(stream)), "gi_dyn_read_state: sync");
  return GI_OK;
}

int gi_dyn_bytes(gi_dyn *d, uint64_t *bytes) {
  if (!d || !bytes) return fail(GI_ERR_INVALID, "gi_dyn_bytes: NULL argument");
  *bytes = d->bytes;
  return GI_OK;
}

int gi_dyn_destroy(gi_dyn *d) {
  if (!d) return GI_OK;
  cudaSetDevice(d->vox->scene->ctx->device);
  const DynDev &q = d->dev;
  cudaFree(q.hdr); cudaFree(q.ptr); cudaFree(q.bits); cudaFree(q.meta); cudaFree(q.mask); cudaFree(q.data); cudaFree(q.look);
  delete d;
  return GI_OK;
}

int gi_rc_set_dyn(gi_rc *r, gi_dyn *d) {
  if (!r) return fail(GI_ERR_INVALID, "gi_rc_set_dyn: NULL rc");
  if (d && d->vox->scene->ctx->device != r->ctx->device) return fail(GI_ERR_INVALID, "gi_rc_set_dyn: layer on another device");
  r->dyn = d;
  r->gen++;
  r->dev.dyn_hdr = d ? d->dev.hdr : nullptr;
  r->dev.dyn_ptr = d ? d->dev.ptr : nullptr;
  r->dev.dyn_data = d ? d->dev.data : nullptr;
  r->dev.dyn_meta = d ? d->dev.meta : nullptr;
  r->dev.dyn_nb = d ? d->dev.nb : 0u;
  if (r->graph) { cudaGraphExecDestroy(r->graph); r->graph = nullptr; r->graph_vox = nullptr; }   // captured without it
  return GI_OK;
}

int gi_rc_set_objects(gi_rc *r, int on) {
  if (!r) return fail(GI_ERR_INVALID, "gi_rc_set_objects: NULL rc");
  r->dev.objects = on ? 1u : 0u;
  r->gen++;
  return GI_OK;
}

int gi_rc_destroy(gi_rc *r) {
  if (!r) return GI_OK;
  cudaSetDevice(r->ctx->device);
  free_rc(r);
  delete r;
  return GI_OK;
}

}  // extern "C"
