// gi_vox_build_noalloc: the voxel clipmap rebuild for callers that cannot allocate device memory.
//
// Some callers of this library cannot call cudaMalloc: a renderer that carves every buffer out of its own fixed
// device-memory pool, a host thread that is capturing a CUDA graph (allocation is not a stream operation and breaks
// the capture), or a serving loop that must not stall the device mid-request (cudaMalloc/cudaFree synchronise).  They
// own their inputs and outputs already; what the rebuild needs besides them is scratch memory (the per-voxel
// representative table, the big-triangle lists, the scans' sums, the work queues).  Here that scratch is a file-scope static
// device array, so this entry point allocates nothing.
//
// The array lives in every GPU that loads the library until the process exits (14.2 MiB).  All calls share it and it
// keeps the last call's contents: the rebuild clears what must start at zero itself (the lists' counters are header
// words of the caller's output, the representatives of every allocated brick are zeroed by the allocation pass), but
// two calls that overlap on the GPU (different streams, different host threads) race on the array and corrupt each
// other's results; serialise them.
#include <cuda_runtime.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>

#include <mutex>
#include <string>

#include "gi_dev.cuh"
#include "gi_internal.h"

using namespace gi;

namespace {

constexpr uint32_t NOALLOC_MAX_BRICKS = 4096;          // representative table: 4096 x 512 words = 8 MiB
constexpr uint32_t NOALLOC_BIG_CAP = 1u << 16;         // per big-triangle list: 16 x 65536 words = 4 MiB
constexpr uint32_t NOALLOC_SCAN_WORDS = 1u << 14;      // chained-scan blocks: levels * G^3 <= 2^25 pointers
// the chained scans' states (64-bit words) start on an even word
constexpr uint32_t NOALLOC_LOOK_AT = (NOALLOC_MAX_BRICKS * 512u + 16u * NOALLOC_BIG_CAP + NOALLOC_MAX_BRICKS + 1u + 4u +
                                      8u * NOALLOC_BIG_CAP + 1u) & ~1u;
constexpr uint32_t NOALLOC_WORDS = NOALLOC_LOOK_AT + 2u * (NOALLOC_SCAN_WORDS + 1u);

// The scratch.  In host code `g_noalloc_scratch` only names the symbol; its device address comes from
// cudaGetSymbolAddress, once per device (see scratch_address).
__device__ __align__(256) uint32_t g_noalloc_scratch[NOALLOC_WORDS];

constexpr int MAX_DEVICES = 64;
std::mutex g_mu;
uint32_t *g_addr[MAX_DEVICES] = {};
uint32_t g_sms[MAX_DEVICES] = {};

int fail(int code, const char *fmt, ...);

// Device address of the scratch on the current device (set-up on the first call per device, with it current).
int scratch_address(int dev, uint32_t **out, uint32_t *sms) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_addr[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return fail(GI_ERR_CUDA, "gi_vox_build_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
    int n = 0;
    e = cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return fail(GI_ERR_CUDA, "gi_vox_build_noalloc: SM count: %s", cudaGetErrorString(e));
    g_addr[dev] = (uint32_t *)p;
    g_sms[dev] = (uint32_t)n;
  }
  *out = g_addr[dev];
  *sms = g_sms[dev];
  return GI_OK;
}

}  // namespace

// The C-ABI's error reporting lives in capi.cu; this file reports through the same gi_last_error.
void gi_set_error(const char *msg);

namespace {
int fail(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  gi_set_error(buf);
  return code;
}
}  // namespace

extern "C" int gi_vox_build_noalloc(const gi_vox_params *p, const double eye[3], const float *pos4, const float *nrm4,
                                    uint32_t nverts, const uint32_t *tri4, uint32_t ntris, const gi_material *mats,
                                    uint32_t nmats, uint32_t *hdr, uint32_t *ptr, uint32_t *occ, uint32_t *base,
                                    uint32_t *code, uint32_t *attr, float *plane, float *sunvis, void *stream) {
  if (!p || !eye) return fail(GI_ERR_INVALID, "gi_vox_build_noalloc: NULL params or eye");
  if (!hdr || !ptr || !occ || !base || !code || !attr || !plane || !sunvis)
    return fail(GI_ERR_INVALID, "gi_vox_build_noalloc: NULL output buffer");
  if (ntris && (!pos4 || !nrm4 || !tri4 || !mats || !nmats)) return fail(GI_ERR_INVALID, "gi_vox_build_noalloc: NULL input");
  if (p->levels < 1 || p->levels > 8) return fail(GI_ERR_INVALID, "gi_vox_build_noalloc: levels %u (1..8)", p->levels);
  if (p->G < 4 || p->G > 256 || p->G % 4) return fail(GI_ERR_INVALID, "gi_vox_build_noalloc: G %u (a multiple of 4, 4..256)", p->G);
  if (!(p->v0 > 0.0)) return fail(GI_ERR_INVALID, "gi_vox_build_noalloc: v0 must be > 0");
  if (p->max_bricks < 1 || p->max_bricks > NOALLOC_MAX_BRICKS)
    return fail(GI_ERR_INVALID, "gi_vox_build_noalloc: max_bricks %u exceeds the static scratch (at most %u bricks)",
                p->max_bricks, NOALLOC_MAX_BRICKS);
  uint64_t nptr = (uint64_t)p->levels * p->G * p->G * p->G;
  if ((nptr + 2047u) / 2048u > NOALLOC_SCAN_WORDS)
    return fail(GI_ERR_INVALID, "gi_vox_build_noalloc: levels * G^3 = %llu pointers exceeds the static scratch (at most %u)",
                (unsigned long long)nptr, NOALLOC_SCAN_WORDS * 2048u);
  if (p->max_voxels < 1 || p->max_voxels >= (1u << 31)) return fail(GI_ERR_INVALID, "gi_vox_build_noalloc: max_voxels %u", p->max_voxels);
  for (int a = 0; a < 3; a++)
    if (!isfinite(eye[a])) return fail(GI_ERR_INVALID, "gi_vox_build_noalloc: eye is not finite");
  if ((((uintptr_t)pos4) | ((uintptr_t)nrm4) | ((uintptr_t)tri4) | ((uintptr_t)occ) | ((uintptr_t)attr)) & 15u)
    return fail(GI_ERR_INVALID, "gi_vox_build_noalloc: pos4, nrm4, tri4, occ and attr must be 16-byte aligned");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(GI_ERR_CUDA, "gi_vox_build_noalloc: cudaGetDevice: %s", cudaGetErrorString(e));
  if (dev < 0 || dev >= MAX_DEVICES) return fail(GI_ERR_INVALID, "gi_vox_build_noalloc: device %d", dev);
  uint32_t *scratch = nullptr, sms = 0;
  int st = scratch_address(dev, &scratch, &sms);
  if (st != GI_OK) return st;

  VoxDev v;
  memset(&v, 0, sizeof v);
  v.v0 = (float)p->v0;
  v.levels = p->levels; v.G = p->G; v.max_bricks = p->max_bricks; v.max_voxels = p->max_voxels;
  v.big_cap = NOALLOC_BIG_CAP;
  v.chunk_log2 = 7;   // the default gi_vox_tuning
  v.blocks = 8;
  vox_derived(v);
  v.scan_cap = NOALLOC_SCAN_WORDS;
  for (uint32_t L = 0; L < p->levels; L++) {
    double bs = p->v0 * ldexp(1.0, (int)L) * 8.0;   // writeUniform (voxel.ts:873-874)
    for (int a = 0; a < 3; a++) {
      double o = floor(eye[a] / bs) - (double)(p->G / 2);
      if (fabs(o) > (double)(1 << 22)) return fail(GI_ERR_INVALID, "gi_vox_build_noalloc: eye too far from the origin");
      v.origin[L][a] = (int32_t)o;
    }
  }
  vox_bounds(v);
  v.hdr = hdr; v.ptr = ptr; v.occ = occ; v.base = base; v.code = code;
  v.attr = reinterpret_cast<uint4 *>(attr); v.plane = plane; v.sunvis = sunvis;
  v.rep = scratch;
  v.big = scratch + NOALLOC_MAX_BRICKS * 512u;
  v.vpre = v.big + 16u * NOALLOC_BIG_CAP;
  v.work = v.vpre + NOALLOC_MAX_BRICKS + 1u;
  v.cpre = v.work + 4u;
  v.look = reinterpret_cast<unsigned long long *>(scratch + NOALLOC_LOOK_AT);

  SceneDev s;
  s.pos = reinterpret_cast<const float4 *>(pos4); s.nrm = reinterpret_cast<const float4 *>(nrm4);
  s.tri = reinterpret_cast<const uint4 *>(tri4); s.mats = mats;
  s.ntris = ntris; s.nverts = nverts; s.nmats = nmats; s.masked = 0;
  s.items = nullptr; s.lists = nullptr; s.inst = nullptr;
  s.nitems = 0; s.threads = ntris; s.key_stride = ntris; s.key_limit = ntris;
  s.uv = nullptr; s.tex = nullptr;   // no textures here: the base colour is the factor
  s.tex_size = s.tex_levels = s.tex_layers = s.tex_layer_texels = 0;
  e = gi_launch_vox_build(v, s, sms, (cudaStream_t)stream);
  if (e != cudaSuccess) return fail(GI_ERR_CUDA, "gi_vox_build_noalloc: launch: %s", cudaGetErrorString(e));
  return GI_OK;
}
