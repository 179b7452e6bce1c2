// Device-side types and helpers of the GI path.  Compiled with -fmad=false: every f32 operation rounds separately,
// in the order the reference's WGSL writes it (left to right), so the integer/index results (voxel bits, DDA hit
// cells) are reproducible bit for bit on any IEEE f32 machine.
#pragma once
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include "../../include/gi.h"

#define GI_EMPTY 0xffffffffu
#define GI_DROP 0xfffffffeu
#define GI_MARK 0xfffffffdu
#define GI_HDR 64
#define GI_BIG_SMALL 8u          // triangles covering more than 8 cells go to the big lists (voxel.ts:223)
#define GI_PI 3.14159265f

namespace gi {

struct f3 { float x, y, z; };
struct i3 { int x, y, z; };

__host__ __device__ __forceinline__ f3 mk(float x, float y, float z) { f3 r; r.x = x; r.y = y; r.z = z; return r; }
__host__ __device__ __forceinline__ i3 mki(int x, int y, int z) { i3 r; r.x = x; r.y = y; r.z = z; return r; }
__device__ __forceinline__ f3 operator+(f3 a, f3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ f3 operator-(f3 a, f3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ f3 operator*(f3 a, f3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ f3 operator*(f3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ f3 operator/(f3 a, float s) { return mk(a.x / s, a.y / s, a.z / s); }
__device__ __forceinline__ f3 operator-(f3 a) { return mk(-a.x, -a.y, -a.z); }
__device__ __forceinline__ f3 adds(f3 a, float s) { return mk(a.x + s, a.y + s, a.z + s); }
__device__ __forceinline__ float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ f3 cross(f3 a, f3 b) { return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
// min/max as `a < b ? a : b` (the oracle's definition; no NaNs reach them)
__device__ __forceinline__ float mn(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float mx(float a, float b) { return a > b ? a : b; }
__device__ __forceinline__ f3 vmin(f3 a, f3 b) { return mk(mn(a.x, b.x), mn(a.y, b.y), mn(a.z, b.z)); }
__device__ __forceinline__ f3 vmax(f3 a, f3 b) { return mk(mx(a.x, b.x), mx(a.y, b.y), mx(a.z, b.z)); }
__device__ __forceinline__ f3 vabs(f3 a) { return mk(fabsf(a.x), fabsf(a.y), fabsf(a.z)); }
__device__ __forceinline__ f3 vfloor(f3 a) { return mk(floorf(a.x), floorf(a.y), floorf(a.z)); }
__device__ __forceinline__ float length3(f3 a) { return sqrtf(dot(a, a)); }
// normalize(v) = v / sqrt(dot(v, v)), IEEE sqrt and division
__device__ __forceinline__ f3 normalize3(f3 a) { float l = length3(a); return mk(a.x / l, a.y / l, a.z / l); }
__device__ __forceinline__ f3 ld3(float4 v) { return mk(v.x, v.y, v.z); }
// f32 -> i32 truncating and saturating (NaN -> 0), WGSL's conversion
__device__ __forceinline__ int f2i(float f) { return __float2int_rz(f); }
__device__ __forceinline__ i3 vf2i(f3 a) { return mki(f2i(a.x), f2i(a.y), f2i(a.z)); }
// f2i(floorf(x)) in one conversion rounding toward -inf (saturating, NaN -> 0: the same integer for every input)
__device__ __forceinline__ i3 vfloori(f3 a) { return mki(__float2int_rd(a.x), __float2int_rd(a.y), __float2int_rd(a.z)); }
__device__ __forceinline__ f3 vi2f(i3 a) { return mk((float)a.x, (float)a.y, (float)a.z); }
__device__ __forceinline__ int iclamp(int x, int lo, int hi) { return min(max(x, lo), hi); }
__device__ __forceinline__ i3 iclamp3(i3 a, i3 lo, i3 hi) {
  return mki(iclamp(a.x, lo.x, hi.x), iclamp(a.y, lo.y, hi.y), iclamp(a.z, lo.z, hi.z));
}
__device__ __forceinline__ float fclampf(float x, float lo, float hi) { return mn(mx(x, lo), hi); }
// exp2 of an integral value is exact; libdevice exp2f otherwise (only non-integral level_map overrides reach it)
__device__ __forceinline__ float exp2_(float x) {
  if (x == floorf(x) && fabsf(x) < 126.0f) return ldexpf(1.0f, (int)x);
  return exp2f(x);
}
// round(log2(x)) exactly: x = m 2^e, m in [0.5, 1): log2 m >= -1/2 <=> m^2 >= 1/2 (exact in double)
__device__ __forceinline__ int round_log2(float x) {
  if (!(x > 0.0f)) return -2147483647 - 1;
  if (isinf(x)) return 2147483647;
  int e;
  float m = frexpf(x, &e);
  double mm = (double)m * (double)m;
  return mm >= 0.5 ? e : e - 1;
}

// log2(x) for x > 0 (the reference's WGSL log2 is implementation-defined; this library defines it): x = m 2^e with m in
// [sqrt(1/2), sqrt(2)), log2 m = 2 atanh(s) / ln 2 with s = (m - 1) / (m + 1) by its series through s^11 (|s| <= 0.172)
// in Horner form with fused multiply-adds.  Exact for powers of two, relative error below 1e-7 elsewhere; the oracle
// evaluates the same f32 sequence.
__device__ __forceinline__ float gi_log2(float x) {
  if (!(x > 0.0f)) return x == 0.0f ? __int_as_float(0xff800000) : __int_as_float(0x7fffffff);
  if (isinf(x)) return x;
  int e;
  float m = frexpf(x, &e);
  if (m < 0.70710678f) { m = m * 2.0f; e -= 1; }
  const float s = (m - 1.0f) / (m + 1.0f);
  const float z = s * s;
  float p = 0.09090909f;
  p = __fmaf_rn(p, z, 0.11111111f);
  p = __fmaf_rn(p, z, 0.14285715f);
  p = __fmaf_rn(p, z, 0.2f);
  p = __fmaf_rn(p, z, 0.33333334f);
  p = __fmaf_rn(p, z, 1.0f);
  return (float)e + (s * p) * 2.8853900817779268f;
}

// e^x of the merge and gather weights: Cody & Waite's two-constant reduction x = k ln2 + r (|r| <= ln2/2, the split of
// ln2 keeps k * hi exact), e^r by its degree-7 Taylor polynomial in Horner form with fused multiply-adds,
// e^x = 2^k e^r.  Relative error below 3e-7 on [-80, 88]; below -80 the result is 0.  The oracle evaluates the same f32
// sequence (the same fmaf steps), so the weights agree bit for bit.
__device__ __forceinline__ float gi_exp(float x);

// acc + a * s per component as one fused multiply-add (the weighted sums of the merge, the SH projection and the
// gather; the oracle uses the same fmaf)
__device__ __forceinline__ f3 fma3(f3 a, float s, f3 acc) {
  return mk(__fmaf_rn(a.x, s, acc.x), __fmaf_rn(a.y, s, acc.y), __fmaf_rn(a.z, s, acc.z));
}

__device__ __forceinline__ float gi_exp(float x) {
  if (x != x) return x;
  if (x < -80.0f) return 0.0f;
  if (x > 88.0f) return __int_as_float(0x7f800000);
  float k = rintf(x * 0x1.715476p+0f);
  float r = (x - k * 0x1.62e4p-1f) - k * 0x1.7f7d1cp-20f;
  float p = 0x1.a01a02p-13f;
  p = __fmaf_rn(p, r, 0x1.6c16c2p-10f);
  p = __fmaf_rn(p, r, 0x1.111112p-7f);
  p = __fmaf_rn(p, r, 0x1.555556p-5f);
  p = __fmaf_rn(p, r, 0x1.555556p-3f);
  p = __fmaf_rn(p, r, 0.5f);
  p = __fmaf_rn(p, r, 1.0f);
  p = __fmaf_rn(p, r, 1.0f);
  // 2^k as a float: k is in [-116, 127] here and p in (0.7, 1.42), so the product is normal and exact (= ldexpf)
  return p * __int_as_float((int)(k + 127.0f) << 23);
}

// ---- WGSL packing builtins (public WGSL spec formulas) -------------------------------------------------------------
__device__ __forceinline__ uint32_t pack4x8unorm(float a, float b, float c, float d) {
  float v[4] = {a, b, c, d};
  uint32_t r = 0;
#pragma unroll
  for (int i = 0; i < 4; i++) {
    float cc = mn(mx(v[i], 0.0f), 1.0f);
    uint32_t q = (uint32_t)floorf(0.5f + 255.0f * cc);
    r |= (q & 0xffu) << (8 * i);
  }
  return r;
}
__device__ __forceinline__ uint32_t pack2x16snorm(float a, float b) {
  float ca = mn(mx(a, -1.0f), 1.0f), cb = mn(mx(b, -1.0f), 1.0f);
  int ia = (int)floorf(0.5f + 32767.0f * ca), ib = (int)floorf(0.5f + 32767.0f * cb);
  return ((uint32_t)ia & 0xffffu) | (((uint32_t)ib & 0xffffu) << 16);
}
// unpack2x16snorm of one half: max(k / 32767, -1) for the 16-bit k, the IEEE quotient from its product with
// r = RN(1 / 32767) and one fused correction step (equal to the quotient for all 65536 k, checked exhaustively on the
// CPU against exact arithmetic)
__device__ __forceinline__ float snorm16(uint32_t h) {
  const float k = (float)(int16_t)(h & 0xffffu);
  const float r = 1.0f / 32767.0f;
  const float q = k * r;
  const float e = __fmaf_rn(-q, 32767.0f, k);
  return mx(__fmaf_rn(e, r, q), -1.0f);
}
__device__ __forceinline__ uint16_t f2h(float x) { return __half_as_ushort(__float2half_rn(x)); }
__device__ __forceinline__ float h2f(uint16_t h) { return __half2float(__ushort_as_half(h)); }
__device__ __forceinline__ uint16_t f2bf(float x) { return __bfloat16_as_ushort(__float2bfloat16_rn(x)); }
__device__ __forceinline__ float bf2f(uint16_t h) { return __uint_as_float((uint32_t)h << 16); }

// ---- atlas storage ---------------------------------------------------------------------------------------------------
// F32: float4 per element; F16 / BF16: 4 x 16 bits in a uint2.
template <int A> struct Atlas;
template <> struct Atlas<GI_ATLAS_F32> {
  typedef float4 T;
  __device__ static __forceinline__ float4 load(const T *p, size_t i) { return p[i]; }
  __device__ static __forceinline__ void store(T *p, size_t i, float4 v) { p[i] = v; }
  __device__ static __forceinline__ float round(float x) { return x; }
};
template <> struct Atlas<GI_ATLAS_F16> {
  typedef uint2 T;
  __device__ static __forceinline__ float4 load(const T *p, size_t i) {
    uint2 u = p[i];
    return make_float4(h2f(u.x & 0xffffu), h2f(u.x >> 16), h2f(u.y & 0xffffu), h2f(u.y >> 16));
  }
  __device__ static __forceinline__ void store(T *p, size_t i, float4 v) {
    p[i] = make_uint2((uint32_t)f2h(v.x) | ((uint32_t)f2h(v.y) << 16), (uint32_t)f2h(v.z) | ((uint32_t)f2h(v.w) << 16));
  }
  __device__ static __forceinline__ float round(float x) { return h2f(f2h(x)); }
};
template <> struct Atlas<GI_ATLAS_BF16> {
  typedef uint2 T;
  __device__ static __forceinline__ float4 load(const T *p, size_t i) {
    uint2 u = p[i];
    return make_float4(bf2f(u.x & 0xffffu), bf2f(u.x >> 16), bf2f(u.y & 0xffffu), bf2f(u.y >> 16));
  }
  __device__ static __forceinline__ void store(T *p, size_t i, float4 v) {
    p[i] = make_uint2((uint32_t)f2bf(v.x) | ((uint32_t)f2bf(v.y) << 16), (uint32_t)f2bf(v.z) | ((uint32_t)f2bf(v.w) << 16));
  }
  __device__ static __forceinline__ float round(float x) { return bf2f(f2bf(x)); }
};

// Waits until the grid this one programmatically depends on (gi_launch) has completed and its writes are visible;
// a no-op without such a dependency.
__device__ __forceinline__ void grid_dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// ---- device views ----------------------------------------------------------------------------------------------------
struct SceneDev {
  const float4 *pos;       // xyz, w = 0
  const float4 *nrm;       // xyz, w = 0
  const uint4 *tri;        // i0, i1, i2, material
  const gi_material *mats;
  uint32_t ntris, nverts, nmats, masked;   // masked: some material has the alpha-mask flag
  // World work items of the voxel build (world.ts, voxel.ts:270-288); items NULL: every row once, instance 0.
  // items: (first thread, source, instance, first level), the source an offset into lists or 0x80000000 | first row;
  // a triangle's key is instance * key_stride + row, moved by inst[instance]
  const uint4 *items;
  const uint32_t *lists;
  const float4 *inst;
  uint32_t nitems, threads, key_stride, key_limit;   // threads of the triangle passes; keys below key_limit
  // Base colour textures (gi_scene_set_textures): a uv per vertex; per layer the mip chain of linear float4 texels
  const float2 *uv;          // null: no texture coordinates (every material untextured)
  const float4 *tex;
  uint32_t tex_size, tex_levels, tex_layers, tex_layer_texels;
};

// 1 + layer of a textured material this scene can sample, else 0
__device__ __forceinline__ uint32_t tex_layer_of(const SceneDev &s, const gi_material &m) {
  return (s.uv && s.tex && m.base_color_tex != 0u && m.base_color_tex <= s.tex_layers) ? m.base_color_tex : 0u;
}
// Bilinear sample of layer (1-based) at level lod (clamped to the chain), repeat addressing: texel (i, j) of a level of
// size n has its centre at ((i + 0.5) / n, (j + 0.5) / n); the four texels around (u, v) weighted in f32 as
// (t00 (1 - ax) + t10 ax) (1 - ay) + (t01 (1 - ax) + t11 ax) ay
__device__ __forceinline__ float4 tex_sample(const SceneDev &s, uint32_t layer1, float u, float v, uint32_t lod) {
  const uint32_t L = lod < s.tex_levels ? lod : s.tex_levels - 1u;
  uint32_t off = 0;
  for (uint32_t k = 0; k < L; k++) off += (s.tex_size >> k) * (s.tex_size >> k);
  const uint32_t n = s.tex_size >> L;
  const float4 *t = s.tex + (size_t)(layer1 - 1u) * s.tex_layer_texels + off;
  const float x = u * (float)n - 0.5f, y = v * (float)n - 0.5f;
  const float fx = floorf(x), fy = floorf(y);
  const float ax = x - fx, ay = y - fy;
  const int m = (int)n - 1;
  const int i0 = f2i(fx) & m, i1 = (int)((uint32_t)f2i(fx) + 1u) & m;
  const int j0 = f2i(fy) & m, j1 = (int)((uint32_t)f2i(fy) + 1u) & m;
  const float4 a = __ldg(&t[j0 * (int)n + i0]), b = __ldg(&t[j0 * (int)n + i1]);
  const float4 c = __ldg(&t[j1 * (int)n + i0]), d = __ldg(&t[j1 * (int)n + i1]);
  const float bx = 1.0f - ax, by = 1.0f - ay;
  return make_float4((a.x * bx + b.x * ax) * by + (c.x * bx + d.x * ax) * ay, (a.y * bx + b.y * ax) * by + (c.y * bx + d.y * ax) * ay,
                     (a.z * bx + b.z * ax) * by + (c.z * bx + d.z * ax) * ay, (a.w * bx + b.w * ax) * by + (c.w * bx + d.w * ax) * ay);
}
// The uv at barycentric weights w of the triangle's vertices (UV(a) w.x + UV(b) w.y + UV(c) w.z, voxel.ts:330)
__device__ __forceinline__ float2 tri_uv(const SceneDev &s, uint4 idx, float wx, float wy, float wz) {
  const float2 a = s.uv[idx.x], b = s.uv[idx.y], c = s.uv[idx.z];
  return make_float2((a.x * wx + b.x * wy) + c.x * wz, (a.y * wx + b.y * wy) + c.y * wz);
}
// The rasters' alpha test (gbuffer.ts:94 and the shadow pass's discard): a masked material's alpha at barycentric
// weights (wa, wb, wc) — the texture at level 0 times the factor, or the factor alone untextured — against the cutoff
__device__ __forceinline__ bool raster_alpha_ok(const SceneDev &s, uint4 idx, float wa, float wb, float wc) {
  const gi_material &m = s.mats[idx.w];
  if ((m.flags & 1u) == 0u) return true;
  float a = m.base_color[3];
  const uint32_t layer = tex_layer_of(s, m);
  if (layer) {
    const float2 uv = tri_uv(s, idx, wa, wb, wc);
    a = tex_sample(s, layer, uv.x, uv.y, 0u).w * m.base_color[3];
  }
  return !(a < m.alpha_cutoff);
}

// Drawn triangle t of a raster: row t of the table, or with drawn instances (inst set) row t mod key_stride of
// instance t / key_stride, moved by its offset
__device__ __forceinline__ uint4 drawn_tri(const SceneDev &s, uint32_t t, f3 &off) {
  off = mk(0.0f, 0.0f, 0.0f);
  if (!s.inst) return s.tri[t];
  const uint32_t i = t / s.key_stride;
  const float4 o = s.inst[i];
  off = mk(o.x, o.y, o.z);
  return s.tri[t - i * s.key_stride];
}

// Voxel world in device memory (struct of arrays; the reference packs the same data in one `vox` buffer,
// voxel.ts:753-760).
struct VoxDev {
  float v0;
  uint32_t levels, G, max_bricks, max_voxels, big_cap;
  uint32_t chunk_log2, blocks;   // tuning: cells per big-triangle work item (log2), resident blocks per SM
  uint32_t citem_cap, scan_cap;  // entries of citem (0: no table); blocks the chained scans may take
  float vs[8];         // voxel size per level, ldexpf(v0, L) (vox_derived)
  int32_t lim_vox[8], lim_brick[8];   // voxRange's limit f2i(G * size * 8 / cell), voxel and brick cells (vox_derived)
  int32_t origin[8][4];
  float inv_vs[8];     // RN(1 / vs[L]) (vox_derived)
  float box_lo[8][4], box_hi[8][4];   // per level the clipmap's box: (origin * vs) * 8 and lo + (G * vs) * 8 (vox_bounds)
  uint32_t *hdr;       // GI_HDR counter words
  uint32_t *ptr;       // levels * G^3 brick pointers
  uint32_t *occ;       // max_bricks * 16 occupancy words (64 bytes per brick)
  uint32_t *base;      // max_bricks first attribute
  uint32_t *code;      // max_bricks level << 27 | bx << 18 | by << 9 | bz
  uint32_t *rep;       // max_bricks * 512 representative triangle + 1 (build temporary)
  uint32_t *big;       // 16 * big_cap big-triangle lists (build temporary)
  uint4 *attr;         // max_voxels: albedo, normal, emissive rg, emissive b (one 16-byte load per hit)
  float *plane;        // max_voxels
  float *sunvis;       // max_voxels
  uint32_t *vpre;      // build temporary: max_bricks + 1 exclusive prefix of the bricks' voxel counts
  uint32_t *work;      // build temporary: 4 words, the big-triangle queues, the chunk total, the items listed whole
  uint32_t *cpre;      // build temporary: 8 * big_cap, per voxBits big-list slot its item's first chunk
  uint32_t *citem;     // build temporary (optional): the big-list slot of each chunk, citem_cap entries
  unsigned long long *look;   // build temporary: scan_cap + 1 words, the chained scans' ticket and block states
  // voxSun (voxel.ts:633-671): with a shadow map, resolveAttr also writes each voxel's sun visibility from it and
  // the frame block (lightViewProj, sun direction, shadow bias); without one the visibility is 1
  const float *sun_frame;
  const float *shadow;        // shadow_layers x shadow_size^2 depths
  uint32_t shadow_size;
  uint32_t shadow_layers;     // 1, or 2 (a world's camera-following pair); layer 1 is read only when the frame asks
  uint32_t scan_hold;          // test hook (gi_vox_debug_hold_scan): part + 1 of the brick scan that never publishes; 0 off
};

__device__ __forceinline__ float vox_size(const VoxDev &v, uint32_t L) { return v.vs[L]; }
__device__ __forceinline__ i3 org(const VoxDev &v, uint32_t L) { return mki(v.origin[L][0], v.origin[L][1], v.origin[L][2]); }
__device__ __forceinline__ uint32_t ptr_index(const VoxDev &v, uint32_t L, i3 b) {
  uint32_t G = v.G;
  return L * G * G * G + ((uint32_t)b.z * G + (uint32_t)b.y) * G + (uint32_t)b.x;
}
// regionLo (voxel.ts:289)
__device__ __forceinline__ f3 region_lo(const VoxDev &v, uint32_t L) { return (vi2f(org(v, L)) * vox_size(v, L)) * 8.0f; }

// Akenine-Moller triangle / box overlap (voxel.ts:231-248)
// The nine edge axes (1,0,0) x e, (0,1,0) x e, (0,0,1) x e have one zero component.  The reference's axis test takes
// three-term dot products (p_i = dot(v_i, a), r = dot(h, |a|)); here the zero term is left out: adding the +-0
// product to a nonzero partial sum leaves it unchanged, and where the sum is zero only its sign can differ, which no
// comparison sees; so for finite inputs each test decides exactly as the full form (the same roundings in the same
// order), with a third fewer operations.
__device__ __forceinline__ bool sep(float p0, float p1, float p2, float r) {
  return !(mn(mn(p0, p1), p2) > r || mx(mx(p0, p1), p2) < -r);
}
__device__ __forceinline__ bool axis_x(f3 e, f3 v0, f3 v1, f3 v2, f3 h) {   // a = (0, -e.z, e.y)
  float ay = -e.z, az = e.y;
  return sep(v0.y * ay + v0.z * az, v1.y * ay + v1.z * az, v2.y * ay + v2.z * az, h.y * fabsf(ay) + h.z * fabsf(az));
}
__device__ __forceinline__ bool axis_y(f3 e, f3 v0, f3 v1, f3 v2, f3 h) {   // a = (e.z, 0, -e.x)
  float ax = e.z, az = -e.x;
  return sep(v0.x * ax + v0.z * az, v1.x * ax + v1.z * az, v2.x * ax + v2.z * az, h.x * fabsf(ax) + h.z * fabsf(az));
}
__device__ __forceinline__ bool axis_z(f3 e, f3 v0, f3 v1, f3 v2, f3 h) {   // a = (-e.y, e.x, 0)
  float ax = -e.y, ay = e.x;
  return sep(v0.x * ax + v0.y * ay, v1.x * ax + v1.y * ay, v2.x * ax + v2.y * ay, h.x * fabsf(ax) + h.y * fabsf(ay));
}
__device__ __forceinline__ bool tri_box(f3 c, f3 h, f3 a, f3 b, f3 cc) {
  f3 v0 = a - c, v1 = b - c, v2 = cc - c;
  f3 lo = vmin(vmin(v0, v1), v2), hi = vmax(vmax(v0, v1), v2);
  if (lo.x > h.x || lo.y > h.y || lo.z > h.z || hi.x < -h.x || hi.y < -h.y || hi.z < -h.z) return false;
  f3 e0 = v1 - v0, e1 = v2 - v1, e2 = v0 - v2;
  f3 n = cross(e0, e1);
  if (fabsf(dot(n, v0)) > dot(h, vabs(n))) return false;
  return axis_x(e0, v0, v1, v2, h) && axis_x(e1, v0, v1, v2, h) && axis_x(e2, v0, v1, v2, h)
      && axis_y(e0, v0, v1, v2, h) && axis_y(e1, v0, v1, v2, h) && axis_y(e2, v0, v1, v2, h)
      && axis_z(e0, v0, v1, v2, h) && axis_z(e1, v0, v1, v2, h) && axis_z(e2, v0, v1, v2, h);
}

// Frame word offsets (frame.ts:4-21).
enum { F_VP = 0, F_IVP = 16, F_EYE = 80, F_FWD = 84, F_SUN = 88, F_SUNE = 92, F_SKY = 96, F_SIZE = 100, F_RC = 104,
       F_RC2 = 108, F_RU = 112, F_RU2 = 116, F_OMEGA = 120, F_STYLE = 136 };

// lightViewProj; lightViewProjFar (the second layer of a world's camera-following pair); shadow layers, layer-0 bias,
// layer-1 bias
enum { F_LVP = 64, F_LVPF = 140, F_SHADOW = 156 };

// x's light clip coordinates under the 16-word matrix m (mat4 * vec4 summed in column order)
__device__ __forceinline__ f3 light_clip(const float *__restrict__ m, f3 x) {
  return mk(m[0] * x.x + m[4] * x.y + m[8] * x.z + m[12] * 1.0f, m[1] * x.x + m[5] * x.y + m[9] * x.z + m[13] * 1.0f,
            m[2] * x.x + m[6] * x.y + m[10] * x.z + m[14] * 1.0f);
}

__device__ __forceinline__ float sun_compare(const float *__restrict__ map, uint32_t S, float u, float v, float ref);

// shadowCoord (frame.ts:35-46) + textureSampleCompareLevel with the 'less-equal' comparison sampler (linear,
// clamp-to-edge within the layer; lighting.ts:162): layer 0 where x projects inside it, else layer 1 (at map + S^2)
// when the frame has two (shadow.x >= 1.5), the four texels around x's map position compared with its biased light
// depth and weighted bilinearly in f32; 1 (lit) outside every layer.
// `layers`: the map's layer count (the host refuses a frame asking for more; a second layer is never read past it).
__device__ __forceinline__ float sun_tap(const float *__restrict__ F, const float *__restrict__ map, uint32_t S,
                                         uint32_t layers, f3 x) {
  const f3 c = light_clip(F + F_LVP, x);
  const float u = c.x * 0.5f + 0.5f, v = c.y * -0.5f + 0.5f;
  if (u >= 0.0f && v >= 0.0f && u <= 1.0f && v <= 1.0f) return sun_compare(map, S, u, v, c.z - F[F_SHADOW + 1]);
  if (F[F_SHADOW] < 1.5f || layers < 2u) return 1.0f;
  const f3 c1 = light_clip(F + F_LVPF, x);
  const float u1 = c1.x * 0.5f + 0.5f, v1 = c1.y * -0.5f + 0.5f;
  if (u1 >= 0.0f && v1 >= 0.0f && u1 <= 1.0f && v1 <= 1.0f)
    return sun_compare(map + (size_t)S * S, S, u1, v1, c1.z - F[F_SHADOW + 2]);
  return 1.0f;
}

__device__ __forceinline__ float sun_compare(const float *__restrict__ map, uint32_t S, float u, float v, float ref) {
  float tx = u * (float)S - 0.5f, ty = v * (float)S - 0.5f;
  float fx = floorf(tx), fy = floorf(ty);
  float ax = tx - fx, ay = ty - fy;
  int i0 = f2i(fx), j0 = f2i(fy), n = (int)S - 1;
  int ia = iclamp(i0, 0, n), ib = iclamp(i0 + 1, 0, n), ja = iclamp(j0, 0, n), jb = iclamp(j0 + 1, 0, n);
  float c00 = ref <= __ldg(&map[(size_t)ja * S + ia]) ? 1.0f : 0.0f, c10 = ref <= __ldg(&map[(size_t)ja * S + ib]) ? 1.0f : 0.0f;
  float c01 = ref <= __ldg(&map[(size_t)jb * S + ia]) ? 1.0f : 0.0f, c11 = ref <= __ldg(&map[(size_t)jb * S + ib]) ? 1.0f : 0.0f;
  return (c00 * (1.0f - ax) + c10 * ax) * (1.0f - ay) + (c01 * (1.0f - ax) + c11 * ax) * ay;
}

// voxSun (voxel.ts:643-671) of one voxel: centre pc, size vs, packed oct normal and plane offset as resolveAttr stored
// them.  The mean of four taps a quarter voxel from the centre's projection on the plane, along two tangents, lifted
// (0.25 voxel + 3 cm) to the sunward side.
__device__ __forceinline__ float voxel_sun(const float *__restrict__ F, const float *__restrict__ map, uint32_t S,
                                           uint32_t layers, f3 pc, float vs, uint32_t npack, float plane) {
  // unpack2x16snorm: k / 32767 as the f64 product rounded to f32 (the f32 quotient for every 16-bit k)
  const double inv32767 = 1.0 / 32767.0;
  float ex = mx(__double2float_rn((double)(int16_t)(npack & 0xffffu) * inv32767), -1.0f);
  float ey = mx(__double2float_rn((double)(int16_t)(npack >> 16) * inv32767), -1.0f);
  f3 n = mk(ex, ey, 1.0f - fabsf(ex) - fabsf(ey));
  float q0 = mx(-n.z, 0.0f);
  n.x += n.x >= 0.0f ? -q0 : q0;
  n.y += n.y >= 0.0f ? -q0 : q0;
  f3 q = pc;
  if (dot(n, n) > 1e-4f) { n = normalize3(n); q = pc + n * plane; }
  else n = mk(0.0f, 1.0f, 0.0f);
  f3 ns = dot(n, mk(F[F_SUN], F[F_SUN + 1], F[F_SUN + 2])) < 0.0f ? -n : n;
  f3 t1 = normalize3(cross(ns, fabsf(ns.y) > 0.9f ? mk(1.0f, 0.0f, 0.0f) : mk(0.0f, 1.0f, 0.0f)));
  f3 t2 = cross(ns, t1);
  float h = 0.25f * vs;
  f3 o = q + ns * (0.25f * vs + 0.03f);
  f3 sp = t1 + t2, sm = t1 - t2;
  return 0.25f * (((sun_tap(F, map, S, layers, o + sp * h) + sun_tap(F, map, S, layers, o + sm * h))
                   + sun_tap(F, map, S, layers, o - sp * h)) + sun_tap(F, map, S, layers, o - sm * h));
}

// worldAt (frame.ts:22-26), mat4 * vec4 summed in column order
__device__ __forceinline__ f3 world_at(const float *__restrict__ F, int px, int py, float d) {
  float nx = ((float)px + 0.5f) * F[F_SIZE + 2] * 2.0f - 1.0f;
  float ny = 1.0f - ((float)py + 0.5f) * F[F_SIZE + 3] * 2.0f;
  const float *m = F + F_IVP;
  float h[4];
#pragma unroll
  for (int i = 0; i < 4; i++) h[i] = m[i] * nx + m[4 + i] * ny + m[8 + i] * d + m[12 + i] * 1.0f;
  return mk(h[0] / h[3], h[1] / h[3], h[2] / h[3]);
}
__device__ __forceinline__ float view_z(const float *__restrict__ F, f3 p) {
  return dot(p - mk(F[F_EYE], F[F_EYE + 1], F[F_EYE + 2]), mk(F[F_FWD], F[F_FWD + 1], F[F_FWD + 2]));
}

// octDecode / dirOf (rc.ts:291-308)
__device__ __forceinline__ f3 dir_of(uint32_t di, uint32_t res) {
  float u = ((float)(di % res) + 0.5f) / (float)res, v = ((float)(di / res) + 0.5f) / (float)res;
  float fx = u * 2.0f - 1.0f, fy = v * 2.0f - 1.0f;
  f3 n = mk(fx, fy, 1.0f - fabsf(fx) - fabsf(fy));
  float t = mx(-n.z, 0.0f);
  n.x += n.x >= 0.0f ? -t : t;
  n.y += n.y >= 0.0f ? -t : t;
  return normalize3(n);
}

// Index of the r-th set bit (from 0) of w, r < popc(w): halves of the word selected by their popcounts, branch-free
// (the same index as clearing the lowest set bit r times)
__device__ __forceinline__ uint32_t nth_set_bit(uint32_t w, uint32_t r) {
  uint32_t pos = 0;
#pragma unroll
  for (uint32_t s = 16; s >= 1; s >>= 1) {
    const uint32_t c = __popc(w & ((1u << s) - 1u));
    const bool up = r >= c;
    r -= up ? c : 0u;
    w >>= up ? s : 0u;
    pos += up ? s : 0u;
  }
  return pos;
}

// Warp-aggregated atomicAdd: one atomic per distinct address among the active lanes would need a match; the lists
// and counters here use one address per call, so the active lanes share it.
__device__ __forceinline__ uint32_t warp_append(uint32_t *counter, bool want) {
  uint32_t active = __activemask();
  uint32_t m = __ballot_sync(active, want);
  if (!want) return 0;
  uint32_t lane = threadIdx.x & 31u;
  uint32_t leader = __ffs(m) - 1u;
  uint32_t rank = __popc(m & ((1u << lane) - 1u));
  uint32_t base = 0;
  if (lane == leader) base = atomicAdd(counter, (uint32_t)__popc(m));
  base = __shfl_sync(m, base, leader);
  return base + rank;
}

}  // namespace gi
