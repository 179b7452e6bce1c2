/* Scalar/vector helpers of the oracle.  Every operation is one IEEE f32 operation in WGSL's evaluation order
 * (left to right, no fused multiply-add: the oracle is built with -ffp-contract=off). */
#ifndef ORC_MATH_H
#define ORC_MATH_H
#include <math.h>
#include <stdint.h>
#include <string.h>

typedef struct { float x, y, z; } v3;
typedef struct { int32_t x, y, z; } i3;

static inline v3 V(float x, float y, float z) { v3 r = {x, y, z}; return r; }
static inline i3 I(int32_t x, int32_t y, int32_t z) { i3 r = {x, y, z}; return r; }
static inline v3 add(v3 a, v3 b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 sub(v3 a, v3 b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 mul(v3 a, v3 b) { return V(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline v3 divv(v3 a, v3 b) { return V(a.x / b.x, a.y / b.y, a.z / b.z); }
static inline v3 muls(v3 a, float s) { return V(a.x * s, a.y * s, a.z * s); }
static inline v3 divs(v3 a, float s) { return V(a.x / s, a.y / s, a.z / s); }
static inline v3 adds(v3 a, float s) { return V(a.x + s, a.y + s, a.z + s); }
/* acc + a * s per component as one fused multiply-add (the definition chosen for the weighted sums of the merge,
 * the SH projection and the gather; the CUDA path uses the same fmaf) */
static inline v3 fmas(v3 a, float s, v3 acc) { return V(fmaf(a.x, s, acc.x), fmaf(a.y, s, acc.y), fmaf(a.z, s, acc.z)); }
static inline v3 neg(v3 a) { return V(-a.x, -a.y, -a.z); }
static inline float dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3 cross(v3 a, v3 b) { return V(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static inline float fminf_(float a, float b) { return a < b ? a : b; }
static inline float fmaxf_(float a, float b) { return a > b ? a : b; }
static inline v3 vmin(v3 a, v3 b) { return V(fminf_(a.x, b.x), fminf_(a.y, b.y), fminf_(a.z, b.z)); }
static inline v3 vmax(v3 a, v3 b) { return V(fmaxf_(a.x, b.x), fmaxf_(a.y, b.y), fmaxf_(a.z, b.z)); }
static inline v3 vabs(v3 a) { return V(fabsf(a.x), fabsf(a.y), fabsf(a.z)); }
static inline v3 vfloor(v3 a) { return V(floorf(a.x), floorf(a.y), floorf(a.z)); }
/* normalize(v) = v / sqrt(dot(v, v)) (IEEE sqrt and division). */
static inline float length3(v3 a) { return sqrtf(dot(a, a)); }
static inline v3 normalize3(v3 a) { float l = length3(a); return V(a.x / l, a.y / l, a.z / l); }
static inline v3 fromf(const float *p) { return V(p[0], p[1], p[2]); }
static inline float comp(v3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }

/* f32 -> i32, truncating, saturating (WGSL's conversion of an out-of-range float). */
static inline int32_t f2i(float f) {
  if (f != f) return 0;
  if (f >= 2147483648.0f) return 2147483647;
  if (f <= -2147483648.0f) return (-2147483647 - 1);
  return (int32_t)f;
}
static inline i3 vf2i(v3 a) { return I(f2i(a.x), f2i(a.y), f2i(a.z)); }
static inline v3 vi2f(i3 a) { return V((float)a.x, (float)a.y, (float)a.z); }
static inline int32_t imin(int32_t a, int32_t b) { return a < b ? a : b; }
static inline int32_t imax(int32_t a, int32_t b) { return a > b ? a : b; }
static inline int32_t iclamp(int32_t x, int32_t lo, int32_t hi) { return imin(imax(x, lo), hi); }
static inline i3 iclamp3(i3 a, i3 lo, i3 hi) { return I(iclamp(a.x, lo.x, hi.x), iclamp(a.y, lo.y, hi.y), iclamp(a.z, lo.z, hi.z)); }
static inline float fclampf(float x, float lo, float hi) { return fminf_(fmaxf_(x, lo), hi); }
static inline float fbits(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }
static inline uint32_t ubits(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }
static inline uint32_t popc(uint32_t x) { return (uint32_t)__builtin_popcount(x); }

/* v0 * 2^L, exact. */
static inline float scale2(float x, int L) { return ldexpf(x, L); }
/* exp2(x): exact for integral x (the only values the configs produce), libm otherwise. */
static inline float exp2_(float x) {
  if (x == floorf(x) && fabsf(x) < 126.0f) return ldexpf(1.0f, (int)x);
  return exp2f(x);
}
/* e^x of the merge and gather weights: Cody & Waite's two-constant reduction x = k ln2 + r (|r| <= ln2/2, the split
 * of ln2 keeps k * hi exact), e^r by its degree-7 Taylor polynomial in Horner form with fused multiply-adds,
 * e^x = 2^k e^r.  Relative error
 * below 3e-7 on [-80, 88]; below -80 the result is 0.  The CUDA path evaluates the same f32 sequence. */
static inline float gi_exp(float x) {
  if (x != x) return x;
  if (x < -80.0f) return 0.0f;
  if (x > 88.0f) return INFINITY;
  float k = rintf(x * 0x1.715476p+0f);
  float r = (x - k * 0x1.62e4p-1f) - k * 0x1.7f7d1cp-20f;
  float p = 0x1.a01a02p-13f;
  p = fmaf(p, r, 0x1.6c16c2p-10f);
  p = fmaf(p, r, 0x1.111112p-7f);
  p = fmaf(p, r, 0x1.555556p-5f);
  p = fmaf(p, r, 0x1.555556p-3f);
  p = fmaf(p, r, 0.5f);
  p = fmaf(p, r, 1.0f);
  p = fmaf(p, r, 1.0f);
  return ldexpf(p, (int)k);
}
/* log2(x) for x > 0: x = m 2^e with m in [sqrt(1/2), sqrt(2)), log2 m = 2 atanh(s) / ln 2 with s = (m - 1) / (m + 1)
 * by its series through s^11 (|s| <= 0.172) in Horner form with fused multiply-adds.  Exact for powers of two,
 * relative error below 1e-7 elsewhere.  The CUDA path evaluates the same f32 sequence. */
static inline float gi_log2(float x) {
  if (!(x > 0.0f)) return x == 0.0f ? -INFINITY : NAN;
  if (isinf(x)) return x;
  int e;
  float m = frexpf(x, &e);
  if (m < 0.70710678f) { m = m * 2.0f; e -= 1; }
  float s = (m - 1.0f) / (m + 1.0f);
  float z = s * s;
  float p = 0.09090909f;
  p = fmaf(p, z, 0.11111111f);
  p = fmaf(p, z, 0.14285715f);
  p = fmaf(p, z, 0.2f);
  p = fmaf(p, z, 0.33333334f);
  p = fmaf(p, z, 1.0f);
  return (float)e + (s * p) * 2.8853900817779268f;
}
#endif
