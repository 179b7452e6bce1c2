/* WGSL builtins as the oracle restates them (public WGSL specification formulas), plus the triangle/box test.
 * Test infrastructure only. */
#include "gi_oracle.h"
#include "orc_math.h"

/* pack4x8unorm: floor(0.5 + 255 * min(1, max(0, e))) per component, x in the low byte. */
uint32_t orc_pack4x8unorm(const float v[4]) {
  uint32_t r = 0;
  for (int i = 0; i < 4; i++) {
    float c = fminf_(fmaxf_(v[i], 0.0f), 1.0f);
    uint32_t b = (uint32_t)floorf(0.5f + 255.0f * c);
    r |= (b & 0xffu) << (8 * i);
  }
  return r;
}

/* pack2x16snorm: floor(0.5 + 32767 * min(1, max(-1, e))) as 16-bit two's complement, a in the low half. */
uint32_t orc_pack2x16snorm(float a, float b) {
  float ca = fminf_(fmaxf_(a, -1.0f), 1.0f), cb = fminf_(fmaxf_(b, -1.0f), 1.0f);
  int32_t ia = (int32_t)floorf(0.5f + 32767.0f * ca), ib = (int32_t)floorf(0.5f + 32767.0f * cb);
  return ((uint32_t)ia & 0xffffu) | (((uint32_t)ib & 0xffffu) << 16);
}

/* f32 -> f16, round to nearest even; overflow to infinity; NaN to a quiet NaN. */
uint16_t orc_f32_to_f16(float x) {
  uint32_t u = ubits(x);
  uint32_t sign = (u >> 16) & 0x8000u;
  uint32_t ex = (u >> 23) & 0xffu, man = u & 0x7fffffu;
  if (ex == 0xffu) return (uint16_t)(sign | (man ? 0x7e00u : 0x7c00u));
  int32_t e = (int32_t)ex - 127 + 15;
  if (e >= 31) return (uint16_t)(sign | 0x7c00u);
  if (e <= 0) {
    if (e < -10) return (uint16_t)sign;
    uint32_t m = man | 0x800000u;              /* 24-bit significand */
    uint32_t shift = (uint32_t)(14 - e);       /* to a 10-bit subnormal significand */
    uint32_t q = m >> shift, rem = m & ((1u << shift) - 1u), half = 1u << (shift - 1u);
    if (rem > half || (rem == half && (q & 1u))) q++;
    return (uint16_t)(sign | q);
  }
  uint32_t q = ((uint32_t)e << 10) | (man >> 13), rem = man & 0x1fffu;
  if (rem > 0x1000u || (rem == 0x1000u && (q & 1u))) q++;   /* may carry into the exponent, up to infinity */
  return (uint16_t)(sign | q);
}

float orc_f16_to_f32(uint16_t h) {
  uint32_t sign = ((uint32_t)h & 0x8000u) << 16, e = (h >> 10) & 0x1fu, m = h & 0x3ffu;
  if (e == 0) {
    float f = ldexpf((float)m, -24);
    return sign ? -f : f;
  }
  if (e == 31) return fbits(sign | 0x7f800000u | (m << 13));
  return fbits(sign | ((e - 15 + 127) << 23) | (m << 13));
}

uint16_t orc_f32_to_bf16(float x) {
  uint32_t u = ubits(x);
  if ((u & 0x7fffffffu) > 0x7f800000u) return (uint16_t)((u >> 16) | 0x40u);
  u += 0x7fffu + ((u >> 16) & 1u);
  return (uint16_t)(u >> 16);
}
float orc_bf16_to_f32(uint16_t h) { return fbits((uint32_t)h << 16); }

/* round(log2(x)) exactly: x = m 2^e, m in [0.5, 1); log2 m >= -1/2 <=> m^2 >= 1/2 (exact in double).
 * The half-way case needs m = 2^-1/2, which no float is. */
uint32_t orc_round_log2(float x) {
  if (!(x > 0.0f)) return 0x80000000u;          /* -inf / NaN: callers clamp to level 0 */
  if (isinf(x)) return 0x7fffffffu;
  int e;
  float m = frexpf(x, &e);
  double mm = (double)m * (double)m;
  return (uint32_t)(mm >= 0.5 ? e : e - 1);
}

/* The merge and gather weights' e^x (orc_math.h gi_exp), for its accuracy test. */
float orc_gi_exp(float x) { return gi_exp(x); }

/* Akenine-Moller triangle / box overlap, voxel.ts:231-248, box at c with half size h. */
static int axis_test(v3 a, v3 v0, v3 v1, v3 v2, v3 h) {
  float p0 = dot(v0, a), p1 = dot(v1, a), p2 = dot(v2, a);
  float r = dot(h, vabs(a));
  return !(fminf_(fminf_(p0, p1), p2) > r || fmaxf_(fmaxf_(p0, p1), p2) < -r);
}
int orc_tri_box(const float cf[3], const float hf[3], const float af[3], const float bf[3], const float ccf[3]) {
  v3 c = fromf(cf), h = fromf(hf);
  v3 v0 = sub(fromf(af), c), v1 = sub(fromf(bf), c), v2 = sub(fromf(ccf), c);
  v3 mn = vmin(vmin(v0, v1), v2), mx = vmax(vmax(v0, v1), v2);
  if (mn.x > h.x || mn.y > h.y || mn.z > h.z || mx.x < -h.x || mx.y < -h.y || mx.z < -h.z) return 0;
  v3 e0 = sub(v1, v0), e1 = sub(v2, v1), e2 = sub(v0, v2);
  v3 n = cross(e0, e1);
  if (fabsf(dot(n, v0)) > dot(h, vabs(n))) return 0;
  return axis_test(V(0.0f, -e0.z, e0.y), v0, v1, v2, h) && axis_test(V(0.0f, -e1.z, e1.y), v0, v1, v2, h)
      && axis_test(V(0.0f, -e2.z, e2.y), v0, v1, v2, h) && axis_test(V(e0.z, 0.0f, -e0.x), v0, v1, v2, h)
      && axis_test(V(e1.z, 0.0f, -e1.x), v0, v1, v2, h) && axis_test(V(e2.z, 0.0f, -e2.x), v0, v1, v2, h)
      && axis_test(V(-e0.y, e0.x, 0.0f), v0, v1, v2, h) && axis_test(V(-e1.y, e1.x, 0.0f), v0, v1, v2, h)
      && axis_test(V(-e2.y, e2.x, 0.0f), v0, v1, v2, h);
}
