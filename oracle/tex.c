/*
 * Base colour textures -- part of the CPU oracle (test infrastructure only; see gi_oracle.h).
 *
 * Restates the library's definition of the reference's base colour sampling (scene_gpu.ts:60-89: rgba8unorm-srgb
 * layers with a mip chain; voxel.ts:325-336 surfaceAt and dynlayer.ts:451-454 shadeSample: textureSampleLevel at level
 * 3 + L, linear filtering, repeat addressing).  The reference's decode, mip generation and filtering run on the GPU's
 * texture hardware and are implementation-defined, so the steps here are the library's own, shared with the CUDA
 * kernels: texels decoded to linear f32 (rgb through the sRGB curve evaluated in double and rounded to f32, alpha
 * k / 255), level k + 1 the mean ((a + b) + (c + d)) / 4 of level k's 2 x 2 texels, a sample the bilinear blend of the
 * four texels around (u n - 0.5, v n - 0.5) of one level with repeat wrapping.  Parity with the reference's pixels is
 * unpinned (no GPU sampler runs here).
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "gi_oracle.h"
#include "orc_math.h"

uint32_t orc_tex_levels(uint32_t size, uint32_t *per_layer) {
  uint32_t levels = 0, per = 0;
  for (uint32_t n = size; n >= 1u; n >>= 1) {
    levels++;
    per += n * n;
    if (n == 1u) break;
  }
  if (per_layer) *per_layer = per;
  return levels;
}

void orc_tex_build(const uint8_t *rgba8, uint32_t size, uint32_t layers, float *out) {
  float lut[256];
  for (int k = 0; k < 256; k++) {
    double c = (double)k / 255.0;
    lut[k] = (float)(c <= 0.04045 ? c / 12.92 : pow((c + 0.055) / 1.055, 2.4));
  }
  uint32_t per = 0, levels = orc_tex_levels(size, &per);
  for (uint32_t l = 0; l < layers; l++) {
    float *t = out + (size_t)l * per * 4u;
    const uint8_t *src = rgba8 + (size_t)l * size * size * 4u;
    for (size_t i = 0; i < (size_t)size * size; i++) {
      t[4 * i] = lut[src[4 * i]];
      t[4 * i + 1] = lut[src[4 * i + 1]];
      t[4 * i + 2] = lut[src[4 * i + 2]];
      t[4 * i + 3] = (float)src[4 * i + 3] / 255.0f;
    }
    uint32_t off = 0;
    for (uint32_t k = 0; k + 1u < levels; k++) {
      uint32_t n = size >> k, m = n / 2u;
      const float *s = t + (size_t)off * 4u;
      float *d = t + (size_t)(off + n * n) * 4u;
      for (uint32_t y = 0; y < m; y++)
        for (uint32_t x = 0; x < m; x++)
          for (int ch = 0; ch < 4; ch++) {
            float a = s[((2u * y) * n + 2u * x) * 4u + ch], b = s[((2u * y) * n + 2u * x + 1u) * 4u + ch];
            float c = s[((2u * y + 1u) * n + 2u * x) * 4u + ch], e = s[((2u * y + 1u) * n + 2u * x + 1u) * 4u + ch];
            d[(y * m + x) * 4u + ch] = ((a + b) + (c + e)) * 0.25f;
          }
      off += n * n;
    }
  }
}

uint32_t orc_tex_layer_of(const orc_scene *s, const orc_material *m) {
  return (s->uv && s->tex && m->base_color_tex != 0u && m->base_color_tex <= s->tex_layers) ? m->base_color_tex : 0u;
}

void orc_tex_sample(const orc_scene *s, uint32_t layer1, float u, float v, uint32_t lod, float out[4]) {
  uint32_t L = lod < s->tex_levels ? lod : s->tex_levels - 1u, off = 0;
  for (uint32_t k = 0; k < L; k++) off += (s->tex_size >> k) * (s->tex_size >> k);
  uint32_t n = s->tex_size >> L;
  const float *t = s->tex + ((size_t)(layer1 - 1u) * s->tex_layer_texels + off) * 4u;
  float x = u * (float)n - 0.5f, y = v * (float)n - 0.5f;
  float fx = floorf(x), fy = floorf(y);
  float ax = x - fx, ay = y - fy;
  int32_t m = (int32_t)n - 1;
  int32_t i0 = f2i(fx) & m, i1 = (int32_t)((uint32_t)f2i(fx) + 1u) & m;
  int32_t j0 = f2i(fy) & m, j1 = (int32_t)((uint32_t)f2i(fy) + 1u) & m;
  const float *a = t + ((size_t)j0 * n + (size_t)i0) * 4u, *b = t + ((size_t)j0 * n + (size_t)i1) * 4u;
  const float *c = t + ((size_t)j1 * n + (size_t)i0) * 4u, *d = t + ((size_t)j1 * n + (size_t)i1) * 4u;
  float bx = 1.0f - ax, by = 1.0f - ay;
  for (int ch = 0; ch < 4; ch++) out[ch] = (a[ch] * bx + b[ch] * ax) * by + (c[ch] * bx + d[ch] * ax) * ay;
}

void orc_tri_uv(const orc_scene *s, const uint32_t idx[3], float wx, float wy, float wz, float uv[2]) {
  const float *a = s->uv + 2u * idx[0], *b = s->uv + 2u * idx[1], *c = s->uv + 2u * idx[2];
  uv[0] = (a[0] * wx + b[0] * wy) + c[0] * wz;
  uv[1] = (a[1] * wx + b[1] * wy) + c[1] * wz;
}

int orc_raster_alpha_ok(const orc_scene *s, const uint32_t idx[4], float wa, float wb, float wc) {
  const orc_material *m = &s->mats[idx[3]];
  if ((m->flags & 1u) == 0u) return 1;
  float a = m->base_color[3];
  uint32_t layer = orc_tex_layer_of(s, m);
  if (layer) {
    float uv[2], t[4];
    orc_tri_uv(s, idx, wa, wb, wc, uv);
    orc_tex_sample(s, layer, uv[0], uv[1], 0u, t);
    a = t[3] * m->base_color[3];
  }
  return !(a < m->alpha_cutoff);
}
