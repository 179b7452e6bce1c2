/* Sequential restatement of the dynamic layer (src/core/dynlayer.ts): its build (mark, parents, count + alloc,
 * finalize, clear, splat, resolve; dynlayer.ts:182-587) and its read by the interval tracers (dynFind, dynWord,
 * dynRead, traceDyn; dynlayer.ts:71-162).  Test infrastructure only.
 *
 * Splat sums are fixed point (x 65536) and so exact: the GPU adds them with atomics in any order and gets these
 * integers.  The reference's splat first gathers a workgroup's samples in a window of workgroup memory and marks a
 * voxel non-zero only when the window's sum is; samples outside the window mark the voxel whenever their weight is
 * positive.  That choice changes no value (a voxel whose words are all zero resolves to zeros either way), so both
 * paths here add every sample straight to the layer and mark the voxel when its weight is positive.
 * Materials are untextured (the sampled colour is the base colour factor).  The albedo words are written only with
 * `albedo` set (the reference's DYN_ALB, configs with the token obj). */
#include <stdlib.h>
#include "gi_oracle.h"
#include "orc_math.h"
#include "orc_rc.h"

#define DYN_HDR 64u
#define DYN_W 13u
#define DYN_FIX 65536.0f
#define DYN_EMPTY 0xffffffffu
#define DYN_DROPPED 0xfffffffdu
#define DYN_NONE 0xffffffffu

static inline uint32_t g3(const orc_vox *vx) { return vx->G * vx->G * vx->G; }
static inline uint32_t nwords(const orc_vox *vx) { return vx->levels * g3(vx) / 32u; }
static inline v3 region_lo(const orc_vox *vx, uint32_t L) { return muls(muls(vi2f(org(vx, L)), vox_size(vx, L)), 8.0f); }
static inline v3 region_hi(const orc_vox *vx, uint32_t L) {
  float e = (float)vx->G * vox_size(vx, L) * 8.0f;
  return adds(region_lo(vx, L), e);
}
static inline v3 P3(const orc_scene *s, uint32_t i) { return fromf(s->pos + 3u * i); }
static inline v3 N3(const orc_scene *s, uint32_t i) { return fromf(s->nrm + 3u * i); }

void orc_dyn_init(const orc_vox *vx, orc_dyn *dl) {
  uint32_t np = vx->levels * g3(vx);
  memset(dl->hdr, 0, DYN_HDR * 4u);
  for (uint32_t k = 32; k < 35; k++) dl->hdr[k] = 0xffffffffu;
  for (uint32_t i = 0; i < np; i++) dl->ptr[i] = DYN_EMPTY;
  memset(dl->bits, 0, (size_t)2u * nwords(vx) * 4u);
  memset(dl->meta, 0, (size_t)dl->nb * 4u);
  memset(dl->mask, 0, (size_t)dl->nb * 16u * 4u);
  memset(dl->data, 0, (size_t)dl->nb * 512u * DYN_W * 4u);
}

/* splatLevel (dynlayer.ts:221-229): the finest level whose clipmap holds the box grown by two voxels */
static uint32_t splat_level(const orc_vox *vx, v3 mn, v3 mx) {
  for (uint32_t L = 0; L < vx->levels; L++) {
    float v = vox_size(vx, L), v2 = 2.0f * v;
    v3 lo = region_lo(vx, L), hi = region_hi(vx, L);
    if (mn.x - v2 > lo.x && mn.y - v2 > lo.y && mn.z - v2 > lo.z && mx.x + v2 < hi.x && mx.y + v2 < hi.y && mx.z + v2 < hi.z)
      return L;
  }
  return DYN_NONE;
}

/* want (dynlayer.ts:236-243): brick b of level L in this frame's bitset */
static void want(const orc_vox *vx, orc_dyn *dl, uint32_t L, i3 b) {
  int32_t G = (int32_t)vx->G;
  if (b.x < 0 || b.y < 0 || b.z < 0 || b.x >= G || b.y >= G || b.z >= G) return;
  uint32_t ug = vx->G, g = (vx->levels - 1u - L) * ug * ug * ug + ((uint32_t)b.z * ug + (uint32_t)b.y) * ug + (uint32_t)b.x;
  uint32_t *cur = dl->bits + (dl->hdr[10] & 1u) * nwords(vx);
  cur[g >> 5] |= 1u << (g & 31u);
}

/* WGSL u32(round(x)) of a non-negative x: round half to even, saturating */
static inline uint32_t fix_of(float x) {
  float q = rintf(x * DYN_FIX);
  if (!(q > 0.0f)) return 0u;
  if (q >= 4294967296.0f) return 0xffffffffu;
  return (uint32_t)q;
}

/* shadeSample (dynlayer.ts:445-455): tc the sampled base colour (texture times factor, or the factor untextured); rgb
 * and the albedo; 0 when the alpha test discards the sample */
static int shade_sample(const orc_material *m, const float tc[4], const float *F, const float *map, uint32_t S, v3 p,
                        v3 n, v3 *rad, v3 *alb) {
  v3 tex = V(tc[0], tc[1], tc[2]);
  if ((m->flags & 1u) != 0u && tc[3] < m->alpha_cutoff) return 0;
  *alb = tex;
  float ndl = fmaxf_(dot(n, fromf(F + F_SUN)), 0.0f);
  if (ndl <= 0.0f) { *rad = V(0.0f, 0.0f, 0.0f); return 1; }
  float vis = 1.0f;
  if (map && S) {
    v3 q = add(p, muls(n, 0.03f));
    float x[3] = {q.x, q.y, q.z};
    vis = orc_sun_tap(F, map, S, x);
  }
  v3 sunE = fromf(F + F_SUNE);
  if ((m->flags & 4u) != 0u && F[F_STYLE] > 0.5f) {
    /* toonSun (style.ts:18-25) */
    float l = dot(tex, V(0.2126f, 0.7152f, 0.0722f));
    v3 t = add(V(l, l, l), muls(sub(tex, V(l, l, l)), 1.6f));
    t = V(fclampf(t.x, 0.0f, 1.0f), fclampf(t.y, 0.0f, 1.0f), fclampf(t.z, 0.0f, 1.0f));
    float x = ndl * vis, ramp = x > 0.3f ? 1.0f : (x > 0.05f ? 0.5f : 0.0f);
    *rad = muls(mul(divs(t, PI_F), sunE), ramp);
    return 1;
  }
  *rad = muls(muls(mul(divs(tex, PI_F), sunE), ndl), vis);
  return 1;
}

/* splatSample (dynlayer.ts:406-441): the sample's trilinear weights over the 8 nearest voxel centres */
static void splat_sample(const orc_vox *vx, orc_dyn *dl, uint32_t L, v3 p, v3 n, float area, v3 rad, v3 alb) {
  float v = vox_size(vx, L);
  v3 g = adds(divs(sub(p, region_lo(vx, L)), v), -0.5f);
  i3 c0 = vf2i(vfloor(g));
  v3 f = sub(g, vi2f(c0));
  float s = area / (v * v);
  v3 pn = vmax(n, V(0.0f, 0.0f, 0.0f)), nn = vmax(neg(n), V(0.0f, 0.0f, 0.0f));
  int32_t G8 = (int32_t)vx->G * 8;
  uint32_t G = vx->G;
  for (uint32_t k = 0; k < 8u; k++) {
    i3 o = I((int32_t)(k & 1u), (int32_t)((k >> 1) & 1u), (int32_t)(k >> 2));
    i3 c = I(c0.x + o.x, c0.y + o.y, c0.z + o.z);
    if (c.x < 0 || c.y < 0 || c.z < 0 || c.x >= G8 || c.y >= G8 || c.z >= G8) continue;
    v3 tw = V(o.x == 1 ? f.x : 1.0f - f.x, o.y == 1 ? f.y : 1.0f - f.y, o.z == 1 ? f.z : 1.0f - f.z);
    float w = tw.x * tw.y * tw.z * s;
    if (w <= 0.0f) continue;
    uint32_t ptr = dl->ptr[L * G * G * G + ((uint32_t)(c.z >> 3) * G + (uint32_t)(c.y >> 3)) * G + (uint32_t)(c.x >> 3)];
    if (ptr >= dl->nb) continue;
    uint32_t vi = (uint32_t)((c.x & 7) + 8 * (c.y & 7) + 64 * (c.z & 7));
    dl->mask[ptr * 16u + (vi >> 5)] |= 1u << (vi & 31u);
    uint32_t *d = dl->data + ((size_t)ptr * 512u + vi) * DYN_W;
    float x[13] = {w * pn.x, w * nn.x, w * pn.y, w * nn.y, w * pn.z, w * nn.z, w, w * rad.x, w * rad.y, w * rad.z,
                   w * alb.x, w * alb.y, w * alb.z};
    uint32_t nw = dl->albedo ? 13u : 10u;
    for (uint32_t q = 0; q < nw; q++) d[q] += fix_of(x[q]);
  }
}

int orc_dyn_build(const orc_scene *s, const orc_vox *vx, orc_dyn *dl, uint32_t first, uint32_t end, const float *F,
                  const float *map, uint32_t S) {
  if (end <= first) return 0;   /* no dynamic triangles: the layer keeps its state (DynLayer.encode) */
  const uint32_t n = vx->levels, G = vx->G, G3 = g3(vx), nw = nwords(vx), nb = dl->nb;
  uint32_t *hdr = dl->hdr;
  /* mark (dynlayer.ts:246-270) */
  for (uint32_t t = first; t < end; t++) {
    const uint32_t *ti = s->tri + 4u * t;
    v3 a = P3(s, ti[0]), b = P3(s, ti[1]), c = P3(s, ti[2]);
    v3 mn = vmin(vmin(a, b), c), mx = vmax(vmax(a, b), c);
    uint32_t Ls = splat_level(vx, mn, mx);
    if (Ls == DYN_NONE) { hdr[38]++; continue; }
    float v = vox_size(vx, Ls), bs = v * 8.0f;
    v3 lo = region_lo(vx, Ls);
    i3 g0 = vf2i(vfloor(divs(sub(adds(mn, -v), lo), bs))), g1 = vf2i(vfloor(divs(sub(adds(mx, v), lo), bs)));
    for (int32_t z = g0.z; z <= g1.z; z++)
      for (int32_t y = g0.y; y <= g1.y; y++)
        for (int32_t x = g0.x; x <= g1.x; x++) want(vx, dl, Ls, I(x, y, z));
    float gv = vox_size(vx, n - 1u);
    for (int k = 0; k < 3; k++) {
      uint32_t blo = (uint32_t)(f2i(floorf((comp(mn, k) - gv) * 100.0f)) + 1073741824);
      uint32_t bhi = (uint32_t)(f2i(ceilf((comp(mx, k) + gv) * 100.0f)) + 1073741824);
      if (blo < hdr[32 + k]) hdr[32 + k] = blo;
      if (bhi > hdr[35 + k]) hdr[35 + k] = bhi;
    }
  }
  /* parents (dynlayer.ts:272-296): every wanted brick below the coarsest level wants its ancestors */
  uint32_t *cur = dl->bits + (hdr[10] & 1u) * nw, *prev = dl->bits + (1u - (hdr[10] & 1u)) * nw;
  for (uint32_t w = G3 / 32u; w < nw; w++) {
    uint32_t m = cur[w];
    while (m) {
      uint32_t bit = (uint32_t)__builtin_ctz(m);
      m &= m - 1u;
      uint32_t g = w * 32u + bit, lr = g / G3, L = n - 1u - lr, r = g - lr * G3;
      i3 b = I((int32_t)(r % G), (int32_t)((r / G) % G), (int32_t)(r / (G * G)));
      while (L + 1u < n) {
        i3 o = org(vx, L), o1 = org(vx, L + 1u);
        b = I(((o.x + b.x) * 8 / 2 - o1.x * 8) >> 3, ((o.y + b.y) * 8 / 2 - o1.y * 8) >> 3, ((o.z + b.z) * 8 / 2 - o1.z * 8) >> 3);
        L++;
        want(vx, dl, L, b);
      }
    }
  }
  /* count + alloc (dynlayer.ts:311-362): slots by rank in bit order; bricks wanted last frame only are emptied */
  uint32_t excl = 0;
  for (uint32_t w = 0; w < nw; w++) {
    uint32_t cw = cur[w], old = prev[w], c = popc(cw);
    if ((w * 32u) % G3 == 0u) hdr[16u + n - 1u - w * 32u / G3] = excl;
    if (w == nw - 1u) hdr[0] = excl + c;
    uint32_t m = cw | old;
    while (m) {
      uint32_t bit = (uint32_t)__builtin_ctz(m);
      m &= m - 1u;
      uint32_t g = w * 32u + bit, lr = g / G3, pi = (n - 1u - lr) * G3 + g - lr * G3;
      if ((cw >> bit) & 1u) {
        uint32_t rank = excl + popc(cw & ((1u << bit) - 1u));
        if (rank < nb) { dl->ptr[pi] = rank; dl->meta[rank] = pi; }
        else dl->ptr[pi] = DYN_DROPPED;
      } else {
        dl->ptr[pi] = DYN_EMPTY;
      }
    }
    prev[w] = 0u;
    excl += c;
  }
  /* finalize (dynlayer.ts:364-386) */
  uint32_t total = hdr[0], al = total < nb ? total : nb;
  hdr[8] = al; hdr[1] = total - al;
  for (uint32_t L = 0; L < n; L++) {
    uint32_t e = L > 0 ? hdr[16u + L - 1u] : total;
    uint32_t s0 = hdr[16u + L] < nb ? hdr[16u + L] : nb;
    uint32_t c = (e < nb ? e : nb) - s0;
    hdr[16u + L] = s0; hdr[24u + L] = c;
  }
  for (int k = 0; k < 3; k++) {
    hdr[2 + k] = hdr[32 + k]; hdr[32 + k] = 0xffffffffu;
    hdr[5 + k] = hdr[35 + k]; hdr[35 + k] = 0u;
  }
  hdr[9] = hdr[38]; hdr[38] = 0u;
  hdr[10]++;
  /* clear (dynlayer.ts:387-392) */
  memset(dl->data, 0, (size_t)al * 512u * DYN_W * 4u);
  memset(dl->mask, 0, (size_t)al * 16u * 4u);
  /* splat (dynlayer.ts:458-526): per dynamic triangle m^2 sub-triangles, a sample at each centroid */
  for (uint32_t t = first; t < end; t++) {
    const uint32_t *ti = s->tri + 4u * t;
    v3 a = P3(s, ti[0]), b = P3(s, ti[1]), c = P3(s, ti[2]);
    uint32_t L = splat_level(vx, vmin(vmin(a, b), c), vmax(vmax(a, b), c));
    if (L == DYN_NONE) continue;
    float area = 0.5f * length3(cross(sub(b, a), sub(c, a)));
    if (area <= 0.0f) continue;
    float e = fmaxf_(fmaxf_(length3(sub(b, a)), length3(sub(c, b))), length3(sub(a, c)));
    uint32_t m = (uint32_t)fclampf(ceilf(e / vox_size(vx, L)), 1.0f, 16.0f);
    float fm = (float)m, sa = area / (fm * fm);
    const orc_material *mat = &s->mats[ti[3]];
    const uint32_t tex_layer = orc_tex_layer_of(s, mat);
    for (uint32_t u = 0; u < m; u++)
      for (uint32_t vv = 0; vv + u < m; vv++)
        for (uint32_t flip = 0; flip < 2u; flip++) {
          if (flip == 1u && u + vv + 1u >= m) continue;
          float off = flip == 1u ? 2.0f / 3.0f : 1.0f / 3.0f;
          float wb = ((float)u + off) / fm, wc = ((float)vv + off) / fm, wa = 1.0f - wb - wc;
          v3 p = add(add(muls(a, wa), muls(b, wb)), muls(c, wc));
          v3 nr = add(add(muls(N3(s, ti[0]), wa), muls(N3(s, ti[1]), wb)), muls(N3(s, ti[2]), wc));
          nr = normalize3(dot(nr, nr) > 1e-12f ? nr : cross(sub(b, a), sub(c, a)));
          v3 rad, alb;
          float tc[4] = {mat->base_color[0], mat->base_color[1], mat->base_color[2], mat->base_color[3]};
          if (tex_layer) {   /* the texture at level 3 + L at the sample's uv, times the factor */
            float uv[2], t[4];
            orc_tri_uv(s, ti, wa, wb, wc, uv);
            orc_tex_sample(s, tex_layer, uv[0], uv[1], 3u + L, t);
            for (int k = 0; k < 4; k++) tc[k] = t[k] * mat->base_color[k];
          }
          if (!shade_sample(mat, tc, F, map, S, p, nr, &rad, &alb)) continue;
          splat_sample(vx, dl, L, p, nr, sa, rad, alb);
        }
  }
  /* resolve (dynlayer.ts:527-587), levels 1 .. n-1 fine to coarse */
  for (uint32_t L = 1; L < n; L++) {
    uint32_t s0 = hdr[16u + L], cnt = hdr[24u + L];
    for (uint32_t slot = s0; slot < s0 + cnt; slot++) {
      uint32_t pi = dl->meta[slot], r = pi % G3;
      for (uint32_t bit = 0; bit < 512u; bit++) {
        i3 c = I((int32_t)(r % G) * 8 + (int32_t)(bit & 7u), (int32_t)((r / G) % G) * 8 + (int32_t)((bit >> 3) & 7u),
                 (int32_t)(r / (G * G)) * 8 + (int32_t)(bit >> 6));
        uint32_t own = (dl->mask[slot * 16u + (bit >> 5)] >> (bit & 31u)) & 1u;
        i3 o = org(vx, L), o1 = org(vx, L - 1u);
        i3 gc = I((o.x * 8 + c.x) * 2 - o1.x * 8, (o.y * 8 + c.y) * 2 - o1.y * 8, (o.z * 8 + c.z) * 2 - o1.z * 8);
        uint32_t cptr = nb;
        int32_t G8 = (int32_t)G * 8;
        if (gc.x >= 0 && gc.y >= 0 && gc.z >= 0 && gc.x < G8 && gc.y < G8 && gc.z < G8)
          cptr = dl->ptr[(L - 1u) * G3 + ((uint32_t)(gc.z >> 3) * G + (uint32_t)(gc.y >> 3)) * G + (uint32_t)(gc.x >> 3)];
        uint32_t kids = 0, kv[8];
        if (cptr < nb)
          for (uint32_t q = 0; q < 8u; q++) {
            i3 l = I((gc.x & 7) + (int32_t)(q & 1u), (gc.y & 7) + (int32_t)((q >> 1) & 1u), (gc.z & 7) + (int32_t)(q >> 2));
            kv[q] = (uint32_t)(l.x + 8 * l.y + 64 * l.z);
            if ((dl->mask[cptr * 16u + (kv[q] >> 5)] >> (kv[q] & 31u)) & 1u) kids |= 1u << q;
          }
        if (own == 0u && kids == 0u) continue;
        uint32_t *d = dl->data + ((size_t)slot * 512u + bit) * DYN_W;
        float acc[13];
        for (uint32_t k = 0; k < DYN_W; k++) acc[k] = (float)d[k] / DYN_FIX;
        for (uint32_t q = 0; q < 8u; q++) {
          if (((kids >> q) & 1u) == 0u) continue;
          const uint32_t *cb = dl->data + ((size_t)cptr * 512u + kv[q]) * DYN_W;
          for (uint32_t k = 0; k < DYN_W; k++) {
            float x = L == 1u ? (float)cb[k] / DYN_FIX : fbits(cb[k]);
            acc[k] += 0.25f * x;
          }
        }
        for (uint32_t k = 0; k < DYN_W; k++) d[k] = ubits(acc[k]);
        if (own == 0u) dl->mask[slot * 16u + (bit >> 5)] |= 1u << (bit & 31u);
      }
    }
  }
  return 0;
}

/* ---- read side (dynlayer.ts:71-162) ---------------------------------------------------------------------------- */

/* dynFind: the data base of the voxel at p of level L, or of the first coarser level whose brick was not dropped;
 * DYN_NONE when empty.  *lvl: the level read. */
static uint32_t dyn_find(const orc_vox *vx, const orc_dyn *dl, uint32_t L, v3 p, uint32_t *lvl) {
  const int32_t G = (int32_t)vx->G;
  const uint32_t ug = vx->G, nl = vx->levels;
  uint32_t l = L;
  for (;;) {
    float v = vox_size(vx, l);
    i3 c = vf2i(vfloor(divs(sub(p, region_lo(vx, l)), v)));
    *lvl = l;
    if (c.x < 0 || c.y < 0 || c.z < 0 || c.x >= G * 8 || c.y >= G * 8 || c.z >= G * 8) return DYN_NONE;
    uint32_t ptr = dl->ptr[l * ug * ug * ug + ((uint32_t)(c.z >> 3) * ug + (uint32_t)(c.y >> 3)) * ug + (uint32_t)(c.x >> 3)];
    if (ptr == DYN_DROPPED && l + 1u < nl) { l++; continue; }
    if (ptr >= dl->nb) return DYN_NONE;
    return (ptr * 512u + (uint32_t)((c.x & 7) + 8 * (c.y & 7) + 64 * (c.z & 7))) * DYN_W;
  }
}
static inline float dyn_word(const orc_dyn *dl, uint32_t base, uint32_t k, uint32_t L) {
  uint32_t u = dl->data[base + k];
  return L == 0u ? (float)u / DYN_FIX : fbits(u);
}
float dyn_word_at(const orc_dyn *dl, uint32_t base, uint32_t k, uint32_t L) { return dyn_word(dl, base, k, L); }
void dyn_add_radiance(orc_dyn *dl, uint32_t base, uint32_t L, const float add[3]) {
  for (uint32_t k = 0; k < 3u; k++) {
    uint32_t *w = &dl->data[base + 7u + k];
    if (L == 0u) *w += fix_of(add[k]);
    else *w = ubits(fbits(*w) + add[k]);
  }
}
/* dynRead: mean radiance and coverage per voxel length for direction d (the three faces against d) */
static void dyn_read(const orc_dyn *dl, uint32_t base, uint32_t L, v3 d, float out[4]) {
  out[0] = out[1] = out[2] = out[3] = 0.0f;
  if (base == DYN_NONE) return;
  float a = dyn_word(dl, base, 6u, L);
  if (a <= 0.0f) return;
  v3 ad = vabs(d);
  uint32_t sx = d.x > 0.0f ? 1u : 0u, sy = d.y > 0.0f ? 1u : 0u, sz = d.z > 0.0f ? 1u : 0u;
  float front = ad.x * dyn_word(dl, base, sx, L) + ad.y * dyn_word(dl, base, 2u + sy, L) + ad.z * dyn_word(dl, base, 4u + sz, L);
  out[0] = dyn_word(dl, base, 7u, L) / a;
  out[1] = dyn_word(dl, base, 8u, L) / a;
  out[2] = dyn_word(dl, base, 9u, L) / a;
  out[3] = fminf_(front, 1.0f);
}

float orc_log2(float x) { return gi_log2(x); }

void orc_trace_dyn(const orc_vox *vx, float o3[3], float d3[3], float t0, float t1, float k, float out[4]) {
  const orc_dyn *dl = vx->dyn;
  out[0] = out[1] = out[2] = out[3] = 0.0f;
  if (!dl || dl->hdr[0] == 0u || t1 <= t0) return;
  v3 o = fromf(o3), d = fromf(d3);
  v3 bmin = muls(adds(V((float)dl->hdr[2], (float)dl->hdr[3], (float)dl->hdr[4]), -1073741824.0f), 0.01f);
  v3 bmax = muls(adds(V((float)dl->hdr[5], (float)dl->hdr[6], (float)dl->hdr[7]), -1073741824.0f), 0.01f);
  v3 dd = V(fabsf(d.x) < 1e-9f ? 1e-9f : d.x, fabsf(d.y) < 1e-9f ? 1e-9f : d.y, fabsf(d.z) < 1e-9f ? 1e-9f : d.z);
  v3 ta = divv(sub(bmin, o), dd), tb = divv(sub(bmax, o), dd);
  v3 tn = vmin(ta, tb), tf = vmax(ta, tb);
  float ba = fmaxf_(fmaxf_(fmaxf_(tn.x, tn.y), tn.z), t0);
  float bb = fminf_(fminf_(fminf_(tf.x, tf.y), tf.z), t1);
  if (ba >= bb) return;
  const float v0 = vx->v0;
  const uint32_t nl = vx->levels;
  v3 rad = V(0.0f, 0.0f, 0.0f);
  float cov = 0.0f, t = t0;
  for (uint32_t i = 0; i < 128u; i++) {
    if (t >= bb || cov >= 1.0f) break;
    float w = fmaxf_(k * t, v0);
    float te = fminf_(t + 0.5f * w, t1);
    if (te > ba) {
      float len = te - t;
      v3 p = add(o, muls(d, 0.5f * (t + te)));
      float lf = fclampf(gi_log2(w / v0), 0.0f, (float)(nl - 1u));
      uint32_t L0 = (uint32_t)floorf(lf);
      float f = lf - (float)L0;
      uint32_t Lw = vox_level_for(vx, L0, p);
      if (Lw != L0) { L0 = Lw; f = 0.0f; }
      uint32_t la, lb;
      float sa[4], sb[4];
      uint32_t fa = dyn_find(vx, dl, L0, p, &la);
      dyn_read(dl, fa, la, d, sa);
      float aa = sa[3] * len / vox_size(vx, la);
      v3 ra = muls(V(sa[0], sa[1], sa[2]), aa);
      if (f > 0.0f && L0 + 1u < nl) {
        uint32_t fb = dyn_find(vx, dl, L0 + 1u, p, &lb);
        dyn_read(dl, fb, lb, d, sb);
        float ab = sb[3] * len / vox_size(vx, lb);
        v3 rb = muls(V(sb[0], sb[1], sb[2]), ab);
        ra = add(muls(ra, 1.0f - f), muls(rb, f));      /* mix(ra, rb, f) */
        aa = aa * (1.0f - f) + ab * f;
      }
      if (aa > 0.0f) {
        float a = fminf_(aa, 1.0f - cov);
        rad = add(rad, muls(ra, a / aa));
        cov += a;
      }
    }
    t = te;
  }
  out[0] = rad.x; out[1] = rad.y; out[2] = rad.z; out[3] = cov;
}

/* traceWorld's read of the dynamic layer (rc.ts:223-231): in front of the static hit (or to t1 on a miss), from at
 * least one level-0 voxel out, the covered radiance composited over the voxel trace's result.  o: the probe, ooff:
 * the trace's start (o moved along the probe normal), k: the cone width per unit distance. */
void dyn_compose(const orc_vox *vx, v3 o, v3 d, float t0, float t1, v3 ooff, float k, trace_t *tr) {
  if (!vx->dyn || vx->dyn->hdr[0] == 0u) return;
  float tS = t1;
  if (tr->T < 0.5f) tS = dot(sub(add(ooff, muls(d, fbits(tr->tin))), o), d);
  float oo[3] = {o.x, o.y, o.z}, dd[3] = {d.x, d.y, d.z}, out[4];
  orc_trace_dyn(vx, oo, dd, fmaxf_(t0, vx->v0), fminf_(t1, tS), k, out);
  if (out[3] > 0.0f) {
    float s = 1.0f - out[3];
    tr->r = out[0] + s * tr->r; tr->g = out[1] + s * tr->g; tr->b = out[2] + s * tr->b;
    tr->T = s * tr->T;
  }
}
