/* Sequential restatement of the voxel clipmap rebuild (src/core/voxel.ts:205-620).  Test infrastructure only.
 *
 * The GPU build is a set of passes whose results do not depend on scheduling (bits are ORed, representatives are the
 * maximum triangle index + 1); this file runs the same passes one after another.  Two allocations depend on the
 * order of an atomic counter in the reference (bricks when the pool holds them all, voxel attribute bases); both
 * are restated here in the fixed order the reference uses when the brick pool overflows (coarse levels first, then
 * pointer index; attribute bases in brick order), which is one of the orders the reference can produce and the one
 * the CUDA path uses. */
#include <stdlib.h>
#include "gi_oracle.h"
#include "orc_math.h"
#include "orc_par.h"

#define BIG 8u

typedef struct { v3 a, b, c; const uint32_t *idx; } tri_t;
typedef struct { i3 lo, n; } range_t;

static inline float vox_size(const orc_vox *vx, uint32_t L) { return scale2(vx->v0, (int)L); }
static inline uint32_t ptr_index(const orc_vox *vx, uint32_t L, i3 b) {
  uint32_t G = vx->G;
  return L * G * G * G + ((uint32_t)b.z * G + (uint32_t)b.y) * G + (uint32_t)b.x;
}
static inline i3 org(const orc_vox *vx, uint32_t L) { return I(vx->origin[L][0], vx->origin[L][1], vx->origin[L][2]); }
/* regionLo (voxel.ts:289): vec3f(origin) * voxSize(L) * 8 */
static inline v3 region_lo(const orc_vox *vx, uint32_t L) { return muls(muls(vi2f(org(vx, L)), vox_size(vx, L)), 8.0f); }
static inline i3 ishr(i3 a, int s) { return I(a.x >> s, a.y >> s, a.z >> s); }

/* loadTri (voxel.ts:270-276): key = instance * key_stride + row; the instance's offset moves the triangle */
static tri_t load_tri(const orc_scene *s, uint32_t key) {
  tri_t T;
  uint32_t inst = s->items ? key / s->key_stride : 0u, row = key - inst * (s->items ? s->key_stride : 0u);
  const uint32_t *i = s->tri + 4u * row;
  T.a = fromf(s->pos + 3u * i[0]); T.b = fromf(s->pos + 3u * i[1]); T.c = fromf(s->pos + 3u * i[2]);
  if (s->items) {
    v3 o = fromf(s->inst + 4u * inst);
    T.a = add(T.a, o); T.b = add(T.b, o); T.c = add(T.c, o);
  }
  T.idx = i;
  return T;
}
/* workAt (voxel.ts:280-288): thread i of a triangle pass -> its key and first level */
static uint32_t work_at(const orc_scene *s, uint32_t i, uint32_t *first) {
  if (!s->items) { *first = 0; return i; }
  uint32_t lo = 0, hi = s->nitems;
  while (hi - lo > 1u) { uint32_t m = (lo + hi) / 2u; if (s->items[m * 4u] <= i) lo = m; else hi = m; }
  const uint32_t *b = s->items + lo * 4u;
  uint32_t j = i - b[0], src = b[1];
  uint32_t row = (src & 0x80000000u) ? (src & 0x7fffffffu) + j : s->lists[src + j];
  *first = b[3];
  return b[2] * s->key_stride + row;
}
static uint32_t threads_of(const orc_scene *s) { return s->items ? s->threads : s->ntris; }
static uint32_t key_limit(const orc_scene *s) { return s->items ? s->ninst * s->key_stride : s->ntris; }

/* voxRange (voxel.ts:293-300) */
static range_t vox_range(const orc_vox *vx, const tri_t *T, uint32_t L, float cell) {
  v3 lo = region_lo(vx, L);
  v3 mn = vmin(vmin(T->a, T->b), T->c), mx = vmax(vmax(T->a, T->b), T->c);
  int32_t lim = f2i((float)vx->G * vox_size(vx, L) * 8.0f / cell);
  i3 a = vf2i(vfloor(divs(sub(mn, lo), cell)));
  i3 b = vf2i(vfloor(divs(sub(mx, lo), cell)));
  a = iclamp3(a, I(0, 0, 0), I(lim, lim, lim));
  b = iclamp3(I(b.x + 1, b.y + 1, b.z + 1), I(0, 0, 0), I(lim, lim, lim));
  range_t r;
  r.lo = a;
  r.n = I(imax(b.x - a.x, 0), imax(b.y - a.y, 0), imax(b.z - a.z, 0));
  return r;
}

/* finerHolds / finerHoldsRange / finerBuilt / finerBuiltRange (voxel.ts:303-320) */
static int finer_holds(const orc_vox *vx, uint32_t L, i3 c) {
  if (L == 0) return 0;
  i3 o = org(vx, L), of = org(vx, L - 1);
  int32_t n = (int32_t)vx->G * 8;
  i3 f = I((o.x * 8 + c.x) * 2 - of.x * 8, (o.y * 8 + c.y) * 2 - of.y * 8, (o.z * 8 + c.z) * 2 - of.z * 8);
  return f.x >= 0 && f.y >= 0 && f.z >= 0 && f.x < n && f.y < n && f.z < n;
}
static int finer_holds_range(const orc_vox *vx, uint32_t L, range_t r, int32_t s) {
  return finer_holds(vx, L, I(r.lo.x * s, r.lo.y * s, r.lo.z * s))
      && finer_holds(vx, L, I((r.lo.x + r.n.x) * s - 1, (r.lo.y + r.n.y) * s - 1, (r.lo.z + r.n.z) * s - 1));
}
static int finer_built(const orc_vox *vx, uint32_t L, i3 c) {
  if (!finer_holds(vx, L, c)) return 0;
  if (vx->hdr[2] == 0) return 1;
  i3 o = org(vx, L), of = org(vx, L - 1);
  i3 f = I((o.x * 8 + c.x) * 2 - of.x * 8, (o.y * 8 + c.y) * 2 - of.y * 8, (o.z * 8 + c.z) * 2 - of.z * 8);
  return vx->ptr[ptr_index(vx, L - 1, ishr(f, 3))] != ORC_DROP;
}
static int finer_built_range(const orc_vox *vx, uint32_t L, range_t r) {
  return vx->hdr[2] == 0 && finer_holds_range(vx, L, r, 1);
}

static int tri_box_v(v3 c, v3 h, const tri_t *T) {
  float cf[3] = {c.x, c.y, c.z}, hf[3] = {h.x, h.y, h.z};
  float af[3] = {T->a.x, T->a.y, T->a.z}, bf[3] = {T->b.x, T->b.y, T->b.z}, cc[3] = {T->c.x, T->c.y, T->c.z};
  return orc_tri_box(cf, hf, af, bf, cc);
}

/* closestBary (voxel.ts:250-267), Ericson 5.1.5 */
static v3 closest_bary(v3 p, v3 a, v3 b, v3 c) {
  v3 ab = sub(b, a), ac = sub(c, a), ap = sub(p, a);
  float d1 = dot(ab, ap), d2 = dot(ac, ap);
  if (d1 <= 0.0f && d2 <= 0.0f) return V(1.0f, 0.0f, 0.0f);
  v3 bp = sub(p, b);
  float d3 = dot(ab, bp), d4 = dot(ac, bp);
  if (d3 >= 0.0f && d4 <= d3) return V(0.0f, 1.0f, 0.0f);
  float vc = d1 * d4 - d3 * d2;
  if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) { float w = d1 / (d1 - d3); return V(1.0f - w, w, 0.0f); }
  v3 cp = sub(p, c);
  float d5 = dot(ab, cp), d6 = dot(ac, cp);
  if (d6 >= 0.0f && d5 <= d6) return V(0.0f, 0.0f, 1.0f);
  float vb = d5 * d2 - d1 * d6;
  if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) { float w = d2 / (d2 - d6); return V(1.0f - w, 0.0f, w); }
  float va = d3 * d6 - d5 * d4;
  if (va <= 0.0f && (d4 - d3) >= 0.0f && (d5 - d6) >= 0.0f) {
    float w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
    return V(0.0f, 1.0f - w, w);
  }
  float dn = 1.0f / (va + vb + vc);
  float v = vb * dn, w = vc * dn;
  return V(1.0f - v - w, v, w);
}

typedef struct { int ok; float albedo[3]; v3 n; float toon; v3 q; } surf_t;
/* surfaceAt (voxel.ts:325-336): the base colour texture at level 3 + L at p's closest point, times the factor
 * (untextured: the factor alone, the reference's white default layer); the alpha test when masked and not wantAttr. */
static surf_t surface_at(const orc_scene *s, const tri_t *T, v3 p, uint32_t L, int want_attr) {
  surf_t r;
  memset(&r, 0, sizeof r);
  const orc_material *m = &s->mats[T->idx[3]];
  int masked = (m->flags & 1u) != 0 && !want_attr;
  r.q = p;
  if (!masked && !want_attr) { r.ok = 1; return r; }
  v3 w = closest_bary(p, T->a, T->b, T->c);
  float tex[4] = {m->base_color[0], m->base_color[1], m->base_color[2], m->base_color[3]};
  uint32_t layer = orc_tex_layer_of(s, m);
  if (layer) {
    float uv[2], t[4];
    orc_tri_uv(s, T->idx, w.x, w.y, w.z, uv);
    orc_tex_sample(s, layer, uv[0], uv[1], 3u + L, t);
    for (int k = 0; k < 4; k++) tex[k] = t[k] * m->base_color[k];
  }
  if (masked && tex[3] < m->alpha_cutoff) { r.ok = 0; return r; }
  v3 n0 = fromf(s->nrm + 3u * T->idx[0]), n1 = fromf(s->nrm + 3u * T->idx[1]), n2 = fromf(s->nrm + 3u * T->idx[2]);
  v3 n = add(add(muls(n0, w.x), muls(n1, w.y)), muls(n2, w.z));
  if (!(dot(n, n) > 1e-12f)) n = cross(sub(T->b, T->a), sub(T->c, T->a));
  r.ok = 1;
  r.albedo[0] = tex[0]; r.albedo[1] = tex[1]; r.albedo[2] = tex[2];
  r.n = normalize3(n);
  r.toon = (m->flags & 4u) ? 1.0f : 0.0f;
  r.q = add(add(muls(T->a, w.x), muls(T->b, w.y)), muls(T->c, w.z));
  return r;
}

/* The triangle passes run on every host thread (orc_parallel).  Their writes commute: a mark sets EMPTY to MARK, an
 * occupancy word takes an OR, a representative the larger key, so atomics give the sequential result whatever the
 * order; the big-triangle lists are collected per chunk of threads and appended in chunk order, the sequential
 * loop's order. */
static void mark_brick(orc_vox *vx, uint32_t i) {
  uint32_t e = ORC_EMPTY;
  __atomic_compare_exchange_n(&vx->ptr[i], &e, ORC_MARK, 0, __ATOMIC_RELAXED, __ATOMIC_RELAXED);
}
static void atomic_max_u32(uint32_t *p, uint32_t v) {
  uint32_t cur = __atomic_load_n(p, __ATOMIC_RELAXED);
  while (cur < v && !__atomic_compare_exchange_n(p, &cur, v, 1, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {}
}

/* (triangle, level) pairs of one chunk of a triangle pass bound for the big lists */
typedef struct { uint32_t *t, n, cap; } biglist_t;
static void big_push(biglist_t *b, uint32_t t, uint32_t L) {
  if (b->n + 2u > b->cap) {
    b->cap = b->cap ? 2u * b->cap : 256u;
    b->t = (uint32_t *)realloc(b->t, (size_t)b->cap * 4u);
  }
  b->t[b->n++] = t; b->t[b->n++] = L;
}
/* appends the chunks' pairs in chunk order to the lists at big + (list0 + L) * cap, counting into hdr[cnt0 + L] */
static void big_merge(orc_vox *vx, biglist_t *ch, uint64_t nch, uint32_t list0, uint32_t cnt0) {
  const uint32_t cap = vx->big_cap;
  for (uint64_t c = 0; c < nch; c++) {
    for (uint32_t j = 0; j < ch[c].n; j += 2u) {
      uint32_t t = ch[c].t[j], L = ch[c].t[j + 1u];
      uint32_t k = vx->hdr[cnt0 + L]++;
      if (k < cap) vx->big[(list0 + L) * cap + k] = t; else vx->hdr[3]++;
    }
    free(ch[c].t);
  }
  free(ch);
}
#define TRI_GRAIN 512u

/* markRange (voxel.ts:348-358), all of the range's bricks */
static void mark_range(orc_vox *vx, const tri_t *T, uint32_t L, range_t r) {
  float bs = vox_size(vx, L) * 8.0f;
  v3 lo = region_lo(vx, L);
  uint32_t n = (uint32_t)(r.n.x * r.n.y * r.n.z);
  for (uint32_t j = 0; j < n; j++) {
    int32_t q = (int32_t)j;
    i3 b = I(r.lo.x + q % r.n.x, r.lo.y + (q / r.n.x) % r.n.y, r.lo.z + q / (r.n.x * r.n.y));
    if (!vx->coarse_from_triangles && finer_holds(vx, L, I(b.x * 8, b.y * 8, b.z * 8))
        && finer_holds(vx, L, I(b.x * 8 + 7, b.y * 8 + 7, b.z * 8 + 7))) continue;
    v3 c = add(lo, muls(adds(vi2f(b), 0.5f), bs));
    float hh = 0.5f * bs * 1.0001f;
    if (n == 1u || tri_box_v(c, V(hh, hh, hh), T)) mark_brick(vx, ptr_index(vx, L, b));
  }
}

/* voxelizeOne (voxel.ts:476-490) */
static void voxelize_one(const orc_scene *s, orc_vox *vx, const tri_t *T, uint32_t t, uint32_t L, i3 c, int single) {
  if (!vx->coarse_from_triangles && finer_built(vx, L, c)) return;
  float v = vox_size(vx, L);
  v3 p = add(region_lo(vx, L), muls(adds(vi2f(c), 0.5f), v));
  float hh = 0.5f * v * 1.0001f;
  if (!single && !tri_box_v(p, V(hh, hh, hh), T)) return;
  uint32_t ptr = vx->ptr[ptr_index(vx, L, ishr(c, 3))];
  if (ptr >= ORC_MARK) return;
  i3 l = I(c.x & 7, c.y & 7, c.z & 7);
  uint32_t bit = (uint32_t)(l.x + 8 * l.y + 64 * l.z);
  if (!surface_at(s, T, p, L, 0).ok) return;
  __atomic_fetch_or(&vx->occ[ptr * 16u + (bit >> 5)], 1u << (bit & 31u), __ATOMIC_RELAXED);
  atomic_max_u32(&vx->rep[ptr * 512u + bit], t + 1u);
}

typedef struct { const orc_scene *s; orc_vox *vx; biglist_t *ch; } tri_pass_t;

/* markBricks (voxel.ts:359-372) over threads [b, e) */
static void mark_pass(void *p, uint64_t b, uint64_t e) {
  tri_pass_t *j = (tri_pass_t *)p;
  orc_vox *vx = j->vx;
  biglist_t *bl = &j->ch[b / TRI_GRAIN];
  for (uint32_t i = (uint32_t)b; i < (uint32_t)e; i++) {
    uint32_t L0, t = work_at(j->s, i, &L0);
    tri_t T = load_tri(j->s, t);
    for (uint32_t L = L0; L < vx->levels; L++) {
      range_t r = vox_range(vx, &T, L, vox_size(vx, L) * 8.0f);
      int32_t n = r.n.x * r.n.y * r.n.z;
      if (n == 0 || (!vx->coarse_from_triangles && finer_holds_range(vx, L, r, 8))) continue;
      if (n > 8) { big_push(bl, t, L); continue; }
      mark_range(vx, &T, L, r);
    }
  }
}
/* markBricksBig (voxel.ts:374-387): item k of the concatenated lists of every level */
typedef struct { const orc_scene *s; orc_vox *vx; uint32_t list0, cnt0, off[9]; } big_pass_t;
static void big_item(const big_pass_t *j, uint32_t k, uint32_t *L, uint32_t *t) {
  uint32_t l = 0;
  while (k >= j->off[l + 1u]) l++;
  *L = l;
  *t = j->vx->big[(j->list0 + l) * j->vx->big_cap + (k - j->off[l])];
}
static void big_pass_init(big_pass_t *j, const orc_scene *s, orc_vox *vx, uint32_t list0, uint32_t cnt0) {
  j->s = s; j->vx = vx; j->list0 = list0; j->cnt0 = cnt0; j->off[0] = 0;
  for (uint32_t L = 0; L < 8; L++) {
    uint32_t n = L < vx->levels ? (vx->hdr[cnt0 + L] < vx->big_cap ? vx->hdr[cnt0 + L] : vx->big_cap) : 0u;
    j->off[L + 1u] = j->off[L] + n;
  }
}
static void mark_big_pass(void *p, uint64_t b, uint64_t e) {
  big_pass_t *j = (big_pass_t *)p;
  for (uint32_t k = (uint32_t)b; k < (uint32_t)e; k++) {
    uint32_t L, t;
    big_item(j, k, &L, &t);
    tri_t T = load_tri(j->s, t);
    mark_range(j->vx, &T, L, vox_range(j->vx, &T, L, vox_size(j->vx, L) * 8.0f));
  }
}
/* voxBits (voxel.ts:492-512) over threads [b, e) */
static void bits_pass(void *p, uint64_t b, uint64_t e) {
  tri_pass_t *j = (tri_pass_t *)p;
  orc_vox *vx = j->vx;
  biglist_t *bl = &j->ch[b / TRI_GRAIN];
  for (uint32_t i = (uint32_t)b; i < (uint32_t)e; i++) {
    uint32_t L0, t = work_at(j->s, i, &L0);
    tri_t T = load_tri(j->s, t);
    for (uint32_t L = L0; L < vx->levels; L++) {
      range_t r = vox_range(vx, &T, L, vox_size(vx, L));
      int32_t n = r.n.x * r.n.y * r.n.z;
      if (n == 0 || (!vx->coarse_from_triangles && finer_built_range(vx, L, r))) continue;
      if ((uint32_t)n > BIG) { big_push(bl, t, L); continue; }
      for (int32_t k = 0; k < n; k++)
        voxelize_one(j->s, vx, &T, t, L, I(r.lo.x + k % r.n.x, r.lo.y + (k / r.n.x) % r.n.y, r.lo.z + k / (r.n.x * r.n.y)), n == 1);
    }
  }
}
/* voxBitsBig (voxel.ts:514-534) */
static void bits_big_pass(void *p, uint64_t b, uint64_t e) {
  big_pass_t *j = (big_pass_t *)p;
  for (uint32_t k = (uint32_t)b; k < (uint32_t)e; k++) {
    uint32_t L, t;
    big_item(j, k, &L, &t);
    tri_t T = load_tri(j->s, t);
    range_t r = vox_range(j->vx, &T, L, vox_size(j->vx, L));
    int32_t n = r.n.x * r.n.y * r.n.z;
    for (int32_t q = 0; q < n; q++)
      voxelize_one(j->s, j->vx, &T, t, L, I(r.lo.x + q % r.n.x, r.lo.y + (q / r.n.x) % r.n.y, r.lo.z + q / (r.n.x * r.n.y)), 0);
  }
}
/* markParents (voxel.ts:390-403) over pointers [b, e) */
static void parents_pass(void *p, uint64_t b, uint64_t e) {
  orc_vox *vx = (orc_vox *)p;
  const uint32_t NL = vx->levels, G = vx->G, per = G * G * G;
  for (uint32_t i = (uint32_t)b; i < (uint32_t)e; i++) {
    if (__atomic_load_n(&vx->ptr[i], __ATOMIC_RELAXED) != ORC_MARK) continue;
    uint32_t L = i / per, r = i % per;
    i3 o = org(vx, L);
    i3 w = I(o.x + (int32_t)(r % G), o.y + (int32_t)((r / G) % G), o.z + (int32_t)(r / (G * G)));
    for (L++; L < NL; L++) {
      w = ishr(w, 1);
      i3 ol = org(vx, L);
      i3 bb = I(w.x - ol.x, w.y - ol.y, w.z - ol.z);
      if (bb.x < 0 || bb.y < 0 || bb.z < 0 || bb.x >= (int32_t)G || bb.y >= (int32_t)G || bb.z >= (int32_t)G) break;
      mark_brick(vx, ptr_index(vx, L, bb));
    }
  }
}

/* reduce of level L (voxel.ts:540-577) for the level L-1 bricks [b, e): their words ORed into the parents, the
 * representatives' maxima taken (atomics: OR and max commute) */
typedef struct { orc_vox *vx; uint32_t L; } reduce_job_t;
static void reduce_pass(void *p, uint64_t b0, uint64_t e0) {
  reduce_job_t *j = (reduce_job_t *)p;
  orc_vox *vx = j->vx;
  const uint32_t L = j->L;
  for (uint32_t ptr = (uint32_t)b0; ptr < (uint32_t)e0; ptr++) {
    uint32_t code = vx->code[ptr];
    uint32_t Lc = code >> 27;
    if (Lc + 1u != L) continue;
    for (uint32_t w = 0; w < 16; w++) {
      uint32_t word = __atomic_load_n(&vx->occ[ptr * 16u + w], __ATOMIC_RELAXED);
      if (word == 0u) continue;
      i3 b = I((int32_t)((code >> 18) & 511u), (int32_t)((code >> 9) & 511u), (int32_t)(code & 511u));
      i3 c0 = I(b.x * 8, b.y * 8 + (int32_t)((w & 1u) * 4u), b.z * 8 + (int32_t)(w >> 1));
      i3 oc = org(vx, Lc), ol = org(vx, L);
      i3 pc0 = I(((oc.x * 8 + c0.x) >> 1) - ol.x * 8, ((oc.y * 8 + c0.y) >> 1) - ol.y * 8, ((oc.z * 8 + c0.z) >> 1) - ol.z * 8);
      uint32_t pptr = vx->ptr[ptr_index(vx, L, ishr(pc0, 3))];
      if (pptr >= ORC_MARK) continue;
      i3 l0 = I(pc0.x & 7, pc0.y & 7, pc0.z & 7);
      uint32_t pbit0 = (uint32_t)(l0.x + 8 * l0.y + 64 * l0.z);
      uint32_t mask = 0, lo[4] = {0, 0, 0, 0}, hi[4] = {0, 0, 0, 0};
      while (word != 0u) {
        uint32_t k = (uint32_t)__builtin_ctz(word);
        word &= word - 1u;
        uint32_t px = (k & 7u) >> 1, py = k >> 4;
        mask |= 1u << ((pbit0 + px + 8u * py) & 31u);
        uint32_t rv = __atomic_load_n(&vx->rep[ptr * 512u + w * 32u + k], __ATOMIC_RELAXED);
        if (py == 0u) { if (rv > lo[px]) lo[px] = rv; } else { if (rv > hi[px]) hi[px] = rv; }
      }
      __atomic_fetch_or(&vx->occ[pptr * 16u + (pbit0 >> 5)], mask, __ATOMIC_RELAXED);
      for (uint32_t px = 0; px < 4; px++)
        for (uint32_t py = 0; py < 2; py++) {
          uint32_t rv = py == 0 ? lo[px] : hi[px];
          if (rv != 0u) atomic_max_u32(&vx->rep[pptr * 512u + pbit0 + px + 8u * py], rv);
        }
    }
  }
}

/* resolveAttr (voxel.ts:596-620) of the bricks [b0, e0) */
typedef struct { const orc_scene *s; orc_vox *vx; } resolve_job_t;
static void resolve_pass(void *p, uint64_t b0, uint64_t e0) {
  resolve_job_t *j = (resolve_job_t *)p;
  const orc_scene *s = j->s;
  orc_vox *vx = j->vx;
  for (uint32_t ptr = (uint32_t)b0; ptr < (uint32_t)e0; ptr++) {
    uint32_t first = vx->base[ptr];
    if (first == ORC_EMPTY) continue;
    uint32_t code = vx->code[ptr];
    uint32_t L = code >> 27;
    i3 b = I((int32_t)((code >> 18) & 511u), (int32_t)((code >> 9) & 511u), (int32_t)(code & 511u));
    uint32_t r = 0;
    for (uint32_t bit = 0; bit < 512u; bit++) {
      uint32_t word = vx->occ[ptr * 16u + (bit >> 5)];
      if ((word & (1u << (bit & 31u))) == 0u) continue;
      uint32_t ai = first + r++;
      i3 c = I(b.x * 8 + (int32_t)(bit & 7u), b.y * 8 + (int32_t)((bit >> 3) & 7u), b.z * 8 + (int32_t)(bit >> 6));
      v3 p = add(region_lo(vx, L), muls(adds(vi2f(c), 0.5f), vox_size(vx, L)));
      uint32_t rv = vx->rep[ptr * 512u + bit];
      if (rv == 0u || rv > key_limit(s)) {   /* no representative (cannot happen for a set bit): no attributes */
        for (int k = 0; k < 4; k++) vx->attr[ai * 4u + k] = 0u;
        vx->plane[ai] = 0.0f; vx->sunvis[ai] = 1.0f;
        continue;
      }
      tri_t T = load_tri(s, rv - 1u);
      surf_t sf = surface_at(s, &T, p, L, 1);
      float alb[4] = {sf.albedo[0], sf.albedo[1], sf.albedo[2], sf.toon};
      /* octEnc (voxel.ts:590-594) */
      v3 n = sf.n;
      float sa = fabsf(n.x) + fabsf(n.y) + fabsf(n.z);
      float px = n.x / sa, py = n.y / sa;
      if (n.z < 0.0f) {
        float ox = px, oy = py;
        px = (1.0f - fabsf(oy)) * (ox >= 0.0f ? 1.0f : -1.0f);
        py = (1.0f - fabsf(ox)) * (oy >= 0.0f ? 1.0f : -1.0f);
      }
      const orc_material *m = &s->mats[T.idx[3]];
      vx->attr[ai * 4u + 0] = orc_pack4x8unorm(alb);
      vx->attr[ai * 4u + 1] = orc_pack2x16snorm(px, py);
      vx->attr[ai * 4u + 2] = (uint32_t)orc_f32_to_f16(m->emissive[0]) | ((uint32_t)orc_f32_to_f16(m->emissive[1]) << 16);
      vx->attr[ai * 4u + 3] = (uint32_t)orc_f32_to_f16(m->emissive[2]);
      vx->plane[ai] = dot(sf.n, sub(sf.q, p));
      vx->sunvis[ai] = 1.0f;
    }
  }
}

void orc_vox_origins(float v0, uint32_t levels, uint32_t G, const double eye[3], int32_t origin_out[8][4]) {
  for (uint32_t L = 0; L < 8; L++) for (int a = 0; a < 4; a++) origin_out[L][a] = 0;
  for (uint32_t L = 0; L < levels; L++) {
    double bs = (double)v0 * ldexp(1.0, (int)L) * 8.0;   /* v0 * 2 ** L * 8 in the host's f64 */
    for (int a = 0; a < 3; a++) origin_out[L][a] = (int32_t)floor(eye[a] / bs) - (int32_t)(G / 2);
  }
}

int orc_vox_build(const orc_scene *s, orc_vox *vx) {
  const uint32_t NL = vx->levels, G = vx->G, per = G * G * G;
  /* clear (voxel.ts:338) */
  memset(vx->hdr, 0, ORC_HDR * 4);
  for (uint32_t i = 0; i < NL * per; i++) vx->ptr[i] = ORC_EMPTY;

  /* markBricks + markBricksBig (voxel.ts:359-387) */
  {
    uint32_t nt = threads_of(s);
    uint64_t nch = ((uint64_t)nt + TRI_GRAIN - 1u) / TRI_GRAIN;
    tri_pass_t j = {s, vx, (biglist_t *)calloc(nch ? nch : 1u, sizeof(biglist_t))};
    orc_parallel(nt, TRI_GRAIN, mark_pass, &j);
    big_merge(vx, j.ch, nch, 8u, 24u);
    big_pass_t bj;
    big_pass_init(&bj, s, vx, 8u, 24u);
    orc_parallel(bj.off[8], 64u, mark_big_pass, &bj);
  }
  /* markParents (voxel.ts:390-403) */
  orc_parallel((uint64_t)(NL - 1) * per, 4096u, parents_pass, vx);
  /* countMarks / scanMarks / allocBricks (voxel.ts:411-470), in the ordered form: coarse levels first, then pointer
   * index; a brick past the pool is dropped. */
  uint32_t marked = 0;
  for (uint32_t i = 0; i < NL * per; i++) marked += vx->ptr[i] == ORC_MARK;
  vx->hdr[5] = marked;
  vx->hdr[0] = marked;
  uint32_t idx = 0;
  for (uint32_t o = 0; o < NL * per; o++) {
    uint32_t L = NL - 1u - o / per, i = L * per + o % per;
    if (vx->ptr[i] != ORC_MARK) continue;
    uint32_t k = idx++;
    if (k >= vx->max_bricks) { vx->ptr[i] = ORC_DROP; vx->hdr[2]++; continue; }
    vx->hdr[8 + L]++;
    vx->ptr[i] = k;
    for (uint32_t w = 0; w < 16; w++) vx->occ[k * 16u + w] = 0;
    vx->base[k] = 0;
    uint32_t r = i % per;
    vx->code[k] = (L << 27) | ((r % G) << 18) | (((r / G) % G) << 9) | (r / (G * G));
  }
  uint32_t nb = marked < vx->max_bricks ? marked : vx->max_bricks;
  /* clearKeys */
  memset(vx->rep, 0, (size_t)nb * 512u * 4u);

  /* voxBits + voxBitsBig (voxel.ts:492-534) */
  {
    uint32_t nt = threads_of(s);
    uint64_t nch = ((uint64_t)nt + TRI_GRAIN - 1u) / TRI_GRAIN;
    tri_pass_t j = {s, vx, (biglist_t *)calloc(nch ? nch : 1u, sizeof(biglist_t))};
    orc_parallel(nt, TRI_GRAIN, bits_pass, &j);
    big_merge(vx, j.ch, nch, 0u, 16u);
    big_pass_t bj;
    big_pass_init(&bj, s, vx, 0u, 16u);
    orc_parallel(bj.off[8], 16u, bits_big_pass, &bj);
  }

  /* reduce, levels 1 .. NL-1 (voxel.ts:540-577), each level's bricks in parallel */
  if (!vx->coarse_from_triangles) {
    for (uint32_t L = 1; L < NL; L++) {
      reduce_job_t j = {vx, L};
      orc_parallel(nb, 64u, reduce_pass, &j);
    }
  }

  /* allocVoxels (voxel.ts:579-588), bases in brick order */
  uint32_t total = 0;
  for (uint32_t b = 0; b < nb; b++) {
    uint32_t n = 0;
    for (uint32_t w = 0; w < 16; w++) n += popc(vx->occ[b * 16u + w]);
    uint32_t first = total;
    total += n;
    if (first + n > vx->max_voxels) { vx->base[b] = ORC_EMPTY; vx->hdr[4]++; continue; }
    vx->base[b] = first;
  }
  vx->hdr[1] = total;

  /* resolveAttr (voxel.ts:596-620), bricks in parallel */
  {
    resolve_job_t j = {s, vx};
    orc_parallel(nb, 16u, resolve_pass, &j);
  }
  return 0;
}
