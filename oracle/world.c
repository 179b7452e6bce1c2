/*
 * World probes over the voxel tracer -- part of the CPU oracle (test infrastructure only; see gi_oracle.h).
 *
 * Restates the reference's method 'world' with the voxel world tracer (config tokens 'world-<P>-voxel[-vrel]'):
 *   hash32, lodFor, spacing, originOf, keyFor, insertKey, lookup      src/core/rc.ts:248-282
 *   relocate (G-buffer plane fit)                                      rc.ts:342-366
 *   voxCell, voxStoredNormal, voxOcc, cubeOff, relocateVox             rc.ts:379-470
 *   registerPixels, registerUp, compact, linkParents                   rc.ts:484-570
 *   trace (world probes) -> traceWorld                                 rc.ts:600-622, :216-245
 *   mergeWorld, projectSH + histBlend (the c0 history)                 rc.ts:688-708, :752-774, :779-816
 *   segOccluded, gatherWorld                                           rc.ts:854-927
 * and the pass order of Rc.encode (rc.ts:1180-1221).
 *
 * Choices where the reference leaves an order open (each is an order the reference can produce):
 *   - insertKey's table layout.  The reference's linear probing places colliding keys in the order its threads
 *     happen to insert them.  Here a larger key takes the slot of a smaller one and the smaller moves on (ordered
 *     linear probing, Amble & Knuth 1974): the layout is the one the reference gets when its keys arrive in
 *     decreasing order, whatever order they arrive in, so the CUDA path's concurrent inserts give the same table.
 *     A key is never stored 256 or more slots past its home slot (the reference's probe limit): such an insert
 *     fails and counts as a hash overflow (counts[16 + c]).
 *   - compact's probe order.  The reference numbers the keys by an atomic counter in thread order; here a key's
 *     probe index is the number of occupied slots before its slot.
 *   - lodFor's floor(log2(y)) is the exact binary exponent of the f32 y >= 1.
 * The c0 history keeps the SH as stored (f16 in the reference's format, f32 when the SH is kept in f32).
 * The toon receiving operator of gatherWorld (S3 style, albedo tag) is not part of this path: every pixel is
 * photoreal and gets alpha 1.
 */
#include <stdlib.h>
#include <string.h>

#include "orc_par.h"
#include "orc_rc.h"

#define W_NONE 0xffffffffu
#define W_HIST_W 0.5f

uint32_t orc_hash32(uint32_t x) {
  uint32_t h = x;
  h ^= h >> 16; h *= 0x7feb352du; h ^= h >> 15; h *= 0x846ca68bu; h ^= h >> 16;
  return h;
}

int32_t orc_lod_for(const float *F, float dist) {
  float y = fmaxf_(dist * F[F_RC + 1] * F[F_RC + 2] / F[F_RC], 1.0f);
  int32_t e = (int32_t)((ubits(y) >> 23) & 0xffu) - 127;
  return iclamp(e, 0, 14);
}

static float spacing(const float *F, int32_t lod, uint32_t c) { return scale2(F[F_RC], lod + (int32_t)c); }
static i3 origin_of(const float *F, float s) {
  i3 o = vf2i(vfloor(divs(fromf(F + F_EYE), s)));
  return I(o.x - 256, o.y - 256, o.z - 256);
}
static uint32_t key_for(const float *F, i3 g, int32_t lod, uint32_t c) {
  i3 o = origin_of(F, spacing(F, lod, c));
  i3 r = I(g.x - o.x, g.y - o.y, g.z - o.z);
  if (r.x < 0 || r.y < 0 || r.z < 0 || r.x >= 512 || r.y >= 512 || r.z >= 512) return W_NONE;
  return 0x80000000u | ((uint32_t)lod << 27) | ((uint32_t)r.x << 18) | ((uint32_t)r.y << 9) | (uint32_t)r.z;
}
static i3 corner(uint32_t k) { return I((int32_t)(k & 1u), (int32_t)((k >> 1) & 1u), (int32_t)((k >> 2) & 1u)); }

/* insertKey, ordered: returns 1 when the key could not be stored */
static int insert_key(uint32_t *keys, uint32_t mask, uint32_t key) {
  uint32_t h = orc_hash32(key) & mask;
  for (uint32_t it = 0; it <= mask + 256u; it++) {
    uint32_t cur = keys[h];
    if (cur == key) return 0;
    if (cur < key) {
      keys[h] = key;
      if (cur == 0u) return 0;
      key = cur;
    }
    h = (h + 1u) & mask;
    if (((h - (orc_hash32(key) & mask)) & mask) >= 256u) return 1;
  }
  return 1;
}
static uint32_t lookup(const orc_wlayout *wl, const uint32_t *keys, const uint32_t *slot_probe, uint32_t c, uint32_t key) {
  if (key == W_NONE) return W_NONE;
  uint32_t mask = wl->hash_mask[c], off = wl->hash_off[c];
  uint32_t h = orc_hash32(key) & mask;
  for (uint32_t i = 0; i < 256u; i++) {
    uint32_t cur = keys[off + h];
    if (cur == key) return slot_probe[off + h];
    if (cur == 0u) return W_NONE;
    h = (h + 1u) & mask;
  }
  return W_NONE;
}
static uint32_t probe_count(const orc_wlayout *wl, const uint32_t *counts, uint32_t c) {
  return counts[c] < wl->base.c[c].cap ? counts[c] : wl->base.c[c].cap;
}

/* F.viewProj * vec4(p, 1), column order */
static void clip4(const float *F, v3 p, float out[4]) {
  const float *m = F + F_VP;
  for (int i = 0; i < 4; i++) out[i] = m[i] * p.x + m[4 + i] * p.y + m[8 + i] * p.z + m[12 + i] * 1.0f;
}

/* relocate (rc.ts:345-366): plane fit to G-buffer samples within 1.5 spacings; n = 0 when nothing moved it */
static void relocate_gbuffer(const orc_gbuf *g, v3 p, float s, v3 *rp, v3 *rn) {
  const float *F = g->frame;
  *rp = p; *rn = V(0.0f, 0.0f, 0.0f);
  float c[4];
  clip4(F, p, c);
  if (c[3] <= F[F_EYE + 3]) return;
  float nx = c[0] / c[3], ny = c[1] / c[3];
  float cx = (nx * 0.5f + 0.5f) * F[F_SIZE], cy = (0.5f - ny * 0.5f) * F[F_SIZE + 1];
  float rpx = s / (c[3] * F[F_RC + 1]);
  v3 sn = V(0.0f, 0.0f, 0.0f);
  float se = 0.0f, cnt = 0.0f;
  int32_t W = (int32_t)g->width, H = (int32_t)g->height;
  for (uint32_t j = 0; j < 16u; j++) {
    float ox = ((float)(j % 4u) - 1.5f) / 1.5f * rpx, oy = ((float)(j / 4u) - 1.5f) / 1.5f * rpx;
    int32_t qx = f2i(floorf(cx + ox)), qy = f2i(floorf(cy + oy));
    if (qx < 0 || qy < 0 || qx >= W || qy >= H) continue;
    size_t q = (size_t)qy * (size_t)W + (size_t)qx;
    float d = g->depth[q];
    if (!(d > 0.0f)) continue;
    v3 x = world_at(F, qx, qy, d);
    if (length3(sub(x, p)) > 1.5f * s) continue;
    v3 n = V(g->normal[4 * q], g->normal[4 * q + 1], g->normal[4 * q + 2]);
    sn = add(sn, n);
    se += dot(n, sub(p, x)) / s;
    cnt += 1.0f;
  }
  if (cnt < 1.0f || length3(sn) < 0.3f * cnt) return;
  v3 m = normalize3(sn);
  float e = se / cnt;
  *rn = m;
  if (e < F[F_RC2]) *rp = add(p, muls(muls(m, F[F_RC2] - e), s));
}

/* voxCell (rc.ts:379-386): (brick, bit), brick ORC_MARK when empty or outside the level's window */
static void vox_cell(const orc_vox *vx, uint32_t L, v3 p, uint32_t out[2]) {
  float v = vox_size(vx, L);
  i3 c = vf2i(vfloor(divs(sub(p, muls(muls(vi2f(org(vx, L)), v), 8.0f)), v)));
  int32_t n8 = (int32_t)vx->G * 8;
  out[0] = ORC_MARK; out[1] = 0;
  if (c.x < 0 || c.y < 0 || c.z < 0 || c.x >= n8 || c.y >= n8 || c.z >= n8) return;
  uint32_t r[3];
  vox_at(vx, L, c, r);
  if (r[0] == ORC_EMPTY) return;
  out[0] = r[0]; out[1] = r[1];
}
static int vox_occ(const orc_vox *vx, uint32_t L, v3 p) {
  uint32_t r[2];
  vox_cell(vx, L, p, r);
  return r[0] != ORC_MARK;
}
/* voxStoredNormal (rc.ts:387-393); a voxel past the attribute pool has normal 0 */
static v3 vox_stored_normal(const orc_vox *vx, uint32_t brick, uint32_t bit) {
  if (vx->base[brick] == ORC_EMPTY) return V(0.0f, 0.0f, 0.0f);
  uint32_t w = vx->attr[vox_rank(vx, brick, bit) * 4u + 1u];
  float a = fmaxf_((float)(int16_t)(w & 0xffffu) / 32767.0f, -1.0f);
  float b = fmaxf_((float)(int16_t)(w >> 16) / 32767.0f, -1.0f);
  v3 n = V(a, b, 1.0f - fabsf(a) - fabsf(b));
  float q = fmaxf_(-n.z, 0.0f);
  n.x += n.x >= 0.0f ? -q : q;
  n.y += n.y >= 0.0f ? -q : q;
  return n;
}
static v3 cube_off(uint32_t k, float vg) {
  return muls(V((float)(k & 3u) - 1.5f, (float)((k >> 2) & 3u) - 1.5f, (float)(k >> 4) - 1.5f), vg);
}

/* relocateVox (rc.ts:414-470) of probe slot */
static void relocate_vox(const orc_vox *vx, const orc_wlayout *wl, const float *F, orc_probe *pr, uint32_t c) {
  i3 g = I(pr->grid[0], pr->grid[1], pr->grid[2]);
  int32_t lod = pr->grid[3];
  float s0 = spacing(F, lod, 0u);
  v3 p = muls(vi2f(g), spacing(F, lod, c));
  uint32_t L = vox_level_for(vx, vox_level(vx, &wl->base, s0, c), p);
  uint32_t Lg = vox_level_for(vx, L + 1u < vx->levels ? L + 1u : vx->levels - 1u, p);
  float vg = vox_size(vx, Lg);
  uint32_t cell[64][2];
  for (uint32_t k = 0; k < 64u; k++) vox_cell(vx, Lg, add(p, cube_off(k, vg)), cell[k]);
  v3 grad = V(0.0f, 0.0f, 0.0f);
  float cnt = 0.0f;
  for (uint32_t k = 0; k < 64u; k++) {
    if (cell[k][0] == ORC_MARK) continue;
    grad = sub(grad, cube_off(k, vg));
    cnt += 1.0f;
  }
  v3 dir = grad;
  uint32_t flag = cnt < 1.0f ? 0u : (length3(grad) < 0.1f * cnt * vg ? 1u : 2u);
  if (flag == 1u) {
    v3 n = V(0.0f, 0.0f, 0.0f);
    for (uint32_t k = 0; k < 64u; k++)
      if (cell[k][0] != ORC_MARK) n = add(n, vox_stored_normal(vx, cell[k][0], cell[k][1]));
    dir = n;
  }
  if (flag != 0u) {
    if (length3(dir) < 1e-4f) flag = 0u; else { dir = normalize3(dir); flag = 2u; }
  }
  if (flag == 0u) {
    pr->nrm[0] = pr->nrm[1] = pr->nrm[2] = 0.0f; pr->nrm[3] = view_z(F, p);
    pr->pos[0] = p.x; pr->pos[1] = p.y; pr->pos[2] = p.z; pr->pos[3] = s0;
    return;
  }
  v3 n = dir;
  float s = s0 * exp2_((float)c);
  float back = F[F_RC2] * s;
  float stp = fmaxf_(0.5f * vox_size(vx, L), 1.5f * s / 16.0f);
  v3 r = p;
  for (uint32_t i = 0; i <= 16u; i++) {
    if ((float)i * stp > 1.5f * s) break;
    v3 q = add(p, muls(n, (float)i * stp));
    if (!vox_occ(vx, L, q) && !vox_occ(vx, L, sub(q, muls(n, back)))) { r = q; break; }
  }
  pr->pos[0] = r.x; pr->pos[1] = r.y; pr->pos[2] = r.z; pr->pos[3] = s0;
  pr->nrm[0] = n.x; pr->nrm[1] = n.y; pr->nrm[2] = n.z; pr->nrm[3] = view_z(F, r);
}

/* the segment test of linkParents and segOccluded (rc.ts:553-558, 854-878): any of min(ceil(|b - a| / v), 16)
 * samples occupied at level L */
static int seg_occluded(const orc_vox *vx, v3 a, v3 b, uint32_t L) {
  v3 d = sub(b, a);
  float kf = fminf_(ceilf(length3(d) / vox_size(vx, L)), 16.0f);
  uint32_t k = (uint32_t)kf;
  for (uint32_t i = 0; i < k; i++)
    if (vox_occ(vx, L, add(a, muls(d, ((float)i + 0.5f) / (float)k)))) return 1;
  return 0;
}

typedef struct {
  const ctx_t *cx; const orc_wlayout *wl; const orc_gbuf *g; orc_wstate *ws; orc_rc_out *o; uint32_t c;
  uint32_t n_traces, n_steps, n_cap;
} wjob;

static void w_trace_range(void *p, uint64_t b, uint64_t e) {
  wjob *j = (wjob *)p;
  const orc_vox *vx = j->cx->vx;
  const orc_layout *ly = &j->wl->base;
  orc_rc_out *o = j->o;
  const orc_casc *L = &ly->c[j->c];
  uint32_t dirs = L->res * L->res;
  uint32_t n_traces = 0, n_steps = 0, n_cap = 0;
  for (uint32_t t = (uint32_t)b; t < (uint32_t)e; t++) {
    uint32_t pi = t / dirs, di = t % dirs;
    const orc_probe *pr = &o->probes[L->probe_off + pi];
    trace_t tr;
    memset(&tr, 0, sizeof tr);
    tr.T = 1.0f; tr.lvl = ORC_EMPTY; tr.ptr = ORC_EMPTY;
    if (pr->pos[3] > 0.0f) {
      v3 dir = dir_of(di, L->res);
      float s0 = pr->pos[3];
      float t0 = L->b0 * s0, t1 = L->b1 * s0;
      v3 po = V(pr->pos[0], pr->pos[1], pr->pos[2]);
      v3 pn = V(pr->nrm[0], pr->nrm[1], pr->nrm[2]);
      uint32_t Lv = vox_level_for(vx, vox_level(vx, ly, s0, j->c), add(po, muls(dir, t1)));
      float v = vox_size(vx, Lv);
      v3 ooff = add(po, muls(pn, ly->vox_offset * v));
      trace_vox(j->cx, ooff, dir, t0, t1, ly->vox_skip * v, Lv, ly->dda_cap, &tr);
      dyn_compose(vx, po, dir, t0, t1, ooff, 3.5449077f / (float)L->res, &tr);
      n_traces += 1;
      n_steps += tr.steps;
      n_cap += tr.steps >= ly->dda_cap ? 1u : 0u;
    }
    float *r = o->rad + 4u * ((size_t)L->rad_off + t);
    r[0] = round_store(tr.r, ly->atlas); r[1] = round_store(tr.g, ly->atlas);
    r[2] = round_store(tr.b, ly->atlas); r[3] = round_store(tr.T, ly->atlas);
    if (o->hit) {
      uint32_t *h = o->hit + 4u * ((size_t)L->rad_off + t);
      h[0] = tr.lvl; h[1] = tr.ptr; h[2] = tr.bit; h[3] = tr.tin;
    }
  }
  __atomic_fetch_add(&j->n_traces, n_traces, __ATOMIC_RELAXED);
  __atomic_fetch_add(&j->n_steps, n_steps, __ATOMIC_RELAXED);
  __atomic_fetch_add(&j->n_cap, n_cap, __ATOMIC_RELAXED);
}

/* mergeWorld (rc.ts:688-708), cascade j->c in place */
static void w_merge_range(void *p, uint64_t b, uint64_t e) {
  wjob *j = (wjob *)p;
  const orc_layout *ly = &j->wl->base;
  orc_rc_out *o = j->o;
  const float *F = j->g->frame;
  uint32_t c = j->c, N = ly->cascades;
  const orc_casc *L = &ly->c[c];
  uint32_t dirs = L->res * L->res;
  for (uint32_t t = (uint32_t)b; t < (uint32_t)e; t++) {
    uint32_t pi = t / dirs, di = t % dirs;
    float *rv = o->rad + 4u * ((size_t)L->rad_off + t);
    v3 up = fromf(F + F_SKY);
    if (c + 1u < N && rv[3] > 0.0f) {
      v3 acc = V(0.0f, 0.0f, 0.0f);
      float ws = 0.0f;
      for (uint32_t k = 0; k < 8u; k++) {
        uint32_t q = j->ws->parents[(size_t)(L->probe_off + pi) * 8u + k];
        if (q == W_NONE) continue;
        acc = add(acc, upper_avg(ly, o->rad, c + 1u, q, di % L->res, di / L->res, L->res));
        ws += 1.0f;
      }
      up = ws > 0.0f ? divs(acc, fmaxf_(ws, 1.0f)) : V(0.0f, 0.0f, 0.0f);
    }
    v3 m = fmas(up, rv[3], V(rv[0], rv[1], rv[2]));
    rv[0] = round_store(m.x, ly->atlas); rv[1] = round_store(m.y, ly->atlas); rv[2] = round_store(m.z, ly->atlas);
    rv[3] = round_store(1.0f, ly->atlas);
  }
}

static uint32_t hist_hash(i3 g, int32_t lod) {
  return orc_hash32(((uint32_t)g.x * 73856093u) ^ ((uint32_t)g.y * 19349663u) ^ ((uint32_t)g.z * 83492791u) ^
                    ((uint32_t)lod * 2654435761u));
}

/* projectSH (rc.ts:752-774) with histBlend (rc.ts:787-812), sequential in probe order */
static void w_project_sh(const orc_wlayout *wl, const orc_gbuf *g, orc_wstate *ws, orc_rc_out *o) {
  const orc_layout *ly = &wl->base;
  const float *F = g->frame;
  const orc_casc *L0 = &ly->c[0];
  uint32_t n = probe_count(wl, o->counts, 0);
  uint32_t H = wl->hash_mask[0] + 1u, cap = L0->cap;
  uint32_t cur = ws->hist_par, prv = 1u - cur;
  uint32_t fmt = ly->f32_out ? 0u : ly->atlas;
  float a_k[3] = {PI_F, 2.0f * PI_F / 3.0f, PI_F / 4.0f};
  for (uint32_t pi = 0; pi < n; pi++) {
    v3 cf[9];
    for (int k = 0; k < 9; k++) cf[k] = V(0.0f, 0.0f, 0.0f);
    for (uint32_t d = 0; d < 16; d++) {
      const float *rp = o->rad + 4u * ((size_t)L0->rad_off + pi * 16u + d);
      v3 r = muls(V(rp[0], rp[1], rp[2]), F[F_OMEGA + d]);
      float y[9];
      sh_basis(dir_of(d, 4u), y);
      for (int k = 0; k < 9; k++) cf[k] = fmas(r, y[k], cf[k]);
    }
    float v[32];
    for (int k = 0; k < 32; k++) v[k] = 0.0f;
    for (int k = 0; k < 9; k++) {
      float a = k == 0 ? a_k[0] : (k < 4 ? a_k[1] : a_k[2]);
      v[k * 3 + 0] = cf[k].x * a; v[k * 3 + 1] = cf[k].y * a; v[k * 3 + 2] = cf[k].z * a;
    }
    /* histBlend */
    const orc_probe *pr = &o->probes[L0->probe_off + pi];
    i3 gg = I(pr->grid[0], pr->grid[1], pr->grid[2]);
    int32_t lod = pr->grid[3];
    uint32_t h0 = hist_hash(gg, lod) & (H - 1u), h = h0, found = W_NONE;
    for (uint32_t i = 0; i < 64u; i++) {
      uint32_t sl = ws->hist_tab[prv * H + h];
      if (sl == 0u) break;
      const int32_t *og = ws->hist_grid + ((size_t)prv * cap + (sl - 1u)) * 4u;
      if (og[0] == gg.x && og[1] == gg.y && og[2] == gg.z && og[3] == lod) { found = sl - 1u; break; }
      h = (h + 1u) & (H - 1u);
    }
    if (found != W_NONE) {
      const float *hs = ws->hist_sh + ((size_t)prv * cap + found) * 32u;
      for (int k = 0; k < 32; k++) v[k] = hs[k] * (1.0f - W_HIST_W) + v[k] * W_HIST_W;
    }
    int32_t *og = ws->hist_grid + ((size_t)cur * cap + pi) * 4u;
    og[0] = gg.x; og[1] = gg.y; og[2] = gg.z; og[3] = lod;
    h = h0;
    for (uint32_t i = 0; i < 64u; i++) {
      if (ws->hist_tab[cur * H + h] == 0u) { ws->hist_tab[cur * H + h] = pi + 1u; break; }
      h = (h + 1u) & (H - 1u);
    }
    float *sh = o->sh + 32u * pi;
    float *hs = ws->hist_sh + ((size_t)cur * cap + pi) * 32u;
    for (int k = 0; k < 32; k++) { sh[k] = k < 27 ? round_store(v[k], fmt) : 0.0f; hs[k] = sh[k]; }
  }
}

static v3 eval_sh(const float *sh, const float y[9]) {
  v3 es = V(0.0f, 0.0f, 0.0f);
  for (int k = 0; k < 9; k++) es = fmas(V(sh[3 * k], sh[3 * k + 1], sh[3 * k + 2]), y[k], es);
  return vmax(es, V(0.0f, 0.0f, 0.0f));
}

/* gatherWorld (rc.ts:880-927), rows [b, e) */
/* toonReceive (style.ts:30-42): ambient from L0, the dominant direction d from the luminance gradient of L1 and its
 * directional colour, the direction through a two-band ramp (smoothstep of half width soft, or a step) */
typedef struct { v3 e; float band, contrast; } toon_recv;
static toon_recv toon_receive(v3 c0, v3 c1y, v3 c1z, v3 c1x, v3 n, float soft) {
  const v3 lw = V(0.2126f, 0.7152f, 0.0722f);
  v3 amb = muls(c0, 0.282095f);
  v3 g = V(dot(c1x, lw), dot(c1y, lw), dot(c1z, lw));
  float gl = length3(g);
  toon_recv out;
  if (gl < 1e-6f) {
    out.e = V(fmaxf_(amb.x, 0.0f), fmaxf_(amb.y, 0.0f), fmaxf_(amb.z, 0.0f));
    out.band = 0.0f; out.contrast = 0.0f;
    return out;
  }
  v3 d = divs(g, gl);
  v3 s = add(add(muls(c1x, d.x), muls(c1y, d.y)), muls(c1z, d.z));
  v3 dir = muls(s, 0.488603f);
  dir = V(fmaxf_(dir.x, 0.0f), fmaxf_(dir.y, 0.0f), fmaxf_(dir.z, 0.0f));
  float x = dot(n, d), ramp;
  if (soft > 0.0f) {
    float t = fminf_(fmaxf_((x - -soft) / (soft - -soft), 0.0f), 1.0f);
    ramp = t * t * (3.0f - 2.0f * t);
  } else {
    ramp = x > 0.0f ? 1.0f : 0.0f;
  }
  v3 e = add(sub(amb, dir), muls(muls(dir, 2.0f), ramp));
  out.e = V(fmaxf_(e.x, 0.0f), fmaxf_(e.y, 0.0f), fmaxf_(e.z, 0.0f));
  out.band = x > 0.0f ? 1.0f : 0.0f;
  out.contrast = dot(dir, lw) / fmaxf_(dot(amb, lw), 1e-6f);
  return out;
}

/* toonReceive on c = (c0, c1y, c1z, c1x) as 12 floats: out = (E rgb, band, contrast) */
void orc_toon_receive(const float c[12], const float n[3], float soft, float out[5]) {
  toon_recv r = toon_receive(V(c[0], c[1], c[2]), V(c[3], c[4], c[5]), V(c[6], c[7], c[8]), V(c[9], c[10], c[11]),
                             V(n[0], n[1], n[2]), soft);
  out[0] = r.e.x; out[1] = r.e.y; out[2] = r.e.z; out[3] = r.band; out[4] = r.contrast;
}

/* shL1 + shAdd (rc.ts:831-840): the L0 and L1 coefficients (basis order 0, y, z, x) of a stored SH, added with
 * weight w */
static void sh_l1_add(const float *sh, float w, v3 acc[4]) {
  for (int k = 0; k < 4; k++) acc[k] = fmas(V(sh[3 * k], sh[3 * k + 1], sh[3 * k + 2]), w, acc[k]);
}

static void w_gather_range(void *p, uint64_t b, uint64_t e) {
  wjob *j = (wjob *)p;
  const orc_wlayout *wl = j->wl;
  const orc_layout *ly = &wl->base;
  const orc_gbuf *g = j->g;
  orc_rc_out *o = j->o;
  const orc_vox *vx = j->cx->vx;
  const float *F = g->frame;
  int32_t W = (int32_t)g->width;
  uint32_t out_fmt = ((ly->atlas == 0 || ly->f32_out) && !ly->irr_f16) ? 0u : 1u;
  for (int32_t py = (int32_t)b; py < (int32_t)e; py++)
    for (int32_t px = 0; px < W; px++) {
      size_t q = (size_t)py * (size_t)W + (size_t)px;
      float *out = o->irr + 4u * q;
      float d = g->depth[q];
      if (!(d > 0.0f)) { out[0] = out[1] = out[2] = out[3] = 0.0f; continue; }
      v3 x = world_at(F, px, py, d);
      v3 n = V(g->normal[4 * q], g->normal[4 * q + 1], g->normal[4 * q + 2]);
      int32_t lod = orc_lod_for(F, length3(sub(x, fromf(F + F_EYE))));
      float s0 = spacing(F, lod, 0u);
      v3 gp = divs(x, s0);
      i3 bb = vf2i(vfloor(gp));
      v3 f = sub(gp, vi2f(bb));
      uint32_t Lo = vox_level_for(vx, vox_level(vx, ly, s0, 0u), x);
      v3 xo1 = add(x, muls(n, 1.0f * vox_size(vx, Lo)));
      float y[9];
      sh_basis(n, y);
      v3 acc = V(0.0f, 0.0f, 0.0f);
      float ws = 0.0f, ww[8];
      uint32_t hidden = 0, qq[8];
      /* the G-buffer's style tag (rc.ts:881-883): toon pixels also interpolate L0 / L1 */
      float tagA = g->tag ? (float)g->tag[q] / 255.0f : 0.0f;
      int toon = tagA > 0.75f;
      v3 l1[4] = {V(0.0f, 0.0f, 0.0f), V(0.0f, 0.0f, 0.0f), V(0.0f, 0.0f, 0.0f), V(0.0f, 0.0f, 0.0f)};
      for (uint32_t k = 0; k < 8u; k++) {
        i3 oo = corner(k);
        uint32_t qi = lookup(wl, j->ws->keys, j->ws->slot_probe, 0u, key_for(F, I(bb.x + oo.x, bb.y + oo.y, bb.z + oo.z), lod, 0u));
        if (qi == W_NONE) continue;
        v3 tw = V(oo.x == 1 ? f.x : 1.0f - f.x, oo.y == 1 ? f.y : 1.0f - f.y, oo.z == 1 ? f.z : 1.0f - f.z);
        const orc_probe *pr = &o->probes[ly->c[0].probe_off + qi];
        v3 pp = fromf(pr->pos);
        v3 dv = sub(pp, x);
        float side = dot(n, dv) / fmaxf_(length3(dv), 1e-5f);
        float w = (tw.x * tw.y * tw.z + 1e-4f) * ((side + 1.0f) * (side + 1.0f) * 0.25f + 0.02f);
        if (wl->relocate == 2u && seg_occluded(vx, xo1, pp, Lo)) { hidden |= 1u << k; ww[k] = w; qq[k] = qi; continue; }
        acc = fmas(eval_sh(o->sh + 32u * qi, y), w, acc);
        ws += w;
        if (toon) sh_l1_add(o->sh + 32u * qi, w, l1);
      }
      if (ws <= 0.0f && hidden != 0u) {
        v3 xo2 = add(x, muls(n, 2.0f * vox_size(vx, Lo)));
        for (uint32_t k = 0; k < 8u; k++) {
          if ((hidden & (1u << k)) == 0u) continue;
          const orc_probe *pr = &o->probes[ly->c[0].probe_off + qq[k]];
          if (seg_occluded(vx, xo2, fromf(pr->pos), Lo)) continue;
          acc = fmas(eval_sh(o->sh + 32u * qq[k], y), ww[k], acc);
          ws += ww[k];
          if (toon) sh_l1_add(o->sh + 32u * qq[k], ww[k], l1);
        }
      }
      if (ws <= 0.0f && hidden != 0u && tagA <= 0.25f) __atomic_fetch_add(&o->counts[72 + (px & 7)], 1u, __ATOMIC_RELAXED);
      v3 r = ws > 0.0f ? divs(acc, ws) : V(0.0f, 0.0f, 0.0f);
      /* alpha (rc.ts:916-925): 1 photoreal; toon 2 + band + 2 when the directional part is at least a tenth of the
       * ambient (the receiving operator's irradiance replacing the physical one when style.y > 0.5); other tagged
       * pixels 2 */
      float alpha = 1.0f;
      if (toon && ws > 0.0f) {
        float iw = 1.0f / ws;
        toon_recv tr = toon_receive(muls(l1[0], iw), muls(l1[1], iw), muls(l1[2], iw), muls(l1[3], iw), n, F[F_STYLE + 2]);
        if (F[F_STYLE + 1] > 0.5f) r = tr.e;
        alpha = 2.0f + tr.band + (tr.contrast >= 0.1f ? 2.0f : 0.0f);
      } else if (toon || tagA > 0.25f) {
        alpha = 2.0f;
      }
      out[0] = out_fmt ? round_store(r.x, 1) : r.x;
      out[1] = out_fmt ? round_store(r.y, 1) : r.y;
      out[2] = out_fmt ? round_store(r.z, 1) : r.z;
      out[3] = out_fmt ? round_store(alpha, 1) : alpha;
    }
}

int orc_world_solve(const orc_vox *vx, const orc_wlayout *wl, const orc_gbuf *g, orc_wstate *ws, orc_rc_out *o) {
  const orc_layout *ly = &wl->base;
  const float *F = g->frame;
  ctx_t cx = {vx, F, {F[F_SKY], F[F_SKY + 1], F[F_SKY + 2]}, NULL, NULL};
  uint32_t N = ly->cascades;
  int32_t W = (int32_t)g->width, H = (int32_t)g->height;
  /* the c0 history's parity flips every solve (Rc.encode, rc.ts:1180); clearHist empties this solve's table */
  ws->hist_par = 1u - ws->hist_par;
  uint32_t H0 = wl->hash_mask[0] + 1u;
  memset(ws->hist_tab + (size_t)ws->hist_par * H0, 0, H0 * 4u);
  /* clearKeys */
  memset(o->counts, 0, 80 * 4);
  memset(ws->keys, 0, (size_t)wl->hash_total * 4u);
  /* registerPixels (rc.ts:484-500) */
  uint32_t st = ((const uint32_t *)F)[F_RU + 2];
  if (st < 1u) st = 1u;
  uint32_t sx = ((uint32_t)W + st - 1u) / st, sy = ((uint32_t)H + st - 1u) / st;
  for (uint32_t i = 0; i < sx * sy; i++) {
    int32_t px = (int32_t)((i % sx) * st + st / 2u), py = (int32_t)((i / sx) * st + st / 2u);
    if (px >= W || py >= H) continue;
    float d = g->depth[(size_t)py * (size_t)W + (size_t)px];
    if (!(d > 0.0f)) continue;
    v3 x = world_at(F, px, py, d);
    int32_t lod = orc_lod_for(F, length3(sub(x, fromf(F + F_EYE))));
    i3 b = vf2i(vfloor(divs(x, spacing(F, lod, 0u))));
    for (uint32_t k = 0; k < 8u; k++) {
      i3 oo = corner(k);
      uint32_t key = key_for(F, I(b.x + oo.x, b.y + oo.y, b.z + oo.z), lod, 0u);
      if (key != W_NONE && insert_key(ws->keys + wl->hash_off[0], wl->hash_mask[0], key)) o->counts[16]++;
    }
  }
  for (uint32_t c = 0; c < N; c++) {
    const orc_casc *L = &ly->c[c];
    if (c > 0) {
      /* registerUp (rc.ts:503-518) */
      const orc_casc *Lb = &ly->c[c - 1u];
      uint32_t nb = probe_count(wl, o->counts, c - 1u);
      for (uint32_t t = 0; t < nb; t++) {
        const orc_probe *pr = &o->probes[Lb->probe_off + t];
        i3 gg = I(pr->grid[0], pr->grid[1], pr->grid[2]);
        i3 lo = I(gg.x >> 1, gg.y >> 1, gg.z >> 1);
        int odd[3] = {(gg.x & 1) != 0, (gg.y & 1) != 0, (gg.z & 1) != 0};
        for (uint32_t k = 0; k < 8u; k++) {
          i3 oo = corner(k);
          if ((oo.x > 0 && !odd[0]) || (oo.y > 0 && !odd[1]) || (oo.z > 0 && !odd[2])) continue;
          uint32_t key = key_for(F, I(lo.x + oo.x, lo.y + oo.y, lo.z + oo.z), pr->grid[3], c);
          if (key != W_NONE && insert_key(ws->keys + wl->hash_off[c], wl->hash_mask[c], key)) o->counts[16 + c]++;
        }
      }
    }
    /* compact (rc.ts:520-537): probe index = occupied slots before the key's slot */
    uint32_t idx = 0;
    for (uint32_t h = 0; h <= wl->hash_mask[c]; h++) {
      uint32_t key = ws->keys[wl->hash_off[c] + h];
      if (key == 0u) continue;
      uint32_t id = idx++;
      if (id >= L->cap) { ws->slot_probe[wl->hash_off[c] + h] = W_NONE; o->counts[8 + c]++; continue; }
      ws->slot_probe[wl->hash_off[c] + h] = id;
      int32_t lod = (int32_t)((key >> 27) & 15u);
      i3 rel = I((int32_t)((key >> 18) & 511u), (int32_t)((key >> 9) & 511u), (int32_t)(key & 511u));
      float s = spacing(F, lod, c);
      i3 oo = origin_of(F, s);
      i3 gg = I(rel.x + oo.x, rel.y + oo.y, rel.z + oo.z);
      v3 pp = muls(vi2f(gg), s), rp = pp, rn = V(0.0f, 0.0f, 0.0f);
      if (wl->relocate == 0u) relocate_gbuffer(g, pp, s, &rp, &rn);
      orc_probe *pr = &o->probes[L->probe_off + id];
      pr->pos[0] = rp.x; pr->pos[1] = rp.y; pr->pos[2] = rp.z; pr->pos[3] = spacing(F, lod, 0u);
      pr->nrm[0] = rn.x; pr->nrm[1] = rn.y; pr->nrm[2] = rn.z; pr->nrm[3] = view_z(F, rp);
      pr->grid[0] = gg.x; pr->grid[1] = gg.y; pr->grid[2] = gg.z; pr->grid[3] = lod;
    }
    o->counts[c] = idx;
    uint32_t n = probe_count(wl, o->counts, c);
    if (wl->relocate == 2u)
      for (uint32_t pi = 0; pi < n; pi++) relocate_vox(vx, wl, F, &o->probes[L->probe_off + pi], c);
    if (c > 0) {
      /* linkParents (rc.ts:541-567) of cascade c - 1 */
      const orc_casc *Lb = &ly->c[c - 1u];
      uint32_t nb = probe_count(wl, o->counts, c - 1u);
      for (uint32_t pi = 0; pi < nb; pi++) {
        const orc_probe *pr = &o->probes[Lb->probe_off + pi];
        i3 gg = I(pr->grid[0], pr->grid[1], pr->grid[2]);
        int odd[3] = {(gg.x & 1) != 0, (gg.y & 1) != 0, (gg.z & 1) != 0};
        for (uint32_t k = 0; k < 8u; k++) {
          i3 oo = corner(k);
          uint32_t q = W_NONE;
          if (!((oo.x > 0 && !odd[0]) || (oo.y > 0 && !odd[1]) || (oo.z > 0 && !odd[2])))
            q = lookup(wl, ws->keys, ws->slot_probe, c,
                       key_for(F, I((gg.x >> 1) + oo.x, (gg.y >> 1) + oo.y, (gg.z >> 1) + oo.z), pr->grid[3], c));
          if (q != W_NONE && wl->relocate == 2u) {
            uint32_t Lv = vox_level_for(vx, vox_level(vx, ly, pr->pos[3], c - 1u), fromf(pr->pos));
            if (seg_occluded(vx, fromf(pr->pos), fromf(o->probes[L->probe_off + q].pos), Lv)) q = W_NONE;
          }
          ws->parents[(size_t)(Lb->probe_off + pi) * 8u + k] = q;
        }
      }
    }
  }
  /* trace (rc.ts:600-622), every cascade */
  wjob j = {&cx, wl, g, ws, o, 0, 0, 0, 0};
  for (uint32_t c = 0; c < N; c++) {
    const orc_casc *L = &ly->c[c];
    j.c = c; j.n_traces = j.n_steps = j.n_cap = 0;
    orc_parallel((uint64_t)probe_count(wl, o->counts, c) * L->res * L->res, 512, w_trace_range, &j);
    if (ly->stats > 0) { o->counts[24 + c] = j.n_traces; o->counts[32 + c] = j.n_steps; o->counts[64 + c] = j.n_cap; }
  }
  /* mergeWorld N-1 .. 0, projectSH with the history, gatherWorld */
  for (int32_t ci = (int32_t)N - 1; ci >= 0; ci--) {
    j.c = (uint32_t)ci;
    const orc_casc *L = &ly->c[j.c];
    orc_parallel((uint64_t)probe_count(wl, o->counts, j.c) * L->res * L->res, 4096, w_merge_range, &j);
  }
  w_project_sh(wl, g, ws, o);
  orc_parallel(g->height, 4, w_gather_range, &j);
  return 0;
}
