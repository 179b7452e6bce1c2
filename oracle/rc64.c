/* FP64 accuracy oracle of the merge and gather (test infrastructure only): mergeScreen (rc.ts:710-743),
 * projectSH (:752-774) and gatherScreen (:929-954, evalSH :819-829) evaluated in double precision from the traced
 * f32 intervals, with no intermediate rounding.  The error of the f32/f16/bf16 GPU atlases is stated against it. */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "gi_oracle.h"
#include "orc_par.h"

enum { F_IVP = 16, F_EYE = 80, F_FWD = 84, F_SKY = 96, F_SIZE = 100, F_OMEGA = 120 };

typedef struct { double x, y, z; } d3;
static inline d3 D(double x, double y, double z) { d3 r = {x, y, z}; return r; }
static inline double ddot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

static d3 world_at(const float *F, int px, int py, double d) {
  double nx = ((double)px + 0.5) * (double)F[F_SIZE + 2] * 2.0 - 1.0;
  double ny = 1.0 - ((double)py + 0.5) * (double)F[F_SIZE + 3] * 2.0;
  const float *m = F + F_IVP;
  double h[4];
  for (int i = 0; i < 4; i++) h[i] = (double)m[i] * nx + (double)m[4 + i] * ny + (double)m[8 + i] * d + (double)m[12 + i];
  return D(h[0] / h[3], h[1] / h[3], h[2] / h[3]);
}
static d3 dir_of(unsigned di, unsigned res) {
  double u = ((double)(di % res) + 0.5) / res, v = ((double)(di / res) + 0.5) / res;
  double fx = u * 2.0 - 1.0, fy = v * 2.0 - 1.0;
  d3 n = D(fx, fy, 1.0 - fabs(fx) - fabs(fy));
  double t = n.z < 0 ? -n.z : 0.0;
  n.x += n.x >= 0.0 ? -t : t;
  n.y += n.y >= 0.0 ? -t : t;
  double l = sqrt(ddot(n, n));
  return D(n.x / l, n.y / l, n.z / l);
}
static void sh_basis(d3 n, double y[9]) {
  y[0] = 0.282095; y[1] = 0.488603 * n.y; y[2] = 0.488603 * n.z; y[3] = 0.488603 * n.x;
  y[4] = 1.092548 * n.x * n.y; y[5] = 1.092548 * n.y * n.z; y[6] = 0.315392 * (3.0 * n.z * n.z - 1.0);
  y[7] = 1.092548 * n.x * n.z; y[8] = 0.546274 * (n.x * n.x - n.y * n.y);
}

typedef struct {
  const orc_layout *ly; const orc_gbuf *g; const orc_probe *probes; double *rad; double *sh; double *irr; unsigned c;
  unsigned f16;   /* cascades whose atlas storage is rounded to f16 */
} job64;

/* x rounded to the nearest f16 value, ties to even, as a double: 11 significant bits, a quantum of 2^-24 below 2^-14
 * (subnormals), infinity past 65504.  The scalings by powers of two are exact; nearbyint rounds half to even. */
static double as_f16(double x) {
  if (x != x || x == 0.0 || isinf(x)) return x;
  double a = fabs(x);
  int e;
  frexp(a, &e);                     /* a = m 2^e, m in [0.5, 1): the 11-bit significand's quantum is 2^(e - 11) */
  int q = e - 11 < -24 ? -24 : e - 11;
  double r = ldexp(nearbyint(ldexp(a, -q)), q);
  if (r > 65504.0) r = INFINITY;
  return x < 0.0 ? -r : r;
}

static void merge64(void *p, uint64_t b, uint64_t e) {
  job64 *j = (job64 *)p;
  const orc_layout *ly = j->ly;
  const float *F = j->g->frame;
  unsigned c = j->c, N = ly->cascades;
  const orc_casc *L = &ly->c[c];
  unsigned dirs = L->res * L->res;
  for (unsigned t = (unsigned)b; t < (unsigned)e; t++) {
    unsigned pi = t / dirs, di = t % dirs;
    double *rv = j->rad + 4u * ((size_t)L->rad_off + t);
    d3 up = D(F[F_SKY], F[F_SKY + 1], F[F_SKY + 2]);
    if (c + 1u < N && rv[3] > 0.0) {
      up = D(0, 0, 0);
      const orc_probe *pr = &j->probes[L->probe_off + pi];
      if (pr->pos[3] > 0.0f) {
        const orc_casc *U = &ly->c[c + 1u];
        double ux = (((double)(pi % L->tiles_x) + 0.5) * L->tile_size) / U->tile_size - 0.5;
        double uy = (((double)(pi / L->tiles_x) + 0.5) * L->tile_size) / U->tile_size - 0.5;
        int bx = (int)floor(ux), by = (int)floor(uy);
        double fx = ux - bx, fy = uy - by;
        unsigned u0 = di % L->res, v0 = di / L->res;
        d3 acc = D(0, 0, 0);
        double ws = 0.0;
        for (unsigned k = 0; k < 4; k++) {
          int ox = (int)(k & 1u), oy = (int)(k >> 1);
          int qx = bx + ox, qy = by + oy;
          qx = qx < 0 ? 0 : (qx > (int)U->tiles_x - 1 ? (int)U->tiles_x - 1 : qx);
          qy = qy < 0 ? 0 : (qy > (int)U->tiles_y - 1 ? (int)U->tiles_y - 1 : qy);
          unsigned qi = (unsigned)qy * U->tiles_x + (unsigned)qx;
          const orc_probe *qp = &j->probes[U->probe_off + qi];
          if (qp->pos[3] <= 0.0f) continue;
          double fwx = ox == 1 ? fx : 1.0 - fx, fwy = oy == 1 ? fy : 1.0 - fy;
          double rel = fabs((double)qp->nrm[3] - (double)pr->nrm[3]) / (double)pr->nrm[3];
          double w = (fwx * fwy + 1e-4) * (exp(-20.0 * rel) + 1e-4);
          d3 ua;
          if (U->res == L->res) {
            const double *q = j->rad + 4u * ((size_t)U->rad_off + qi * U->res * U->res + v0 * U->res + u0);
            ua = D(q[0], q[1], q[2]);
          } else {
            size_t base = (size_t)U->rad_off + qi * U->res * U->res + v0 * 2u * U->res + u0 * 2u;
            const double *a = j->rad + 4u * base, *bb = j->rad + 4u * (base + 1u), *cc = j->rad + 4u * (base + U->res),
                         *dd = j->rad + 4u * (base + U->res + 1u);
            ua = D(0.25 * (a[0] + bb[0] + cc[0] + dd[0]), 0.25 * (a[1] + bb[1] + cc[1] + dd[1]), 0.25 * (a[2] + bb[2] + cc[2] + dd[2]));
          }
          acc.x += w * ua.x; acc.y += w * ua.y; acc.z += w * ua.z;
          ws += w;
        }
        if (ws > 0.0) up = D(acc.x / ws, acc.y / ws, acc.z / ws);
      }
    }
    rv[0] = rv[0] + rv[3] * up.x; rv[1] = rv[1] + rv[3] * up.y; rv[2] = rv[2] + rv[3] * up.z; rv[3] = 1.0;
    if (c > 0u && ((j->f16 >> c) & 1u)) { rv[0] = as_f16(rv[0]); rv[1] = as_f16(rv[1]); rv[2] = as_f16(rv[2]); }
  }
}

static void sh64(void *p, uint64_t b, uint64_t e) {
  job64 *j = (job64 *)p;
  const float *F = j->g->frame;
  const orc_casc *L0 = &j->ly->c[0];
  const double PI = 3.14159265;
  for (unsigned pi = (unsigned)b; pi < (unsigned)e; pi++) {
    double cf[9][3];
    memset(cf, 0, sizeof cf);
    for (unsigned d = 0; d < 16; d++) {
      const double *rp = j->rad + 4u * ((size_t)L0->rad_off + pi * 16u + d);
      double y[9];
      sh_basis(dir_of(d, 4u), y);
      for (int k = 0; k < 9; k++)
        for (int i = 0; i < 3; i++) cf[k][i] += rp[i] * (double)F[F_OMEGA + d] * y[k];
    }
    for (int k = 0; k < 9; k++) {
      double a = k == 0 ? PI : (k < 4 ? 2.0 * PI / 3.0 : PI / 4.0);
      for (int i = 0; i < 3; i++) j->sh[27u * pi + 3u * (unsigned)k + (unsigned)i] = cf[k][i] * a;
    }
  }
}

static void gather64(void *p, uint64_t b, uint64_t e) {
  job64 *j = (job64 *)p;
  const orc_gbuf *g = j->g;
  const float *F = g->frame;
  const orc_casc *L0 = &j->ly->c[0];
  int W = (int)g->width;
  d3 eye = D(F[F_EYE], F[F_EYE + 1], F[F_EYE + 2]), fwd = D(F[F_FWD], F[F_FWD + 1], F[F_FWD + 2]);
  for (int py = (int)b; py < (int)e; py++)
    for (int px = 0; px < W; px++) {
      size_t q = (size_t)py * (size_t)W + (size_t)px;
      double *out = j->irr + 4u * q;
      double d = g->depth[q];
      if (!(d > 0.0)) { out[0] = out[1] = out[2] = out[3] = 0.0; continue; }
      d3 x = world_at(F, px, py, d);
      d3 n = D(g->normal[4 * q], g->normal[4 * q + 1], g->normal[4 * q + 2]);
      double z = ddot(D(x.x - eye.x, x.y - eye.y, x.z - eye.z), fwd);
      double ux = ((double)px + 0.5) / L0->tile_size - 0.5, uy = ((double)py + 0.5) / L0->tile_size - 0.5;
      int bx = (int)floor(ux), by = (int)floor(uy);
      double fx = ux - bx, fy = uy - by;
      double y[9];
      sh_basis(n, y);
      double acc[3] = {0, 0, 0}, ws = 0.0;
      for (unsigned k = 0; k < 4; k++) {
        int ox = (int)(k & 1u), oy = (int)(k >> 1);
        int qx = bx + ox, qy = by + oy;
        qx = qx < 0 ? 0 : (qx > (int)L0->tiles_x - 1 ? (int)L0->tiles_x - 1 : qx);
        qy = qy < 0 ? 0 : (qy > (int)L0->tiles_y - 1 ? (int)L0->tiles_y - 1 : qy);
        unsigned qi = (unsigned)qy * L0->tiles_x + (unsigned)qx;
        const orc_probe *pr = &j->probes[L0->probe_off + qi];
        if (pr->pos[3] <= 0.0f) continue;
        double fwx = ox == 1 ? fx : 1.0 - fx, fwy = oy == 1 ? fy : 1.0 - fy;
        double rel = fabs((double)pr->nrm[3] - z) / z;
        double nd = ddot(n, D(pr->nrm[0], pr->nrm[1], pr->nrm[2]));
        nd = nd > 0.0 ? nd : 0.0;
        double w = (fwx * fwy + 1e-4) * (exp(-20.0 * rel) + 1e-4) * (nd * nd * nd * nd + 1e-3);
        const double *sh = j->sh + 27u * qi;
        for (int i = 0; i < 3; i++) {
          double s = 0.0;
          for (int k2 = 0; k2 < 9; k2++) s += sh[3 * k2 + i] * y[k2];
          acc[i] += w * (s > 0.0 ? s : 0.0);
        }
        ws += w;
      }
      for (int i = 0; i < 3; i++) out[i] = ws > 0.0 ? acc[i] / ws : 0.0;
      out[3] = 1.0;
    }
}

int orc_rc_merge_gather_f64(const orc_layout *ly, const orc_gbuf *g, const orc_probe *probes, const float *rad_in,
                            double *irr_out) {
  return orc_rc_merge_gather_f64_rounded(ly, g, probes, rad_in, 0u, irr_out);
}

int orc_rc_merge_gather_f64_rounded(const orc_layout *ly, const orc_gbuf *g, const orc_probe *probes,
                                    const float *rad_in, unsigned f16_cascades, double *irr_out) {
  size_t nrad = 0;
  for (unsigned c = 0; c < ly->cascades; c++) {
    size_t end = (size_t)ly->c[c].rad_off + (size_t)ly->c[c].tiles_x * ly->c[c].tiles_y * ly->c[c].res * ly->c[c].res;
    if (end > nrad) nrad = end;
  }
  unsigned np0 = ly->c[0].tiles_x * ly->c[0].tiles_y;
  double *rad = (double *)malloc(nrad * 4 * sizeof(double));
  double *sh = (double *)malloc((size_t)np0 * 27 * sizeof(double));
  if (!rad || !sh) { free(rad); free(sh); return -1; }
  for (size_t i = 0; i < nrad * 4; i++) rad[i] = rad_in[i];
  for (unsigned c = 0; c < ly->cascades; c++) {
    if (!((f16_cascades >> c) & 1u)) continue;
    size_t a = 4u * (size_t)ly->c[c].rad_off;
    size_t n = 4u * (size_t)ly->c[c].tiles_x * ly->c[c].tiles_y * ly->c[c].res * ly->c[c].res;
    for (size_t i = a; i < a + n; i++) rad[i] = as_f16(rad[i]);
  }
  job64 j = {ly, g, probes, rad, sh, irr_out, 0, f16_cascades};
  for (int ci = (int)ly->cascades - 1; ci >= 0; ci--) {
    j.c = (unsigned)ci;
    const orc_casc *L = &ly->c[j.c];
    orc_parallel((uint64_t)L->tiles_x * L->tiles_y * L->res * L->res, 4096, merge64, &j);
  }
  orc_parallel(np0, 256, sh64, &j);
  orc_parallel(g->height, 4, gather64, &j);
  free(rad); free(sh);
  return 0;
}
