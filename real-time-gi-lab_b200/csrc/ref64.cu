// FP64 reference of the merge, SH projection and gather: the accuracy yardstick of the f32/f16/bf16 atlases.
//
// mergeScreen (rc.ts:710-743), projectSH (rc.ts:752-774) and gatherScreen (rc.ts:929-954, evalSH rc.ts:819-829)
// evaluated in double precision from the f32 intervals of the last trace (kept by gi_rc_set_debug_hits), with no
// rounding between the stages.  The inputs that are f32 in every atlas mode (frame, G-buffer, probes, solid angles)
// are widened, not recomputed, so the difference to the f32/f16/bf16 irradiance is the rounding of the merge and
// gather arithmetic and of the atlas stores alone.  This is the one place the library computes in f64.
#include "gi_internal.h"

namespace gi {

struct __align__(16) dbl4 { double x, y, z, w; };
struct d3 { double x, y, z; };
__device__ __forceinline__ d3 D3(double x, double y, double z) { d3 r = {x, y, z}; return r; }
__device__ __forceinline__ double ddot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

__device__ __forceinline__ d3 dir_of64(uint32_t di, uint32_t res) {
  double u = ((double)(di % res) + 0.5) / res, v = ((double)(di / res) + 0.5) / res;
  double fx = u * 2.0 - 1.0, fy = v * 2.0 - 1.0;
  d3 n = D3(fx, fy, 1.0 - fabs(fx) - fabs(fy));
  double t = n.z < 0.0 ? -n.z : 0.0;
  n.x += n.x >= 0.0 ? -t : t;
  n.y += n.y >= 0.0 ? -t : t;
  double l = sqrt(ddot(n, n));
  return D3(n.x / l, n.y / l, n.z / l);
}

__device__ __forceinline__ void sh_basis64(d3 n, double y[9]) {
  y[0] = 0.282095; y[1] = 0.488603 * n.y; y[2] = 0.488603 * n.z; y[3] = 0.488603 * n.x;
  y[4] = 1.092548 * n.x * n.y; y[5] = 1.092548 * n.y * n.z; y[6] = 0.315392 * (3.0 * n.z * n.z - 1.0);
  y[7] = 1.092548 * n.x * n.z; y[8] = 0.546274 * (n.x * n.x - n.y * n.y);
}

// a value as an f16 atlas stores it (round to nearest even), back in double
__device__ __forceinline__ double as_f16(double x) { return (double)__half2float(__double2half(x)); }

// the traced intervals [first, first + n) widened to double; f16: rounded to f16 first (the storage-rounding study)
__global__ void k_widen64(const float4 *__restrict__ src, dbl4 *__restrict__ dst, uint32_t first, uint32_t n, bool f16) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float4 s = src[first + i];
    dbl4 d = {s.x, s.y, s.z, s.w};
    if (f16) { d.x = as_f16(d.x); d.y = as_f16(d.y); d.z = as_f16(d.z); d.w = as_f16(d.w); }
    dst[first + i] = d;
  }
}

// mergeScreen for cascade c, in place on the f64 atlas: radiance + T * (weighted average of the upper cascade)
// f16: the merged radiance is rounded to f16 as it is stored (cascades above 0; cascade 0's feeds projectSH unstored)
__global__ void __launch_bounds__(256) k_merge64(RcDev r, dbl4 *rad, uint32_t c, bool f16) {
  const CascDev &L = r.c[c];
  uint32_t dirs = L.res * L.res;
  uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= L.tiles_x * L.tiles_y * dirs) return;
  const float *F = r.frame;
  uint32_t pi = t / dirs, di = t % dirs;
  dbl4 rv = rad[(size_t)L.rad_off + t];
  d3 up = D3(F[F_SKY], F[F_SKY + 1], F[F_SKY + 2]);
  if (c + 1u < r.cascades && rv.w > 0.0) {
    up = D3(0, 0, 0);
    ProbeDev pr = r.probes[L.probe_off + pi];
    if (pr.pos.w > 0.0f) {
      const CascDev &U = r.c[c + 1u];
      double ux = (((double)(pi % L.tiles_x) + 0.5) * L.tile_size) / U.tile_size - 0.5;
      double uy = (((double)(pi / L.tiles_x) + 0.5) * L.tile_size) / U.tile_size - 0.5;
      int bx = (int)floor(ux), by = (int)floor(uy);
      double fx = ux - bx, fy = uy - by;
      uint32_t u0 = di % L.res, v0 = di / L.res;
      d3 acc = D3(0, 0, 0);
      double ws = 0.0;
      for (uint32_t k = 0; k < 4; k++) {
        int ox = (int)(k & 1u), oy = (int)(k >> 1);
        int qx = iclamp(bx + ox, 0, (int)U.tiles_x - 1), qy = iclamp(by + oy, 0, (int)U.tiles_y - 1);
        uint32_t qi = (uint32_t)qy * U.tiles_x + (uint32_t)qx;
        ProbeDev qp = r.probes[U.probe_off + qi];
        if (qp.pos.w <= 0.0f) continue;
        double fwx = ox == 1 ? fx : 1.0 - fx, fwy = oy == 1 ? fy : 1.0 - fy;
        double rel = fabs((double)qp.nrm.w - (double)pr.nrm.w) / (double)pr.nrm.w;
        double w = (fwx * fwy + 1e-4) * (exp(-20.0 * rel) + 1e-4);
        d3 ua;
        if (U.res == L.res) {
          dbl4 q = rad[(size_t)U.rad_off + qi * U.res * U.res + v0 * U.res + u0];
          ua = D3(q.x, q.y, q.z);
        } else {
          size_t base = (size_t)U.rad_off + qi * U.res * U.res + v0 * 2u * U.res + u0 * 2u;
          dbl4 a = rad[base], b = rad[base + 1u], cc = rad[base + U.res], d = rad[base + U.res + 1u];
          ua = D3(0.25 * (a.x + b.x + cc.x + d.x), 0.25 * (a.y + b.y + cc.y + d.y), 0.25 * (a.z + b.z + cc.z + d.z));
        }
        acc.x += w * ua.x; acc.y += w * ua.y; acc.z += w * ua.z;
        ws += w;
      }
      if (ws > 0.0) up = D3(acc.x / ws, acc.y / ws, acc.z / ws);
    }
  }
  dbl4 o = {rv.x + rv.w * up.x, rv.y + rv.w * up.y, rv.z + rv.w * up.z, 1.0};
  if (f16) { o.x = as_f16(o.x); o.y = as_f16(o.y); o.z = as_f16(o.z); }
  rad[(size_t)L.rad_off + t] = o;
}

// projectSH: 27 doubles (9 coefficients x rgb) per cascade-0 probe
__global__ void __launch_bounds__(256) k_project_sh64(RcDev r, const dbl4 *__restrict__ rad, double *__restrict__ sh) {
  const CascDev &L = r.c[0];
  uint32_t pi = blockIdx.x * blockDim.x + threadIdx.x;
  if (pi >= L.tiles_x * L.tiles_y) return;
  const float *F = r.frame;
  double cf[27];
  for (int k = 0; k < 27; k++) cf[k] = 0.0;
  for (uint32_t d = 0; d < 16; d++) {
    dbl4 rp = rad[(size_t)L.rad_off + pi * 16u + d];
    double om = F[F_OMEGA + d];
    double y[9];
    sh_basis64(dir_of64(d, 4u), y);
    for (int k = 0; k < 9; k++) {
      cf[3 * k] += rp.x * om * y[k];
      cf[3 * k + 1] += rp.y * om * y[k];
      cf[3 * k + 2] += rp.z * om * y[k];
    }
  }
  const double PI = 3.14159265;
  for (int k = 0; k < 9; k++) {
    double a = k == 0 ? PI : (k < 4 ? 2.0 * PI / 3.0 : PI / 4.0);
    for (int i = 0; i < 3; i++) sh[27u * (size_t)pi + 3 * k + i] = cf[3 * k + i] * a;
  }
}

// gatherScreen: per pixel, the 4 surrounding cascade-0 probes weighted by bilinear x depth x normal similarity
__global__ void __launch_bounds__(256) k_gather64(RcDev r, const double *__restrict__ sh, dbl4 *__restrict__ irr) {
  uint32_t px = blockIdx.x * 16u + (threadIdx.x & 15u), py = blockIdx.y * 16u + (threadIdx.x >> 4);
  if (px >= r.width || py >= r.height) return;
  size_t q = (size_t)py * r.width + px;
  const float *F = r.frame;
  double d = r.depth[q];
  dbl4 out = {0.0, 0.0, 0.0, 0.0};
  if (d > 0.0) {
    const CascDev &L = r.c[0];
    double nx = ((double)px + 0.5) * (double)F[F_SIZE + 2] * 2.0 - 1.0;
    double ny = 1.0 - ((double)py + 0.5) * (double)F[F_SIZE + 3] * 2.0;
    const float *m = F + F_IVP;
    double h[4];
    for (int i = 0; i < 4; i++)
      h[i] = (double)m[i] * nx + (double)m[4 + i] * ny + (double)m[8 + i] * d + (double)m[12 + i];
    d3 x = D3(h[0] / h[3], h[1] / h[3], h[2] / h[3]);
    uint2 nn = r.normal[q];
    d3 n = D3(h2f(nn.x & 0xffffu), h2f(nn.x >> 16), h2f(nn.y & 0xffffu));
    double z = ddot(D3(x.x - F[F_EYE], x.y - F[F_EYE + 1], x.z - F[F_EYE + 2]), D3(F[F_FWD], F[F_FWD + 1], F[F_FWD + 2]));
    double ux = ((double)px + 0.5) / L.tile_size - 0.5, uy = ((double)py + 0.5) / L.tile_size - 0.5;
    int bx = (int)floor(ux), by = (int)floor(uy);
    double fx = ux - bx, fy = uy - by;
    double y[9];
    sh_basis64(n, y);
    double acc[3] = {0.0, 0.0, 0.0}, ws = 0.0;
    for (uint32_t k = 0; k < 4; k++) {
      int ox = (int)(k & 1u), oy = (int)(k >> 1);
      int qx = iclamp(bx + ox, 0, (int)L.tiles_x - 1), qy = iclamp(by + oy, 0, (int)L.tiles_y - 1);
      uint32_t qi = (uint32_t)qy * L.tiles_x + (uint32_t)qx;
      ProbeDev pr = r.probes[L.probe_off + qi];
      if (pr.pos.w <= 0.0f) continue;
      double fwx = ox == 1 ? fx : 1.0 - fx, fwy = oy == 1 ? fy : 1.0 - fy;
      double rel = fabs((double)pr.nrm.w - z) / z;
      double nd = ddot(n, D3(pr.nrm.x, pr.nrm.y, pr.nrm.z));
      nd = nd > 0.0 ? nd : 0.0;
      double w = (fwx * fwy + 1e-4) * (exp(-20.0 * rel) + 1e-4) * (nd * nd * nd * nd + 1e-3);
      const double *s = sh + 27u * (size_t)qi;
      for (int i = 0; i < 3; i++) {
        double e = 0.0;
        for (int k2 = 0; k2 < 9; k2++) e += s[3 * k2 + i] * y[k2];
        acc[i] += w * (e > 0.0 ? e : 0.0);
      }
      ws += w;
    }
    out.x = ws > 0.0 ? acc[0] / ws : 0.0;
    out.y = ws > 0.0 ? acc[1] / ws : 0.0;
    out.z = ws > 0.0 ? acc[2] / ws : 0.0;
    out.w = 1.0;
  }
  irr[q] = out;
}

}  // namespace gi

using namespace gi;

cudaError_t gi_launch_merge_gather_f64(const RcDev &r, const float4 *traced, void *rad64, double *sh64, void *irr64,
                                       uint32_t f16_cascades, cudaStream_t st) {
  dbl4 *rad = reinterpret_cast<dbl4 *>(rad64);
  for (uint32_t c = 0; c < r.cascades; c++) {
    const CascDev &L = r.c[c];
    const uint32_t n = L.tiles_x * L.tiles_y * L.res * L.res;
    k_widen64<<<min((n + 255u) / 256u, 1024u), 256, 0, st>>>(traced, rad, L.rad_off, n, ((f16_cascades >> c) & 1u) != 0u);
  }
  for (int c = (int)r.cascades - 1; c >= 0; c--) {
    const CascDev &L = r.c[c];
    uint32_t n = L.tiles_x * L.tiles_y * L.res * L.res;
    k_merge64<<<(n + 255u) / 256u, 256, 0, st>>>(r, rad, (uint32_t)c, c > 0 && ((f16_cascades >> c) & 1u) != 0u);
  }
  k_project_sh64<<<(r.c[0].tiles_x * r.c[0].tiles_y + 255u) / 256u, 256, 0, st>>>(r, rad, sh64);
  dim3 gg((r.width + 15u) / 16u, (r.height + 15u) / 16u);
  k_gather64<<<gg, 256, 0, st>>>(r, sh64, reinterpret_cast<dbl4 *>(irr64));
  return cudaGetLastError();
}
