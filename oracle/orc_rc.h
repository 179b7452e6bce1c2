/* Shared internals of the oracle's cascade files (rc.c: screen probes, world.c: world probes).  Test infrastructure
 * only. */
#ifndef ORC_RC_H
#define ORC_RC_H
#include "gi_oracle.h"
#include "orc_math.h"

#define PI_F 3.14159265f

/* Frame word offsets (frame.ts:4-21, packFrame :76-93). */
enum { F_VP = 0, F_IVP = 16, F_EYE = 80, F_FWD = 84, F_SUN = 88, F_SUNE = 92, F_SKY = 96, F_SIZE = 100, F_RC = 104,
       F_RC2 = 108, F_RU = 112, F_RU2 = 116, F_OMEGA = 120, F_STYLE = 136 };

typedef struct {
  const orc_vox *vx;
  const float *F;
  float sky[3];
  const orc_bounce *bn;   /* the volume's own rays: read the previous volume bn_prev at the hit (bounce.ts:90-93) */
  const float *bn_prev;
} ctx_t;

static inline float vox_size(const orc_vox *vx, uint32_t L) { return scale2(vx->v0, (int)L); }
static inline i3 org(const orc_vox *vx, uint32_t L) { return I(vx->origin[L][0], vx->origin[L][1], vx->origin[L][2]); }
static inline uint32_t ptr_index(const orc_vox *vx, uint32_t L, i3 b) {
  uint32_t G = vx->G;
  return L * G * G * G + ((uint32_t)b.z * G + (uint32_t)b.y) * G + (uint32_t)b.x;
}

typedef struct { float r, g, b, T; uint32_t lvl, ptr, bit, tin; uint32_t steps; } trace_t;

/* rc.c */
v3 world_at(const float *F, int32_t px, int32_t py, float d);
float view_z(const float *F, v3 p);
v3 dir_of(uint32_t di, uint32_t res);
float round_store(float x, uint32_t atlas);
uint32_t vox_rank(const orc_vox *vx, uint32_t brick, uint32_t bit);
void vox_at(const orc_vox *vx, uint32_t L, i3 c, uint32_t out[3]);
uint32_t vox_level_for(const orc_vox *vx, uint32_t L, v3 e);
uint32_t vox_level(const orc_vox *vx, const orc_layout *ly, float s0, uint32_t c);
void trace_vox(const ctx_t *cx, v3 o, v3 d, float t0, float t1, float tskip, uint32_t L, uint32_t cap, trace_t *out);
void sh_basis(v3 n, float y[9]);
v3 upper_avg(const orc_layout *ly, const float *rad, uint32_t cu, uint32_t q, uint32_t u, uint32_t v, uint32_t lr);
/* dyn.c */
void dyn_compose(const orc_vox *vx, v3 o, v3 d, float t0, float t1, v3 ooff, float k, trace_t *tr);
/* word k of the voxel at data base `base` of level L: level 0 fixed point (/ 65536), the levels above f32 */
float dyn_word_at(const orc_dyn *dl, uint32_t base, uint32_t k, uint32_t L);
/* dynInject's store (dynlayer.ts:186-189): add[0..2] added to the voxel's radiance words 7..9, level 0 in fixed point
 * (u32(round(x * 65536)), the sum wrapping as u32), the levels above in f32 */
void dyn_add_radiance(orc_dyn *dl, uint32_t base, uint32_t L, const float add[3]);
#endif
