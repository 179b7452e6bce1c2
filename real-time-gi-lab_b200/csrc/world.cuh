// World probes over the voxel tracer on sm_100a (the reference's method 'world' with the voxel world tracer, config
// tokens 'world-<P>-voxel[-vrel]'): registerPixels / registerUp / compact / relocate / relocateVox / linkParents
// (src/core/rc.ts:253-570), trace over the world probes (:600-622), mergeWorld (:688-708), projectSH with the c0 history
// (:752-816), gatherWorld with segOccluded (:854-927), in Rc.encode's pass order (:1180-1221).
//
// Included by rc_solve.cu (it shares the tracer, the atlas formats and the SH helpers); not a translation unit of its
// own.  Form changes from the reference, each an order the reference can produce, results unchanged otherwise:
//  * insertKey is ordered linear probing (a larger key takes a smaller one's slot and the smaller moves on), so the
//    table does not depend on the order of the concurrent inserts (the phase-concurrent deterministic hash table of
//    Shun & Blelloch, SPAA 2014); compact numbers the keys in slot order with a chained scan instead of an atomic
//    counter.  The whole solve is then deterministic and equal to the oracle's state word for word;
//  * registerPixels inserts the 8 keys of each distinct grid cell of a warp once (the lanes in the same cell and LOD
//    agree on a leader);
//  * relocateVox and linkParents run one warp per probe (64 and 8 x 8 threads in the reference); the sums the
//    reference takes on one thread are still taken by one lane, in the same order;
//  * indirect dispatches become grid-stride loops over the device-side probe counts;
//  * the trace is the persistent ray loop of the screen path over the rays of every cascade's live probes.

constexpr uint32_t W_NONE = 0xffffffffu;
constexpr uint32_t W_COMPACT_SLOTS = 2048;   // hash slots per compact block (8 a thread)

// hash32 (rc.ts:248-250)
__device__ __forceinline__ uint32_t w_hash32(uint32_t x) {
  uint32_t h = x;
  h ^= h >> 16; h *= 0x7feb352du; h ^= h >> 15; h *= 0x846ca68bu; h ^= h >> 16;
  return h;
}
// lodFor (rc.ts:252): floor(log2(y)) of the f32 y >= 1 taken exactly as its binary exponent
__device__ __forceinline__ int w_lod_for(const float *__restrict__ F, float dist) {
  const float y = mx(dist * F[F_RC + 1] * F[F_RC + 2] / F[F_RC], 1.0f);
  return iclamp((int)((__float_as_uint(y) >> 23) & 0xffu) - 127, 0, 14);
}
// spacing (rc.ts:253): sMin * 2^(lod + c), exact
__device__ __forceinline__ float w_spacing(const float *__restrict__ F, int lod, uint32_t c) {
  return ldexpf(F[F_RC], lod + (int)c);
}
// originOf (rc.ts:254)
__device__ __forceinline__ i3 w_origin(const float *__restrict__ F, float s) {
  const i3 o = vfloori(mk(F[F_EYE] / s, F[F_EYE + 1] / s, F[F_EYE + 2] / s));
  return mki(o.x - 256, o.y - 256, o.z - 256);
}
// keyFor (rc.ts:255-259) with the origin of (lod, c) given: the origin depends only on them, so callers that make
// several keys of one LOD and cascade compute it once
__device__ __forceinline__ uint32_t w_key_at(i3 g, i3 o, int lod) {
  const i3 r = mki(g.x - o.x, g.y - o.y, g.z - o.z);
  if (r.x < 0 || r.y < 0 || r.z < 0 || r.x >= 512 || r.y >= 512 || r.z >= 512) return W_NONE;
  return 0x80000000u | ((uint32_t)lod << 27) | ((uint32_t)r.x << 18) | ((uint32_t)r.y << 9) | (uint32_t)r.z;
}
__device__ __forceinline__ uint32_t w_key(const float *__restrict__ F, i3 g, int lod, uint32_t c) {
  return w_key_at(g, w_origin(F, w_spacing(F, lod, c)), lod);
}
__device__ __forceinline__ i3 w_corner(uint32_t k) { return mki((int)(k & 1u), (int)((k >> 1) & 1u), (int)((k >> 2) & 1u)); }

// insertKey (rc.ts:260-273), ordered: false when the key could not be stored (it would sit 256 or more slots past its
// home).  Every slot's key only grows, so every compare-and-swap that fails has seen another insert make progress;
// the loop is bounded all the same.
__device__ __forceinline__ bool w_insert(uint32_t *keys, uint32_t mask, uint32_t key) {
  uint32_t h = w_hash32(key) & mask;
  for (uint32_t it = 0; it < mask + 256u + 65536u; it++) {
    const uint32_t cur = *reinterpret_cast<volatile uint32_t *>(&keys[h]);
    if (cur == key) return true;
    if (cur < key) {   // the empty key 0 is below every key
      if (atomicCAS(&keys[h], cur, key) != cur) continue;   // the slot changed: look at it again
      if (cur == 0u) return true;
      key = cur;        // carry the displaced key on
    }
    h = (h + 1u) & mask;
    if (((h - (w_hash32(key) & mask)) & mask) >= 256u) return false;
  }
  return false;
}
// lookup (rc.ts:274-284)
__device__ __forceinline__ uint32_t w_lookup(const WorldDev &w, uint32_t c, uint32_t key) {
  if (key == W_NONE) return W_NONE;
  const uint32_t mask = w.hash_mask[c], off = w.hash_off[c];
  uint32_t h = w_hash32(key) & mask;
  for (uint32_t i = 0; i < 256u; i++) {
    const uint32_t cur = w.keys[off + h];
    if (cur == key) return w.slot_probe[off + h];
    if (cur == 0u) return W_NONE;
    h = (h + 1u) & mask;
  }
  return W_NONE;
}

// voxCell (rc.ts:379-386): (brick, bit), brick GI_MARK when empty or outside the level's window
__device__ __forceinline__ uint2 w_vox_cell(const VoxDev &v, uint32_t L, f3 p) {
  const float vs = vox_size(v, L);
  const i3 c = vfloori((p - (vi2f(org(v, L)) * vs) * 8.0f) / vs);
  const int n = (int)v.G * 8;
  if (c.x < 0 || c.y < 0 || c.z < 0 || c.x >= n || c.y >= n || c.z >= n) return make_uint2(GI_MARK, 0u);
  const uint3 r = vox_at(v, L, c);
  return r.x == GI_EMPTY ? make_uint2(GI_MARK, 0u) : make_uint2(r.x, r.y);
}
__device__ __forceinline__ bool w_vox_occ(const VoxDev &v, uint32_t L, f3 p) { return w_vox_cell(v, L, p).x != GI_MARK; }
// voxStoredNormal (rc.ts:387-393); a voxel past the attribute pool has normal 0
__device__ __forceinline__ f3 w_stored_normal(const VoxDev &v, uint2 cell) {
  if (v.base[cell.x] == GI_EMPTY) return mk(0.0f, 0.0f, 0.0f);
  const uint32_t e = v.attr[vox_rank(v, cell.x, cell.y)].y;
  const float a = mx((float)(int16_t)(e & 0xffffu) / 32767.0f, -1.0f), b = mx((float)(int16_t)(e >> 16) / 32767.0f, -1.0f);
  f3 n = mk(a, b, 1.0f - fabsf(a) - fabsf(b));
  const float q = mx(-n.z, 0.0f);
  n.x += n.x >= 0.0f ? -q : q;
  n.y += n.y >= 0.0f ? -q : q;
  return n;
}
// cubeOff (rc.ts:395)
__device__ __forceinline__ f3 w_cube_off(uint32_t k, float vg) {
  return mk((float)(k & 3u) - 1.5f, (float)((k >> 2) & 3u) - 1.5f, (float)(k >> 4) - 1.5f) * vg;
}
// The segment test of linkParents and segOccluded (rc.ts:553-558, 854-878): sample i of min(ceil(|b - a| / v), 16)
__device__ __forceinline__ uint32_t w_seg_samples(const VoxDev &v, f3 d, uint32_t L) {
  return (uint32_t)mn(ceilf(length3(d) / vox_size(v, L)), 16.0f);
}
// (i + 0.5) / k for k = 1..16, i < k: the IEEE quotients, tabulated on the host (gi_world_tables)
__device__ float g_seg_t[16 * 16];
__device__ __forceinline__ float w_seg_t(uint32_t i, uint32_t k) { return g_seg_t[(k - 1u) * 16u + i]; }
__device__ __forceinline__ bool w_seg_occluded(const VoxDev &v, f3 a, f3 b, uint32_t L) {
  const f3 d = b - a;
  const uint32_t k = w_seg_samples(v, d, L);
  for (uint32_t i = 0; i < k; i++)
    if (w_vox_occ(v, L, a + d * w_seg_t(i, k))) return true;
  return false;
}

// relocate (rc.ts:345-366): the probe pushed out along a plane fitted to G-buffer samples within 1.5 spacings.  Half a
// warp per probe, lane j reading tap j (the 16 taps' loads in flight together); every lane then takes the sums in tap
// order from its half's lanes.
__device__ __forceinline__ void w_relocate_gbuffer(const RcDev &r, const WorldDev &w, uint32_t c, uint32_t bid,
                                                   uint32_t nblk) {
  const float *F = r.frame;
  const uint32_t lane = threadIdx.x & 31u, j = lane & 15u, n = w.state[8 + c];
  // a warp's two probes: 2 * warp and 2 * warp + 1 (the loop bound is the warp's, so every lane shuffles)
  for (uint32_t wp = (bid * blockDim.x + threadIdx.x) >> 5; 2u * wp < n; wp += (nblk * blockDim.x) >> 5) {
    const uint32_t pi = 2u * wp + (lane >> 4);
    const bool live = pi < n;
    ProbeDev *prp = &r.probes[r.c[c].probe_off + (live ? pi : 2u * wp)];
    const int4 g = prp->grid;
    const float s = w_spacing(F, g.w, c);
    const f3 p = vi2f(mki(g.x, g.y, g.z)) * s;
    const float *m = F + F_VP;
    float c4[4];
#pragma unroll
    for (int i = 0; i < 4; i++) c4[i] = m[i] * p.x + m[4 + i] * p.y + m[8 + i] * p.z + m[12 + i] * 1.0f;
    const bool front = live && !(c4[3] <= F[F_EYE + 3]);
    bool ok = false;
    f3 tn = mk(0.0f, 0.0f, 0.0f);
    float te = 0.0f;
    if (front) {
      const float nx = c4[0] / c4[3], ny = c4[1] / c4[3];
      const float cx = (nx * 0.5f + 0.5f) * F[F_SIZE], cy = (0.5f - ny * 0.5f) * F[F_SIZE + 1];
      const float rpx = s / (c4[3] * F[F_RC + 1]);
      const float ox = ((float)(j % 4u) - 1.5f) / 1.5f * rpx, oy = ((float)(j / 4u) - 1.5f) / 1.5f * rpx;
      const int qx = __float2int_rd(cx + ox), qy = __float2int_rd(cy + oy);
      if (qx >= 0 && qy >= 0 && qx < (int)r.width && qy < (int)r.height) {
        const size_t q = (size_t)qy * r.width + (size_t)qx;
        const float d = r.depth[q];
        if (d > 0.0f) {
          const f3 x = world_at(F, qx, qy, d);
          if (!(length3(x - p) > 1.5f * s)) {
            const uint2 nn = r.normal[q];
            tn = mk(h2f(nn.x & 0xffffu), h2f(nn.x >> 16), h2f(nn.y & 0xffffu));
            te = dot(tn, p - x) / s;
            ok = true;
          }
        }
      }
    }
    f3 sn = mk(0.0f, 0.0f, 0.0f);
    float se = 0.0f, cnt = 0.0f;
    const unsigned okm = __ballot_sync(0xffffffffu, ok);
#pragma unroll
    for (uint32_t t = 0; t < 16u; t++) {
      const int src = (int)((lane & 16u) | t);
      const f3 nt = mk(__shfl_sync(0xffffffffu, tn.x, src), __shfl_sync(0xffffffffu, tn.y, src),
                       __shfl_sync(0xffffffffu, tn.z, src));
      const float et = __shfl_sync(0xffffffffu, te, src);
      if ((okm >> src) & 1u) {
        sn = sn + nt;
        se += et;
        cnt += 1.0f;
      }
    }
    if (!front || j != 0u || cnt < 1.0f || length3(sn) < 0.3f * cnt) continue;
    const f3 mm = normalize3(sn);
    const float e = se / cnt;
    const f3 rp = e < F[F_RC2] ? p + (mm * (F[F_RC2] - e)) * s : p;
    prp->pos = make_float4(rp.x, rp.y, rp.z, prp->pos.w);
    prp->nrm = make_float4(mm.x, mm.y, mm.z, view_z(F, rp));
  }
}

// clearKeys (rc.ts:472-476) + clearHist of this solve's parity; the counters, the trace's ray counter (word 80) and
// the compactions' scan states
__global__ void k_w_clear(RcDev r, WorldDev w) {
  grid_dep_wait();
  const uint32_t nxt = w.state[0] ^ 1u;
  const uint32_t n = max(max(w.hash_total, w.look_total), max(w.hist_h, 96u));
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (i < w.hash_total) w.keys[i] = 0u;
    if (i < w.look_total) w.look[i] = 0ull;
    if (i < w.hist_h) w.hist_tab[nxt * w.hist_h + i] = 0u;
    if (i < 81u) r.counts[i] = 0u;
  }
}

// registerPixels (rc.ts:484-500), launched for a stride of 1; the frame's stride (word 114) picks the pixels.  The
// history parity flips here (Rc.encode, rc.ts:1180), after k_w_clear has read it.
__global__ void __launch_bounds__(256) k_w_register_pixels(RcDev r, WorldDev w) {
  grid_dep_wait();
  if (blockIdx.x == 0 && threadIdx.x == 0) { w.state[0] ^= 1u; w.state[16] = 0u; w.state[7] = 0u; }
  const float *F = r.frame;
  const uint32_t st = max(reinterpret_cast<const uint32_t *>(F)[F_RU + 2], 1u);
  const uint32_t sx = (r.width + st - 1u) / st, sy = (r.height + st - 1u) / st;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x, lane = threadIdx.x & 31u;
  int lod = 0;
  i3 b = mki(0, 0, 0), org0 = mki(0, 0, 0);
  bool live = false;
  if (i < sx * sy) {
    const int px = (int)((i % sx) * st + st / 2u), py = (int)((i / sx) * st + st / 2u);
    if (px < (int)r.width && py < (int)r.height) {
      const float d = r.depth[(size_t)py * r.width + (size_t)px];
      if (d > 0.0f) {
        const f3 x = world_at(F, px, py, d);
        lod = w_lod_for(F, length3(x - mk(F[F_EYE], F[F_EYE + 1], F[F_EYE + 2])));
        const float s = w_spacing(F, lod, 0u);
        b = vfloori(mk(x.x / s, x.y / s, x.z / s));
        org0 = w_origin(F, s);
        live = true;
      }
    }
  }
  // the lanes whose pixels fall in the same grid cell at the same LOD hold the same 8 keys: one of them inserts them
  const unsigned long long xy = ((unsigned long long)(uint32_t)b.x << 32) | (uint32_t)b.y;
  const unsigned long long zl = live ? (((unsigned long long)(uint32_t)b.z << 32) | (uint32_t)lod) : ~0ull;
  const unsigned grp = __match_any_sync(0xffffffffu, xy) & __match_any_sync(0xffffffffu, zl);
  if (live && (uint32_t)(__ffs(grp) - 1) == lane) {
    for (uint32_t k = 0; k < 8u; k++) {
      const i3 o = w_corner(k);
      const uint32_t key = w_key_at(mki(b.x + o.x, b.y + o.y, b.z + o.z), org0, lod);
      if (key != W_NONE && !w_insert(w.keys + w.hash_off[0], w.hash_mask[0], key)) atomicAdd(&r.counts[16], 1u);
    }
  }
}

// registerUp (rc.ts:503-518): the grid points of cascade c with a non-zero trilinear weight at each probe of c - 1
__device__ __forceinline__ void w_register_up(const RcDev &r, const WorldDev &w, uint32_t c, uint32_t bid, uint32_t nblk) {
  const float *F = r.frame;
  const uint32_t n = w.state[8 + c - 1u] * 8u;   // one thread per (probe, corner)
  for (uint32_t t = bid * blockDim.x + threadIdx.x; t < n; t += nblk * blockDim.x) {
    const int4 g = r.probes[r.c[c - 1u].probe_off + (t >> 3)].grid;
    const i3 o = w_corner(t & 7u);
    if ((o.x > 0 && (g.x & 1) == 0) || (o.y > 0 && (g.y & 1) == 0) || (o.z > 0 && (g.z & 1) == 0)) continue;
    const uint32_t key = w_key(F, mki((g.x >> 1) + o.x, (g.y >> 1) + o.y, (g.z >> 1) + o.z), g.w, c);
    if (key != W_NONE && !w_insert(w.keys + w.hash_off[c], w.hash_mask[c], key)) atomicAdd(&r.counts[16 + c], 1u);
  }
}

// compact's write for the key in slot h with probe index idx: slotProbe, and the probe at its grid point with its voxel
// level (the relocation step that follows moves it)
__device__ __forceinline__ void w_compact_slot(const RcDev &r, const VoxDev &v, const WorldDev &w, uint32_t c, uint32_t h,
                                               uint32_t key, uint32_t idx) {
  const float *F = r.frame;
  if (idx >= w.cap[c]) { w.slot_probe[w.hash_off[c] + h] = W_NONE; return; }
  w.slot_probe[w.hash_off[c] + h] = idx;
  const int lod = (int)((key >> 27) & 15u);
  const float s = w_spacing(F, lod, c);
  const i3 o = w_origin(F, s);
  const i3 g = mki((int)((key >> 18) & 511u) + o.x, (int)((key >> 9) & 511u) + o.y, (int)(key & 511u) + o.z);
  const f3 p = vi2f(g) * s;
  const float s0 = w_spacing(F, lod, 0u);
  ProbeDev pr;
  pr.pos = make_float4(p.x, p.y, p.z, s0);
  pr.nrm = make_float4(0.0f, 0.0f, 0.0f, view_z(F, p));
  pr.grid = make_int4(g.x, g.y, g.z, lod);
  r.probes[r.c[c].probe_off + idx] = pr;
  r.plevel[r.c[c].probe_off + idx] = vox_level(v, r, s0, c);
}

// compact (rc.ts:520-537): a chained scan over the table's slots (W_COMPACT_SLOTS a block, 8 a thread) numbers the
// keys in slot order; the last part publishes the count and the first ray of the next cascade.
__device__ __forceinline__ void w_compact(const RcDev &r, const VoxDev &v, const WorldDev &w, uint32_t c) {
  const uint32_t size = w.hash_mask[c] + 1u, nblk = (size + W_COMPACT_SLOTS - 1u) / W_COMPACT_SLOTS, cap = w.cap[c];
  unsigned long long *look = w.look + w.look_off[c];
  const uint32_t blk = chain_ticket(look);
  const uint32_t h0 = blk * W_COMPACT_SLOTS + threadIdx.x * 8u;
  uint32_t keys8[8] = {0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u};
  if (h0 + 8u <= size && (w.hash_off[c] & 3u) == 0u) {   // two aligned 128-bit loads
    const uint4 *kp = reinterpret_cast<const uint4 *>(w.keys + w.hash_off[c] + h0);
    const uint4 ka = kp[0], kb = kp[1];
    keys8[0] = ka.x; keys8[1] = ka.y; keys8[2] = ka.z; keys8[3] = ka.w;
    keys8[4] = kb.x; keys8[5] = kb.y; keys8[6] = kb.z; keys8[7] = kb.w;
  } else {
    for (uint32_t k = 0; k < 8u && h0 + k < size; k++) keys8[k] = w.keys[w.hash_off[c] + h0 + k];
  }
  uint32_t mine = 0;
#pragma unroll
  for (int k = 0; k < 8; k++) mine += keys8[k] != 0u ? 1u : 0u;
  uint32_t tot;
  const uint32_t ex = block_scan_256(mine, &tot);
  __shared__ uint32_t s_pre, s_over;
  if (threadIdx.x == 0) {
    s_pre = chain_prefix(look, blk, tot, w.state + 1);   // a give-up sets state[7]
    s_over = 0u;
  }
  __syncthreads();
  const uint32_t first = s_pre + ex;
  const uint32_t over = first >= cap ? mine : (first + mine > cap ? first + mine - cap : 0u);
  if (over) atomicAdd(&s_over, over);
  __syncthreads();
  if (threadIdx.x == 0) {
    if (s_over) atomicAdd(&r.counts[8 + c], s_over);
    if (blk == nblk - 1u) {
      const uint32_t total = s_pre + tot, np = min(total, cap);
      r.counts[c] = total;
      w.state[8 + c] = np;
      w.state[16 + c + 1u] = w.state[16 + c] + (np << r.c[c].dirs_log2);
    }
  }
  uint32_t idx = first;
#pragma unroll
  for (uint32_t k = 0; k < 8u; k++)
    if (keys8[k] != 0u) w_compact_slot(r, v, w, c, h0 + k, keys8[k], idx++);
}

// relocateVox (rc.ts:414-470), one warp per probe: lane l reads cube cells l and l + 32; lane 0 takes the sums in the
// serial order; lanes 0..16 test the 17 steps of the march.
__device__ __forceinline__ void w_relocate_vox(const RcDev &r, const VoxDev &v, const WorldDev &w, uint32_t c, uint32_t bid,
                                               uint32_t nblk) {
  const float *F = r.frame;
  const uint32_t lane = threadIdx.x & 31u, n = w.state[8 + c];
  for (uint32_t pi = (bid * blockDim.x + threadIdx.x) >> 5; pi < n; pi += (nblk * blockDim.x) >> 5) {
    ProbeDev *prp = &r.probes[r.c[c].probe_off + pi];
    const int4 g = prp->grid;
    const int lod = g.w;
    const float s0 = w_spacing(F, lod, 0u);
    const f3 p = vi2f(mki(g.x, g.y, g.z)) * w_spacing(F, lod, c);
    const uint32_t L = vox_level_for(v, vox_level(v, r, s0, c), p);
    const uint32_t Lg = vox_level_for(v, L + 1u < v.levels ? L + 1u : v.levels - 1u, p);
    const float vg = vox_size(v, Lg);
    const uint2 ca = w_vox_cell(v, Lg, p + w_cube_off(lane, vg)), cb = w_vox_cell(v, Lg, p + w_cube_off(lane + 32u, vg));
    const unsigned long long occ = (unsigned long long)__ballot_sync(0xffffffffu, ca.x != GI_MARK) |
                                   ((unsigned long long)__ballot_sync(0xffffffffu, cb.x != GI_MARK) << 32);
    f3 dir = mk(0.0f, 0.0f, 0.0f);
    uint32_t flag = 0;
    if (lane == 0) {
      float cnt = 0.0f;
      for (unsigned long long m = occ; m; m &= m - 1ull) {
        dir = dir - w_cube_off((uint32_t)(__ffsll((long long)m) - 1), vg);
        cnt += 1.0f;
      }
      flag = cnt < 1.0f ? 0u : (length3(dir) < 0.1f * cnt * vg ? 1u : 2u);
    }
    flag = __shfl_sync(0xffffffffu, flag, 0);
    if (flag == 1u) {   // ambiguous: the stored normals decide, summed in cube order
      const f3 na = ca.x != GI_MARK ? w_stored_normal(v, ca) : mk(0.0f, 0.0f, 0.0f);
      const f3 nb = cb.x != GI_MARK ? w_stored_normal(v, cb) : mk(0.0f, 0.0f, 0.0f);
      f3 sum = mk(0.0f, 0.0f, 0.0f);
      for (uint32_t k = 0; k < 64u; k++) {
        const f3 x = k < 32u ? na : nb;
        const f3 y = mk(__shfl_sync(0xffffffffu, x.x, (int)(k & 31u)), __shfl_sync(0xffffffffu, x.y, (int)(k & 31u)),
                        __shfl_sync(0xffffffffu, x.z, (int)(k & 31u)));
        if ((occ >> k) & 1ull) sum = sum + y;
      }
      dir = sum;
    }
    if (lane == 0 && flag != 0u) {
      if (length3(dir) < 1e-4f) flag = 0u; else { dir = normalize3(dir); flag = 2u; }
    }
    flag = __shfl_sync(0xffffffffu, flag, 0);
    if (flag == 0u) {
      if (lane == 0) {
        prp->nrm = make_float4(0.0f, 0.0f, 0.0f, view_z(F, p));
        prp->pos = make_float4(p.x, p.y, p.z, s0);
      }
      continue;
    }
    const f3 nd = mk(__shfl_sync(0xffffffffu, dir.x, 0), __shfl_sync(0xffffffffu, dir.y, 0), __shfl_sync(0xffffffffu, dir.z, 0));
    const float s = s0 * exp2_((float)c);
    const float back = F[F_RC2] * s;
    const float stp = mx(0.5f * vox_size(v, L), 1.5f * s / 16.0f);
    const float fi = (float)lane * stp;
    const bool stop = lane <= 16u && fi > 1.5f * s;
    bool free_ = false;
    if (lane <= 16u && !stop) {
      const f3 q = p + nd * fi;
      free_ = !w_vox_occ(v, L, q) && !w_vox_occ(v, L, q - nd * back);
    }
    const uint32_t ms = __ballot_sync(0xffffffffu, stop), mf = __ballot_sync(0xffffffffu, free_);
    if (lane == 0) {
      f3 rr = p;
      const uint32_t any = ms | mf;
      if (any) {
        const uint32_t i = (uint32_t)(__ffs(any) - 1);
        if ((mf >> i) & 1u) rr = p + nd * ((float)i * stp);
      }
      prp->pos = make_float4(rr.x, rr.y, rr.z, s0);
      prp->nrm = make_float4(nd.x, nd.y, nd.z, view_z(F, rr));
    }
  }
}

// linkParents (rc.ts:541-567) of cascade c, one warp per probe: parent k on lanes 4k..4k+3, which share its segment's
// samples (hidden parents are not merged, relocate 'voxel' only)
__device__ __forceinline__ void w_link_parents(const RcDev &r, const VoxDev &v, const WorldDev &w, uint32_t c, uint32_t bid,
                                               uint32_t nblk) {
  const float *F = r.frame;
  const uint32_t lane = threadIdx.x & 31u, k = lane >> 2, j = lane & 3u, n = w.state[8 + c];
  for (uint32_t pi = (bid * blockDim.x + threadIdx.x) >> 5; pi < n; pi += (nblk * blockDim.x) >> 5) {
    const ProbeDev pr = r.probes[r.c[c].probe_off + pi];
    uint32_t q = W_NONE;
    if (j == 0u) {
      const i3 o = w_corner(k);
      const bool ox = (pr.grid.x & 1) != 0, oy = (pr.grid.y & 1) != 0, oz = (pr.grid.z & 1) != 0;
      if (!((o.x > 0 && !ox) || (o.y > 0 && !oy) || (o.z > 0 && !oz)))
        q = w_lookup(w, c + 1u, w_key(F, mki((pr.grid.x >> 1) + o.x, (pr.grid.y >> 1) + o.y, (pr.grid.z >> 1) + o.z), pr.grid.w, c + 1u));
    }
    q = __shfl_sync(0xffffffffu, q, (int)(lane & ~3u));
    bool hid = false;
    if (q != W_NONE && w.relocate == 2u) {
      const f3 a = ld3(pr.pos);
      const uint32_t Lv = vox_level_for(v, vox_level(v, r, pr.pos.w, c), a);
      const f3 d = ld3(r.probes[r.c[c + 1u].probe_off + q].pos) - a;
      const uint32_t kk = w_seg_samples(v, d, Lv);
      for (uint32_t i = j; i < kk; i += 4u)
        if (w_vox_occ(v, Lv, a + d * w_seg_t(i, kk))) { hid = true; break; }
    }
    const uint32_t hm = __ballot_sync(0xffffffffu, hid);
    if (j == 0u) w.parents[(size_t)(r.c[c].probe_off + pi) * 8u + k] = ((hm >> (lane & ~3u)) & 0xFu) ? W_NONE : q;
  }
}

// giBuild's steps after registerPixels, two to a launch where they are independent (the launch's blocks split between
// them): compact of cascade c, relocateVox and registerUp (both need only the compaction before them), linkParents
// (needs both cascades' probes in place).  A task's blocks see the task's own block index and count.
enum { W_NONE_TASK = 0, W_COMPACT = 1, W_RELOCATE = 2, W_REGISTER_UP = 3, W_LINK = 4 };
__device__ __forceinline__ void w_task(const RcDev &r, const VoxDev &v, const WorldDev &w, uint32_t task, uint32_t c,
                                       uint32_t bid, uint32_t nblk) {
  switch (task) {
    case W_COMPACT: w_compact(r, v, w, c); break;
    case W_RELOCATE:
      if (w.relocate == 2u) w_relocate_vox(r, v, w, c, bid, nblk);
      else w_relocate_gbuffer(r, w, c, bid, nblk);
      break;
    case W_REGISTER_UP: w_register_up(r, w, c, bid, nblk); break;
    case W_LINK: w_link_parents(r, v, w, c, bid, nblk); break;
    default: break;
  }
}
__global__ void __launch_bounds__(256) k_w_build(RcDev r, VoxDev v, WorldDev w, uint32_t ta, uint32_t ca, uint32_t na,
                                                 uint32_t tb, uint32_t cb, uint32_t nb) {
  grid_dep_wait();
  if (blockIdx.x < na) w_task(r, v, w, ta, ca, blockIdx.x, na);
  else w_task(r, v, w, tb, cb, blockIdx.x - na, nb);
}

// trace (rc.ts:600-622) of ray (pi, di) of a world probe of cascade c into atlas element i
template <int A, bool DYN>
__device__ __forceinline__ bool w_trace_ray(const RcDev &r, const VoxDev &v, uint32_t c, uint32_t pi, uint32_t di,
                                            size_t i, TraceOut &out) {
  typedef typename Atlas<A>::T T;
  out.rad = mk(0.0f, 0.0f, 0.0f); out.T = 1.0f; out.lvl = GI_EMPTY; out.ptr = GI_EMPTY; out.bit = 0; out.tin = 0;
  out.steps = 0;
  bool traced = false;
  const CascDev &L = r.c[c];
  const ProbeDev pr = r.probes[L.probe_off + pi];
  if (pr.pos.w > 0.0f) {
    const float4 dv = r.dirs[L.dir_off + di];
    const f3 dir = mk(dv.x, dv.y, dv.z);
    const float s0 = pr.pos.w, t0 = L.b0 * s0, t1 = L.b1 * s0;
    const f3 po = ld3(pr.pos), pn = ld3(pr.nrm);
    const uint32_t Lv = vox_level_for(v, r.plevel[L.probe_off + pi], po + dir * t1);
    const float vs = vox_size(v, Lv);
    const f3 ooff = po + pn * (r.vox_offset * vs);
    trace_vox(v, r.frame, r.unorm8, ooff, dir, t0, t1, r.vox_skip * vs, Lv, r.dda_cap, out, InjectedBounce{r.bn_inj},
              r.idirs + L.dir_off + di);
    if (DYN) dyn_compose(r, v, po, dir, t0, t1, ooff, 3.5449077f / (float)L.res, out);
    traced = true;
  }
  Atlas<A>::store(reinterpret_cast<T *>(r.rad), i, make_float4(out.rad.x, out.rad.y, out.rad.z, out.T));
  if (r.hits) r.hits[i] = make_uint4(out.lvl, out.ptr, out.bit, out.tin);
  if (r.rad_traced) Atlas<A>::store(reinterpret_cast<T *>(r.rad_traced), i, make_float4(out.rad.x, out.rad.y, out.rad.z, out.T));
  return traced;
}

// Persistent trace over the rays of every cascade's live probes (first rays in state[16 ..]), probe-major
template <int A, bool DYN>
__global__ void __launch_bounds__(256) k_w_trace(RcDev r, VoxDev v, WorldDev w, uint32_t *ray_counter) {
  grid_dep_wait();
  __shared__ uint32_t s_first[9];
  if (threadIdx.x <= r.cascades) s_first[threadIdx.x] = w.state[16 + threadIdx.x];
  __syncthreads();
  const uint32_t lane = threadIdx.x & 31u, total = s_first[r.cascades], per = 32u * r.trace_rays;
  uint32_t steps_acc = 0, traces_acc = 0, cap_acc = 0, cur_c = 0xffffffffu;
  for (;;) {
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(ray_counter, per);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= total) break;
    for (uint32_t k = 0; k < r.trace_rays; k++) {
      const uint32_t j0 = base + k * 32u + lane;
      const bool live = j0 < total;
      const uint32_t j = live ? total - 1u - j0 : 0u;   // the top cascade first: the queue ends on the shortest walks
      uint32_t c = 0;
      for (uint32_t q = 1; q < r.cascades; q++)
        if (j >= s_first[q]) c = q;
      TraceOut out;
      out.steps = 0;
      bool traced = false;
      if (live) {
        const CascDev &L = r.c[c];
        const uint32_t t = j - s_first[c];
        traced = w_trace_ray<A, DYN>(r, v, c, t >> L.dirs_log2, t & ((1u << L.dirs_log2) - 1u), (size_t)L.rad_off + t, out);
      }
      if (r.stats && live && traced) {   // per-cascade counters (rc.ts:232-235)
        if (c != cur_c && cur_c != 0xffffffffu) {
          atomicAdd(&r.counts[24 + cur_c], traces_acc); atomicAdd(&r.counts[32 + cur_c], steps_acc);
          atomicAdd(&r.counts[64 + cur_c], cap_acc);
          traces_acc = steps_acc = cap_acc = 0;
        }
        cur_c = c;
        traces_acc++; steps_acc += out.steps; cap_acc += out.steps >= r.dda_cap ? 1u : 0u;
      }
    }
  }
  if (r.stats) {
    const unsigned grp = __match_any_sync(0xffffffffu, cur_c);
    const uint32_t tr = __reduce_add_sync(grp, traces_acc), sp = __reduce_add_sync(grp, steps_acc);
    const uint32_t cp = __reduce_add_sync(grp, cap_acc);
    if (cur_c != 0xffffffffu && (uint32_t)(__ffs(grp) - 1) == lane) {
      atomicAdd(&r.counts[24 + cur_c], tr); atomicAdd(&r.counts[32 + cur_c], sp); atomicAdd(&r.counts[64 + cur_c], cp);
    }
  }
}

// mergeWorld (rc.ts:688-708) of cascade c in place, one thread per (probe, direction): the mean of the parents'
// upperAvg (rc.ts:681-686, the 2x2 texel block when the cascade above has twice the resolution)
template <int A>
__global__ void __launch_bounds__(256) k_w_merge(RcDev r, WorldDev w, uint32_t c) {
  grid_dep_wait();
  typedef typename Atlas<A>::T T;
  T *rad = reinterpret_cast<T *>(r.rad);
  const CascDev &L = r.c[c];
  const float *F = r.frame;
  const uint32_t n = w.state[8 + c] << L.dirs_log2;
  const bool has_up = c + 1u < r.cascades;
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const uint32_t pi = t >> L.dirs_log2, di = t & ((1u << L.dirs_log2) - 1u);
    const size_t idx = (size_t)L.rad_off + t;
    const float4 vv = Atlas<A>::load(rad, idx);
    f3 up = mk(F[F_SKY], F[F_SKY + 1], F[F_SKY + 2]);
    if (has_up && vv.w > 0.0f) {
      const CascDev &U = r.c[c + 1u];
      const uint32_t u0 = di % L.res, v0 = di / L.res;
      const uint4 *pp = reinterpret_cast<const uint4 *>(w.parents + (size_t)(L.probe_off + pi) * 8u);
      const uint4 pa = pp[0], pb = pp[1];
      const uint32_t par[8] = {pa.x, pa.y, pa.z, pa.w, pb.x, pb.y, pb.z, pb.w};
      f3 acc = mk(0.0f, 0.0f, 0.0f);
      float ws = 0.0f;
#pragma unroll
      for (uint32_t k = 0; k < 8u; k++) {
        const uint32_t q = par[k];
        if (q == W_NONE) continue;
        f3 ua;
        if (U.res == L.res) {
          const float4 a = Atlas<A>::load(rad, (size_t)U.rad_off + ((size_t)q << U.dirs_log2) + v0 * U.res + u0);
          ua = mk(a.x, a.y, a.z);
        } else {
          const size_t b0 = (size_t)U.rad_off + ((size_t)q << U.dirs_log2) + (size_t)v0 * 2u * U.res + u0 * 2u;
          const float4 a = Atlas<A>::load(rad, b0), b = Atlas<A>::load(rad, b0 + 1u);
          const float4 cc = Atlas<A>::load(rad, b0 + U.res), d = Atlas<A>::load(rad, b0 + U.res + 1u);
          ua = (((mk(a.x, a.y, a.z) + mk(b.x, b.y, b.z)) + mk(cc.x, cc.y, cc.z)) + mk(d.x, d.y, d.z)) * 0.25f;
        }
        acc = acc + ua;
        ws += 1.0f;
      }
      up = ws > 0.0f ? acc / mx(ws, 1.0f) : mk(0.0f, 0.0f, 0.0f);
    }
    const f3 m = fma3(up, vv.w, mk(vv.x, vv.y, vv.z));
    Atlas<A>::store(rad, idx, make_float4(m.x, m.y, m.z, 1.0f));
  }
}

// histHash (rc.ts:784-786)
__device__ __forceinline__ uint32_t w_hist_hash(int4 g) {
  return w_hash32(((uint32_t)g.x * 73856093u) ^ ((uint32_t)g.y * 19349663u) ^ ((uint32_t)g.z * 83492791u) ^
                  ((uint32_t)g.w * 2654435761u));
}

// projectSH (rc.ts:752-774) of the c0 world probes, one thread per probe, with histBlend (rc.ts:787-812): the SH mixed
// half and half with the SH the probe at the same grid point and LOD stored in the previous solve
template <int A>
__global__ void __launch_bounds__(256) k_w_project_sh(RcDev r, WorldDev w) {
  grid_dep_wait();
  typedef typename Atlas<A>::T T;
  const T *rad = reinterpret_cast<const T *>(r.rad);
  const CascDev &L0 = r.c[0];
  const float *F = r.frame;
  const uint32_t n = w.state[8], cap = w.cap[0], H = w.hist_h, cur = w.state[0], prv = cur ^ 1u;
  for (uint32_t pi = blockIdx.x * blockDim.x + threadIdx.x; pi < n; pi += gridDim.x * blockDim.x) {
    f3 cf[9];
#pragma unroll
    for (int k = 0; k < 9; k++) cf[k] = mk(0.0f, 0.0f, 0.0f);
    for (uint32_t d = 0; d < 16u; d++) {
      const float4 rv = Atlas<A>::load(rad, (size_t)L0.rad_off + (size_t)pi * 16u + d);
      const f3 rr = mk(rv.x, rv.y, rv.z) * F[F_OMEGA + d];
      const float4 dv = r.dirs[L0.dir_off + d];
      float y[9];
      sh_basis(mk(dv.x, dv.y, dv.z), y);
#pragma unroll
      for (int k = 0; k < 9; k++) cf[k] = fma3(rr, y[k], cf[k]);
    }
    float vals[32];
#pragma unroll
    for (int k = 0; k < 32; k++) vals[k] = 0.0f;
    const float a0 = GI_PI, a1 = 2.0f * GI_PI / 3.0f, a2 = GI_PI / 4.0f;
#pragma unroll
    for (int k = 0; k < 9; k++) {
      const float a = k == 0 ? a0 : (k < 4 ? a1 : a2);
      vals[k * 3 + 0] = cf[k].x * a; vals[k * 3 + 1] = cf[k].y * a; vals[k * 3 + 2] = cf[k].z * a;
    }
    const int4 g = r.probes[L0.probe_off + pi].grid;
    const uint32_t h0 = w_hist_hash(g) & (H - 1u);
    uint32_t h = h0, found = W_NONE;
    for (uint32_t i = 0; i < 64u; i++) {
      const uint32_t sl = w.hist_tab[prv * H + h];
      if (sl == 0u) break;
      const int4 og = w.hist_grid[(size_t)prv * cap + (sl - 1u)];
      if (og.x == g.x && og.y == g.y && og.z == g.z && og.w == g.w) { found = sl - 1u; break; }
      h = (h + 1u) & (H - 1u);
    }
    if (found != W_NONE) {
      const float4 *hs = w.hist_sh + ((size_t)prv * cap + found) * 8u;
#pragma unroll
      for (int q = 0; q < 8; q++) {
        const float4 o = hs[q];
        vals[4 * q] = o.x * (1.0f - 0.5f) + vals[4 * q] * 0.5f;
        vals[4 * q + 1] = o.y * (1.0f - 0.5f) + vals[4 * q + 1] * 0.5f;
        vals[4 * q + 2] = o.z * (1.0f - 0.5f) + vals[4 * q + 2] * 0.5f;
        vals[4 * q + 3] = o.w * (1.0f - 0.5f) + vals[4 * q + 3] * 0.5f;
      }
    }
    w.hist_grid[(size_t)cur * cap + pi] = g;
    h = h0;
    for (uint32_t i = 0; i < 64u; i++) {
      if (atomicCAS(&w.hist_tab[cur * H + h], 0u, pi + 1u) == 0u) break;
      h = (h + 1u) & (H - 1u);
    }
    float4 *hd = w.hist_sh + ((size_t)cur * cap + pi) * 8u;
#pragma unroll
    for (uint32_t q = 0; q < 8u; q++) {
      float4 val = make_float4(vals[4 * q], vals[4 * q + 1], vals[4 * q + 2], vals[4 * q + 3]);
      if (r.f32_out) {
        reinterpret_cast<float4 *>(r.sh)[(size_t)pi * 8u + q] = val;
      } else {
        Atlas<A>::store(reinterpret_cast<T *>(r.sh), (size_t)pi * 8u + q, val);
        val = make_float4(Atlas<A>::round(val.x), Atlas<A>::round(val.y), Atlas<A>::round(val.z), Atlas<A>::round(val.w));
      }
      hd[q] = val;
    }
  }
}

template <int A>
__device__ __forceinline__ f3 w_eval_sh(const RcDev &r, uint32_t qi, const float y[9]) {
  float v[32];
#pragma unroll
  for (int j = 0; j < 8; j++) {
    const float4 sc = sh_load<A>(r, (size_t)qi * 8u + j);
    v[4 * j] = sc.x; v[4 * j + 1] = sc.y; v[4 * j + 2] = sc.z; v[4 * j + 3] = sc.w;
  }
  f3 es = mk(0.0f, 0.0f, 0.0f);
#pragma unroll
  for (int k = 0; k < 9; k++) es = fma3(mk(v[3 * k], v[3 * k + 1], v[3 * k + 2]), y[k], es);
  return vmax(es, mk(0.0f, 0.0f, 0.0f));
}

// The L0 and L1 coefficients (basis order 0, y, z, x) of a probe's stored SH, added with weight wt (shL1 + shAdd,
// rc.ts:831-840)
template <int A>
__device__ __forceinline__ void w_sh_l1_add(const RcDev &r, uint32_t qi, float wt, f3 &c0, f3 &cy, f3 &cz, f3 &cx) {
  const float4 a = sh_load<A>(r, (size_t)qi * 8u), b = sh_load<A>(r, (size_t)qi * 8u + 1u),
               c = sh_load<A>(r, (size_t)qi * 8u + 2u);
  c0 = fma3(mk(a.x, a.y, a.z), wt, c0);
  cy = fma3(mk(a.w, b.x, b.y), wt, cy);
  cz = fma3(mk(b.z, b.w, c.x), wt, cz);
  cx = fma3(mk(c.y, c.z, c.w), wt, cx);
}

// toonReceive (style.ts:30-42): from L0 an ambient colour, from the luminance gradient of L1 a dominant direction d
// and its directional colour, the direction put through a two-band ramp (smoothstep of half width soft, or a step):
// E = max(amb - dir + 2 dir ramp(n . d), 0); band = n . d > 0; contrast = lum(dir) / max(lum(amb), 1e-6)
struct ToonRecv { f3 e; float band, contrast; };
__device__ __forceinline__ ToonRecv toon_receive(f3 c0, f3 c1y, f3 c1z, f3 c1x, f3 n, float soft) {
  const f3 lw = mk(0.2126f, 0.7152f, 0.0722f);
  const f3 amb = c0 * 0.282095f;
  const f3 g = mk(dot(c1x, lw), dot(c1y, lw), dot(c1z, lw));
  const float gl = length3(g);
  ToonRecv out;
  if (gl < 1e-6f) { out.e = vmax(amb, mk(0.0f, 0.0f, 0.0f)); out.band = 0.0f; out.contrast = 0.0f; return out; }
  const f3 d = g / gl;
  const f3 dir = vmax(((c1x * d.x + c1y * d.y) + c1z * d.z) * 0.488603f, mk(0.0f, 0.0f, 0.0f));
  const float x = dot(n, d);
  float ramp;
  if (soft > 0.0f) {
    const float t = fclampf((x - -soft) / (soft - -soft), 0.0f, 1.0f);
    ramp = t * t * (3.0f - 2.0f * t);
  } else {
    ramp = x > 0.0f ? 1.0f : 0.0f;
  }
  out.e = vmax((amb - dir) + (dir * 2.0f) * ramp, mk(0.0f, 0.0f, 0.0f));
  out.band = x > 0.0f ? 1.0f : 0.0f;
  out.contrast = dot(dir, lw) / mx(dot(amb, lw), 1e-6f);
  return out;
}

// gatherWorld (rc.ts:880-927), one thread per pixel: the eight c0 probes of the pixel's grid cell, weighted
// trilinearly and by the side of the surface they are on; with relocate 'voxel' the probes voxels hide are skipped
// (retested from two voxels out when every probe is hidden).  Photoreal pixels left black count in words 72-79.
// TAG (once the G-buffer carries style tags): toon pixels (tag > 0.75) also interpolate the L0/L1 coefficients and
// go through the receiving operator (the irradiance replaced when the frame's style.y > 0.5), alpha 2 + band + 2 when
// the directional part is at least a tenth of the ambient; other tagged pixels (tag > 0.25) get alpha 2.
template <int A, bool TAG>
__global__ void __launch_bounds__(256) k_w_gather(RcDev r, VoxDev v, WorldDev w) {
  grid_dep_wait();
  // a warp takes a 4 x 8 tile of the block's 16 x 16 pixels (neighbouring pixels share probes and segment lengths;
  // 0.378 ms on the colonnade with 16 x 2 rows, 0.360 with 8 x 4 tiles, 0.354 with 4 x 8, 0.360 with 2 x 16)
  const uint32_t lane = threadIdx.x & 31u, wp = threadIdx.x >> 5;
  const uint32_t px = blockIdx.x * 16u + (wp & 3u) * 4u + (lane & 3u), py = blockIdx.y * 16u + (wp >> 2) * 8u + (lane >> 2);
  if (px >= r.width || py >= r.height) return;
  const size_t q = (size_t)py * r.width + px;
  const float *F = r.frame;
  const float d = r.depth[q];
  f3 res = mk(0.0f, 0.0f, 0.0f);
  float alpha = 0.0f;
  bool black = false;
  if (d > 0.0f) {
    alpha = 1.0f;
    const f3 x = world_at(F, (int)px, (int)py, d);
    const uint2 nn = r.normal[q];
    const f3 n = mk(h2f(nn.x & 0xffffu), h2f(nn.x >> 16), h2f(nn.y & 0xffffu));
    const int lod = w_lod_for(F, length3(x - mk(F[F_EYE], F[F_EYE + 1], F[F_EYE + 2])));
    const float s0 = w_spacing(F, lod, 0u);
    const f3 gp = mk(x.x / s0, x.y / s0, x.z / s0);
    const i3 bb = vfloori(gp), org0 = w_origin(F, s0);
    const f3 f = gp - vi2f(bb);
    const uint32_t Lo = vox_level_for(v, vox_level(v, r, s0, 0u), x);
    const f3 xo1 = x + n * (1.0f * vox_size(v, Lo));
    float y[9];
    sh_basis(n, y);
    f3 e = mk(0.0f, 0.0f, 0.0f);
    float ws = 0.0f, ww[8];
    uint32_t hidden = 0, qq[8];
    const bool vrel = w.relocate == 2u;
    const float tagA = TAG ? r.unorm8[r.tag[q]] : 0.0f;
    const bool toon = TAG && tagA > 0.75f;
    f3 l0 = mk(0.0f, 0.0f, 0.0f), ly = l0, lz = l0, lx = l0;   // toon pixels: the L0 / L1 sums
    for (uint32_t k = 0; k < 8u; k++) {
      const i3 o = w_corner(k);
      const uint32_t qi = w_lookup(w, 0u, w_key_at(mki(bb.x + o.x, bb.y + o.y, bb.z + o.z), org0, lod));
      if (qi == W_NONE) continue;
      const f3 tw = mk(o.x == 1 ? f.x : 1.0f - f.x, o.y == 1 ? f.y : 1.0f - f.y, o.z == 1 ? f.z : 1.0f - f.z);
      const f3 pp = ld3(r.probes[r.c[0].probe_off + qi].pos);
      const f3 dv = pp - x;
      const float side = dot(n, dv) / mx(length3(dv), 1e-5f);
      const float wt = (tw.x * tw.y * tw.z + 1e-4f) * ((side + 1.0f) * (side + 1.0f) * 0.25f + 0.02f);
      if (vrel && w_seg_occluded(v, xo1, pp, Lo)) { hidden |= 1u << k; ww[k] = wt; qq[k] = qi; continue; }
      e = fma3(w_eval_sh<A>(r, qi, y), wt, e);
      ws += wt;
      if (toon) w_sh_l1_add<A>(r, qi, wt, l0, ly, lz, lx);
    }
    if (ws <= 0.0f && hidden != 0u) {
      const f3 xo2 = x + n * (2.0f * vox_size(v, Lo));
      for (uint32_t k = 0; k < 8u; k++) {
        if ((hidden & (1u << k)) == 0u) continue;
        if (w_seg_occluded(v, xo2, ld3(r.probes[r.c[0].probe_off + qq[k]].pos), Lo)) continue;
        e = fma3(w_eval_sh<A>(r, qq[k], y), ww[k], e);
        ws += ww[k];
        if (toon) w_sh_l1_add<A>(r, qq[k], ww[k], l0, ly, lz, lx);
      }
    }
    black = ws <= 0.0f && hidden != 0u && tagA <= 0.25f;
    if (ws > 0.0f) res = e / ws;
    if (TAG) {
      if (toon && ws > 0.0f) {
        const float iw = 1.0f / ws;
        const ToonRecv tr = toon_receive(l0 * iw, ly * iw, lz * iw, lx * iw, n, F[F_STYLE + 2]);
        if (F[F_STYLE + 1] > 0.5f) res = tr.e;
        alpha = 2.0f + tr.band + (tr.contrast >= 0.1f ? 2.0f : 0.0f);
      } else if (toon || tagA > 0.25f) {
        alpha = 2.0f;
      }
    }
  }
  // black pixels: one atomic per counter word among the warp's lanes
  const unsigned act = __activemask();
  const unsigned grp = __match_any_sync(act, black ? (px & 7u) : 8u);
  if (black && (uint32_t)(__ffs(grp) - 1) == (threadIdx.x & 31u)) atomicAdd(&r.counts[72 + (px & 7u)], (uint32_t)__popc(grp));
  if ((A == GI_ATLAS_F32 || r.f32_out) && !r.irr_f16) reinterpret_cast<float4 *>(r.irr)[q] = make_float4(res.x, res.y, res.z, alpha);
  else reinterpret_cast<uint2 *>(r.irr)[q] = make_uint2((uint32_t)f2h(res.x) | ((uint32_t)f2h(res.y) << 16),
                                                       (uint32_t)f2h(res.z) | ((uint32_t)f2h(alpha) << 16));
}

// One world-probe solve (Rc.encode, rc.ts:1180-1221): giBuild (clear .. linkParents), giTrace (the bounce volume, the
// trace), giMerge (mergeWorld N-1 .. 0, projectSH), giGather
template <int A>
static cudaError_t launch_world(const RcDev &r, const VoxDev &v, const WorldDev &w, uint32_t sm_count, cudaStream_t st,
                                cudaEvent_t *ev, const RcLaunch *ls, const BounceDev *bn) {
  uint32_t *counter = r.counts + 80;
  const uint32_t persist = sm_count * 8u, N = r.cascades;
  auto blocks = [&](uint64_t n) {
    const uint64_t b = (n + 255u) / 256u;
    return (uint32_t)(b < 1u ? 1u : (b > persist ? persist : b));
  };
  if (ev) cudaEventRecord(ev[0], st);
  const uint32_t clear_n = max(max(w.hash_total, w.look_total), max(w.hist_h, 96u));
  GI_TRY(gi_launch(k_w_clear, blocks(clear_n), 256, st, r, w));
  GI_TRY(gi_launch(k_w_register_pixels, (r.width * r.height + 255u) / 256u, 256, st, r, w));
  // blocks of each task (compact: one per 2048 slots; the others grid-stride over the probes' warps or threads)
  auto nb_compact = [&](uint32_t c) { return (w.hash_mask[c] + W_COMPACT_SLOTS) / W_COMPACT_SLOTS; };
  auto nb_warps = [&](uint32_t c) { return blocks((uint64_t)w.cap[c] * 32u); };
  auto nb_up = [&](uint32_t c) { return blocks((uint64_t)w.cap[c - 1u] * 8u); };
  auto pair = [&](uint32_t ta, uint32_t ca, uint32_t na, uint32_t tb, uint32_t cb, uint32_t nb) {
    return gi_launch(k_w_build, na + nb, 256, st, r, v, w, ta, ca, na, tb, cb, nb);
  };
  const bool rel = w.relocate != 1u;   // 'gbuffer' and 'voxel' relocate in a step of their own
  // compact(c) waits on registerUp(c); relocateVox(c) and registerUp(c + 1) wait on compact(c) only; linkParents(c - 1)
  // waits on compact(c) and on relocateVox(c - 1) and (c); so each launch pairs two steps that share their inputs
  GI_TRY(pair(W_COMPACT, 0, nb_compact(0), W_NONE_TASK, 0, 0));
  for (uint32_t c = 0; c < N; c++) {
    const bool up = c + 1u < N;
    if (rel) {
      GI_TRY(pair(W_RELOCATE, c, nb_warps(c), up ? W_REGISTER_UP : W_NONE_TASK, c + 1u, up ? nb_up(c + 1u) : 0u));
      if (up) GI_TRY(pair(W_COMPACT, c + 1u, nb_compact(c + 1u), c >= 1u ? W_LINK : W_NONE_TASK, c - 1u, c >= 1u ? nb_warps(c - 1u) : 0u));
    } else {
      if (up) GI_TRY(pair(W_REGISTER_UP, c + 1u, nb_up(c + 1u), c >= 1u ? W_LINK : W_NONE_TASK, c - 1u, c >= 1u ? nb_warps(c - 1u) : 0u));
      if (up) GI_TRY(pair(W_COMPACT, c + 1u, nb_compact(c + 1u), W_NONE_TASK, 0, 0));
    }
  }
  if (N >= 2) GI_TRY(pair(W_LINK, N - 2u, nb_warps(N - 2u), W_NONE_TASK, 0, 0));
  if (ev) cudaEventRecord(ev[1], st);
  if (bn) GI_TRY(launch_bounce(*bn, v, r, sm_count, st));
  const uint32_t tb = sm_count * (ls ? ls->trace_blocks : 8u);
  if (r.dyn_hdr) GI_TRY(gi_launch(k_w_trace<A, true>, tb, 256, st, r, v, w, counter));
  else GI_TRY(gi_launch(k_w_trace<A, false>, tb, 256, st, r, v, w, counter));
  if (ev) cudaEventRecord(ev[2], st);
  for (int c = (int)N - 1; c >= 0; c--)
    GI_TRY(gi_launch(k_w_merge<A>, blocks((uint64_t)w.cap[c] << r.c[c].dirs_log2), 256, st, r, w, (uint32_t)c));
  GI_TRY(gi_launch(k_w_project_sh<A>, blocks(w.cap[0]), 256, st, r, w));
  if (ev) cudaEventRecord(ev[3], st);
  if (r.tag_any) GI_TRY(gi_launch(k_w_gather<A, true>, dim3((r.width + 15u) / 16u, (r.height + 15u) / 16u), 256, st, r, v, w));
  else GI_TRY(gi_launch(k_w_gather<A, false>, dim3((r.width + 15u) / 16u, (r.height + 15u) / 16u), 256, st, r, v, w));
  if (ev) cudaEventRecord(ev[4], st);
  return cudaGetLastError();
}
