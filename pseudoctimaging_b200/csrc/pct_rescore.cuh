// Exact FP32 rescoring of the learned form (EXEC_CHOICE 7): the device code of the proposal
// rescoring (rows of 4 x 4 blocks sharing one proposal) and of the no-network centre prior.
//
// This text is compiled twice:
//  * by the library build, included inside its namespace: the volume's x extent and the atlas
//    row pitch are kernel arguments;
//  * at run time by NVRTC, once per (device, x extent, pitch, window), with PCT_RS_NX,
//    PCT_RS_PITCH and PCT_RS_HW defined and PCT_RS_JIT selecting the extern "C" entry points at
//    the end. Both strides are
//    then constants, so each of an offset's 22 tap loads is one base address plus an immediate
//    (the run-time strides cost about 45 % of the instructions in address arithmetic).
// So it includes nothing, opens no namespace and uses CUDA built-ins only.
//
// Work items: one warp = 4 x-rows of one z plane x 32 lanes along y (lanes 1..30 own output
// voxels, lanes 0 and 31 carry the y halo); the 4 warps of a CTA take the 4 z planes of one
// 4 x 4 (z, x) block, which share a proposal and most of their atlas footprint in L1. The last
// item of an x band is shifted back to end at the last interior row, the rows the previous item
// owns left out, so no load needs a clamp. Needs at least 4 interior x-rows and an atlas volume
// below 2^31 elements (32-bit offsets). The z-pair entry points (pct_rescore8_*, 2 or more
// interior planes) give a warp the same 4 x-rows in two consecutive planes of a block: the two
// patches share two of their three atlas planes, so an offset takes 24 tap loads for 8 rows
// instead of 36 (learned step at 222x222x112, 10 atlases, k = 32: 5.19 ms against 5.31 with the
// one-plane items; 96 registers at 5 CTAs per SM; 4 CTAs 5.33 ms, 6 CTAs 5.24 with spills).
//
// Per offset the 3 z x 6 x tap rows the 4 rows need are loaded once, D = (s A - s I)^2 (the
// weight scale s folded into the differences, x-rows in pairs on packed FP32 FMAs), z summed in
// registers, x across the rows and y by warp shuffles, w = 2^-SSD', P += w * CT, W += w: the
// plain kernel's arithmetic (the reference's PatchSimilarity and weighted sums,
// NewPatchedBrainPureC.cpp:1184-1212,1350-1449), over the kept offsets only.

// Offsets in flight per warp (unroll of the offset loop) and CTAs per SM, measured on the learned
// step at 222x222x112, 10 atlases, k = 32. Constant strides: one offset at 7 CTAs (72 registers)
// 5.33 ms; 1/6 5.55, 1/8 5.63, 2/6 5.44, 2/7 5.66, 2/4 5.59, 3/4 5.52, 3/6 5.75. Run-time
// strides (the library build; its address registers need 128): one offset at 4 CTAs 6.28 ms,
// two 6.44.
#ifndef PCT_RS_UNROLL
#define PCT_RS_UNROLL 1
#endif
#ifndef PCT_RS_MIN_CTAS
#define PCT_RS_MIN_CTAS 7  // of the run-time compiled entry points
#endif
#ifndef PCT_RS_MIN_CTAS8
#define PCT_RS_MIN_CTAS8 5  // of the run-time compiled z-pair entry points (measured above)
#endif
#ifndef PCT_RS_UNROLL8
#define PCT_RS_UNROLL8 1  // offsets in flight per warp of the z-pair items
#endif
// z-pair entry points, offsets in flight / CTAs per SM (learned step, same workload): 1/5 5.20
// ms, 2/4 5.29, 2/5 5.60, 1/6 5.24 (spills).

constexpr int kRsAxis = 11;       // offsets per axis of the NH = 11 window
constexpr int kRsTopK = 32;       // the largest kept set (level 4)
constexpr int kRowOut = 30;       // output voxels per warp row (lanes 1..30)
constexpr int kRescoreWarps = 4;  // warps per CTA
constexpr int kRows = 4;          // x-rows per warp item (the block edge)
constexpr int kMaxPrior = 125;    // offsets of the no-network prior (5 x 5 x 5 around the centre)
constexpr int kRsUnroll = PCT_RS_UNROLL;
constexpr int kRsUnroll8 = PCT_RS_UNROLL8;
static_assert(kRescoreWarps == kRows, "a CTA's warps cover the z planes of one block");

// The proposal of one row segment (30 voxels along y) of a block anchor row: the 4 most probable
// offsets per axis (index 0..10) and each voxel's probability mass on the kept rank triples.
struct RowProp {
  signed char top[12];  // [axis][rank]
  float conf[kRowOut];  // per output voxel of the segment (lane - 1)
};

// The plain kernel's tile grid, for skipping the items of tiles that fell back to it.
struct RescoreTiles {
  int zt, xc, tiles_x, tiles_y;
};

// The no-network prior's offsets as 32-bit element offsets into an atlas volume.
struct PriorList {
  int n;
  int off[kMaxPrior];
};

// The kept set's rank triples (i, j, k), i + j + k <= 4, packed as i | j << 2 | k << 4, in order
// of rank sum: the first 10, 20 or 32 are the kept sets of levels 2, 3 and 4.
__constant__ unsigned char kRankTriples[kRsTopK] = {
    0x00, 0x01, 0x04, 0x10, 0x02, 0x05, 0x08, 0x11, 0x14, 0x20, 0x03, 0x06, 0x09, 0x0c, 0x12, 0x15,
    0x18, 0x21, 0x24, 0x30, 0x07, 0x0a, 0x0d, 0x13, 0x16, 0x19, 0x1c, 0x22, 0x25, 0x28, 0x31, 0x34};

__device__ __forceinline__ float rs_ex2(float x) {
  float r;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ int pick4(const int (&t)[4], int i) {
  return i == 0 ? t[0] : i == 1 ? t[1] : i == 2 ? t[2] : t[3];
}

// One offset for the 4 rows of a warp item. `a` points at the atlas voxel (z - 1 + dw, x0 - 1 +
// du, yc + dv), `l` at the label voxel (z + dw, x0 + du, yc + dv). MASKED: only the rows set in
// `take` accumulate (the full-search path, whose rows differ in which offsets they keep);
// otherwise every row accumulates and the caller stores only the rows it owns.
template <bool MASKED>
__device__ __forceinline__ void eval_offset4(const float *__restrict__ a,
                                             const float *__restrict__ l,
                                             const float2 (&in)[3][(kRows + 2) / 2], int axy,
                                             int apitch, unsigned take, float2 s2,
                                             float (&P)[kRows], float (&W)[kRows]) {
  // x-rows in pairs: packed FP32 FMAs (the same roundings as two scalar FMAs)
  float Z[kRows + 2];
#pragma unroll
  for (int xp = 0; xp < (kRows + 2) / 2; ++xp) {
    const int ro = 2 * xp * apitch;
    float2 z = make_float2(0.f, 0.f);
#pragma unroll
    for (int dz = 0; dz < 3; ++dz) {
      const float2 av = make_float2(__ldg(a + (ro + dz * axy)), __ldg(a + (ro + apitch + dz * axy)));
      const float2 t = __ffma2_rn(av, s2, in[dz][xp]);
      z = __ffma2_rn(t, t, z);
    }
    Z[2 * xp] = z.x;
    Z[2 * xp + 1] = z.y;
  }
#pragma unroll
  for (int r = 0; r < kRows; ++r) {
    const float x = Z[r] + Z[r + 1] + Z[r + 2];
    const float e =
        __shfl_up_sync(0xffffffffu, x, 1) + x + __shfl_down_sync(0xffffffffu, x, 1);
    if (!MASKED || ((take >> r) & 1u)) {
      const float w = rs_ex2(-e);
      P[r] = fmaf(w, __ldg(l + r * apitch), P[r]);
      W[r] += w;
    }
  }
}

// The placement of one warp item and its input taps.
struct RsItem {
  int z, xb, x0, seg, bx, y;
  bool out;  // the lane owns an output voxel of the segment
  unsigned owned, take;
};

// Item `it` of the interior grid (first interior index lo): false when its z plane lies past
// the interior.
__device__ __forceinline__ bool rs_place(long long it, int nx, int ny, int nz, int lo, int segs,
                                         int nbx, int lane, RsItem &t) {
  const long long r0 = it / kRows;
  t.seg = (int)(r0 % segs);
  const long long r1 = r0 / segs;
  t.bx = (int)(r1 % nbx);
  t.z = (int)(r1 / nbx) * kRows + (int)(it % kRows) + lo;
  if (t.z >= nz - lo) return false;
  t.xb = lo + t.bx * kRows;
  t.x0 = min(t.xb, nx - lo - kRows);
  t.y = lo + t.seg * kRowOut - 1 + lane;
  t.out = lane >= 1 && lane <= kRowOut && t.y < ny - lo;
  t.owned = 0;
#pragma unroll
  for (int r = 0; r < kRows; ++r)
    if (t.x0 + r >= t.xb) t.owned |= 1u << r;
  t.take = t.out ? t.owned : 0u;
  return true;
}

// Input taps I(z + dz - 1, x0 - 1 + xr, yc), negated and scaled, x-rows in pairs.
__device__ __forceinline__ void rs_inputs(const float *__restrict__ img, int nx, int ny,
                                          const RsItem &t, int yc, float scale,
                                          float2 (&in)[3][(kRows + 2) / 2]) {
  const long long nxy = (long long)nx * ny;
#pragma unroll
  for (int dz = 0; dz < 3; ++dz)
#pragma unroll
    for (int xp = 0; xp < (kRows + 2) / 2; ++xp) {
      const float *pi = img + (long long)(t.z + dz - 1) * nxy + (long long)(t.x0 - 1 + 2 * xp) * ny + yc;
      in[dz][xp] = make_float2(-__ldg(pi) * scale, -__ldg(pi + ny) * scale);
    }
}

__device__ __forceinline__ void rs_store(const RsItem &t, int nx, int ny, const float (&P)[kRows],
                                         const float (&W)[kRows], float *__restrict__ pacc,
                                         float *__restrict__ wacc) {
  const long long nxy = (long long)nx * ny;
#pragma unroll
  for (int r = 0; r < kRows; ++r)
    if ((t.take >> r) & 1u) {
      const long long v = (long long)t.z * nxy + (long long)(t.x0 + r) * ny + t.y;
      pacc[v] += P[r];
      wacc[v] += W[r];
    }
}

// Rescoring of the kept offsets of each row segment's block proposal (LEVEL 2, 3, 4: 10, 20 or
// 32 rank triples) for the NH = 2 hw + 1 window (hw 3, 4 or 5; the interior starts at hw + 1).
// A voxel whose confidence is below conf_thr sends its item through all NH^3 offsets (rows keep what the proposal kept, or everything for the low-confidence voxels);
// items of tiles flagged in tile_flag were left to the plain kernel and are skipped.
template <int LEVEL>
__device__ __forceinline__ void rescore4_body(
    const RowProp *__restrict__ props, const float *__restrict__ img, const float *__restrict__ atl,
    const float *__restrict__ lab, int nx, int ny, int nz, int apitch, float scale, float conf_thr,
    float *__restrict__ pacc, float *__restrict__ wacc, unsigned long long *__restrict__ fallbacks,
    unsigned long long *__restrict__ evaluated, const unsigned char *__restrict__ tile_flag,
    const RescoreTiles ts, int hw) {
  __shared__ int s_off[kRescoreWarps][kRsTopK];  // per warp: the item's kept offsets, 32-bit
#ifdef PCT_RS_NX
  nx = PCT_RS_NX;
#endif
#ifdef PCT_RS_PITCH
  apitch = PCT_RS_PITCH;
#endif
#ifdef PCT_RS_HW
  hw = PCT_RS_HW;
#endif
  const int lane = threadIdx.x & 31;
  int *w_off = s_off[threadIdx.x >> 5];
  const int lo = hw + 1;  // first interior index of the NH = 2 hw + 1 window
  const int ix = nx - 2 * lo, iz = nz - 2 * lo, iy = ny - 2 * lo;
  if (ix < kRows || iy <= 0 || iz <= 0) return;
  const int segs = (iy + kRowOut - 1) / kRowOut;
  const int nbx = (ix + kRows - 1) / kRows;
  const long long items = (long long)((iz + kRows - 1) / kRows) * kRows * nbx * segs;
  const int axy = nx * apitch;
  unsigned long long my_fallbacks = 0, my_evals = 0;
  for (long long it = (long long)blockIdx.x * kRescoreWarps + (threadIdx.x >> 5); it < items;
       it += (long long)gridDim.x * kRescoreWarps) {
    RsItem t;
    if (!rs_place(it, nx, ny, nz, lo, segs, nbx, lane, t)) continue;
    // items of tiles that fell back to the plain kernel are left to it (warp-uniform)
    if (tile_flag &&
        tile_flag[((t.z - lo) / ts.zt * ts.tiles_x + (t.xb - lo) / ts.xc) * ts.tiles_y + t.seg])
      continue;
    const int yc = min(t.y, ny - lo);
    const RowProp &rp = props[((long long)((t.z - lo) / kRows) * nbx + t.bx) * segs + t.seg];
    int top[3][4];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int r = 0; r < 4; ++r) top[a][r] = rp.top[a * 4 + r];
    // lane c: the offset of kept triple c
    {
      const int code = kRankTriples[lane];
      const int dw = pick4(top[0], code & 3) - 5, du = pick4(top[1], (code >> 2) & 3) - 5,
                dv = pick4(top[2], code >> 4) - 5;
      __syncwarp();
      w_off[lane] = dw * axy + du * apitch + dv;
      __syncwarp();
    }
    const bool full = t.out && conf_thr > 0.f && rp.conf[lane - 1] < conf_thr;
    const unsigned any_full = __ballot_sync(0xffffffffu, full);
    if (full) my_fallbacks += __popc(t.take);
    float2 in[3][(kRows + 2) / 2];
    rs_inputs(img, nx, ny, t, yc, scale, in);
    const float2 s2 = make_float2(scale, scale);
    const float *ab = atl + ((long long)(t.z - 1) * axy + (long long)(t.x0 - 1) * apitch + yc);
    const float *lb = lab + ((long long)t.z * axy + (long long)t.x0 * apitch + yc);
    float P[kRows], W[kRows];
#pragma unroll
    for (int r = 0; r < kRows; ++r) P[r] = W[r] = 0.f;
    if (!any_full) {
      constexpr int kept = LEVEL <= 2 ? 10 : LEVEL == 3 ? 20 : 32;
#pragma unroll kRsUnroll
      for (int c = 0; c < kept; ++c) {
        const int off = w_off[c];
        eval_offset4<false>(ab + off, lb + off, in, axy, apitch, t.take, s2, P, W);
      }
      my_evals += (unsigned long long)kept * __popc(t.owned);
    } else {
      unsigned long long rank[3];
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        rank[a] = 0x77777777777ULL;  // nibble j: rank of offset j - 5 on axis a, 7 = not kept
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          rank[a] &= ~(0xFULL << (4 * top[a][r]));
          rank[a] |= (unsigned long long)r << (4 * top[a][r]);
        }
      }
      // the NH^3 window: offset indices 5 - hw .. 5 + hw of each axis
      for (int jw = 5 - hw; jw <= 5 + hw; ++jw) {
        const int rw = (int)((rank[0] >> (4 * jw)) & 0xF);
        for (int ju = 5 - hw; ju <= 5 + hw; ++ju) {
          const int ru = rw + (int)((rank[1] >> (4 * ju)) & 0xF);
          for (int jv = 5 - hw; jv <= 5 + hw; ++jv) {
            const bool mine = full || (ru + (int)((rank[2] >> (4 * jv)) & 0xF) <= LEVEL);
            const int off = (jw - 5) * axy + (ju - 5) * apitch + (jv - 5);
            eval_offset4<true>(ab + off, lb + off, in, axy, apitch, mine ? t.take : 0u, s2, P, W);
          }
        }
      }
      const unsigned long long nw = 2 * hw + 1;
      my_evals += nw * nw * nw * __popc(t.owned);
    }
    rs_store(t, nx, ny, P, W, pacc, wacc);
  }
  if (my_fallbacks) atomicAdd(fallbacks, my_fallbacks);
  if (lane == 0 && my_evals) atomicAdd(evaluated, my_evals);
}

// ---- z-pair items: one warp = the same 4 x-rows in two consecutive z planes of one block

// One offset for the 8 rows of a z-pair item: rows r (plane z0) and 4 + r (plane z0 + 1). `a`
// points at the atlas voxel (z0 - 1 + dw, x0 - 1 + du, yc + dv), `l` at the label voxel (z0 + dw,
// x0 + du, yc + dv). The two planes' patches share their middle two atlas planes, so an offset
// loads 4 x 6 tap rows instead of 2 x 3 x 6; each row's arithmetic is eval_offset4's, in the same
// order, so a row's sums are the same bits either way.
template <bool MASKED>
__device__ __forceinline__ void eval_offset8(const float *__restrict__ a,
                                             const float *__restrict__ l,
                                             const float2 (&in)[4][(kRows + 2) / 2], int axy,
                                             int apitch, unsigned take, float2 s2,
                                             float (&P)[2 * kRows], float (&W)[2 * kRows]) {
  float Z[2][kRows + 2];
#pragma unroll
  for (int xp = 0; xp < (kRows + 2) / 2; ++xp) {
    const int ro = 2 * xp * apitch;
    float2 t[4];
#pragma unroll
    for (int dz = 0; dz < 4; ++dz) {
      const float2 av = make_float2(__ldg(a + (ro + dz * axy)), __ldg(a + (ro + apitch + dz * axy)));
      t[dz] = __ffma2_rn(av, s2, in[dz][xp]);
    }
#pragma unroll
    for (int pz = 0; pz < 2; ++pz) {
      float2 z = make_float2(0.f, 0.f);
#pragma unroll
      for (int dz = 0; dz < 3; ++dz) z = __ffma2_rn(t[pz + dz], t[pz + dz], z);
      Z[pz][2 * xp] = z.x;
      Z[pz][2 * xp + 1] = z.y;
    }
  }
#pragma unroll
  for (int pz = 0; pz < 2; ++pz)
#pragma unroll
    for (int r = 0; r < kRows; ++r) {
      const float x = Z[pz][r] + Z[pz][r + 1] + Z[pz][r + 2];
      const float e =
          __shfl_up_sync(0xffffffffu, x, 1) + x + __shfl_down_sync(0xffffffffu, x, 1);
      if (!MASKED || ((take >> (pz * kRows + r)) & 1u)) {
        const float w = rs_ex2(-e);
        P[pz * kRows + r] = fmaf(w, __ldg(l + (pz * axy + r * apitch)), P[pz * kRows + r]);
        W[pz * kRows + r] += w;
      }
    }
}

// Item `it` = ((z block * nbx + bx) * segs + seg) * 2 + pair of the interior grid: planes zq, zq + 1
// with zq = lo + 4 z block + 2 pair; a pair whose second plane lies past the interior is shifted
// back by one plane and owns only its second plane (needs 2 or more interior planes). Bits r and
// 4 + r of `owned` / `take` are row r of the first and the second plane.
__device__ __forceinline__ bool rs_place2(long long it, int nx, int ny, int nz, int lo, int segs,
                                          int nbx, int lane, RsItem &t, int &zq) {
  const long long r0 = it / 2;
  t.seg = (int)(r0 % segs);
  const long long r1 = r0 / segs;
  t.bx = (int)(r1 % nbx);
  zq = (int)(r1 / nbx) * kRows + 2 * (int)(it % 2) + lo;
  if (zq >= nz - lo) return false;
  t.z = min(zq, nz - lo - 2);
  t.xb = lo + t.bx * kRows;
  t.x0 = min(t.xb, nx - lo - kRows);
  t.y = lo + t.seg * kRowOut - 1 + lane;
  t.out = lane >= 1 && lane <= kRowOut && t.y < ny - lo;
  t.owned = 0;
#pragma unroll
  for (int r = 0; r < kRows; ++r)
    if (t.x0 + r >= t.xb) t.owned |= (t.z == zq ? 1u : 0u) << r | 1u << (kRows + r);
  t.take = t.out ? t.owned : 0u;
  return true;
}

// Input taps I(z0 + dz - 1, x0 - 1 + xr, yc) of a z-pair item (4 planes), negated and scaled.
__device__ __forceinline__ void rs_inputs2(const float *__restrict__ img, int nx, int ny,
                                           const RsItem &t, int yc, float scale,
                                           float2 (&in)[4][(kRows + 2) / 2]) {
  const long long nxy = (long long)nx * ny;
#pragma unroll
  for (int dz = 0; dz < 4; ++dz)
#pragma unroll
    for (int xp = 0; xp < (kRows + 2) / 2; ++xp) {
      const float *pi = img + (long long)(t.z + dz - 1) * nxy + (long long)(t.x0 - 1 + 2 * xp) * ny + yc;
      in[dz][xp] = make_float2(-__ldg(pi) * scale, -__ldg(pi + ny) * scale);
    }
}

__device__ __forceinline__ void rs_store2(const RsItem &t, int nx, int ny,
                                          const float (&P)[2 * kRows],
                                          const float (&W)[2 * kRows], float *__restrict__ pacc,
                                          float *__restrict__ wacc) {
  const long long nxy = (long long)nx * ny;
#pragma unroll
  for (int pz = 0; pz < 2; ++pz)
#pragma unroll
    for (int r = 0; r < kRows; ++r)
      if ((t.take >> (pz * kRows + r)) & 1u) {
        const long long v = (long long)(t.z + pz) * nxy + (long long)(t.x0 + r) * ny + t.y;
        pacc[v] += P[pz * kRows + r];
        wacc[v] += W[pz * kRows + r];
      }
}

// rescore4_body over z-pair items (2 or more interior planes): the same proposals, offsets,
// fallback rule and per-row arithmetic, 8 rows per warp.
template <int LEVEL>
__device__ __forceinline__ void rescore8_body(
    const RowProp *__restrict__ props, const float *__restrict__ img, const float *__restrict__ atl,
    const float *__restrict__ lab, int nx, int ny, int nz, int apitch, float scale, float conf_thr,
    float *__restrict__ pacc, float *__restrict__ wacc, unsigned long long *__restrict__ fallbacks,
    unsigned long long *__restrict__ evaluated, const unsigned char *__restrict__ tile_flag,
    const RescoreTiles ts, int hw) {
  __shared__ int s_off[kRescoreWarps][kRsTopK];
#ifdef PCT_RS_NX
  nx = PCT_RS_NX;
#endif
#ifdef PCT_RS_PITCH
  apitch = PCT_RS_PITCH;
#endif
#ifdef PCT_RS_HW
  hw = PCT_RS_HW;
#endif
  const int lane = threadIdx.x & 31;
  int *w_off = s_off[threadIdx.x >> 5];
  const int lo = hw + 1;
  const int ix = nx - 2 * lo, iz = nz - 2 * lo, iy = ny - 2 * lo;
  if (ix < kRows || iy <= 0 || iz < 2) return;
  const int segs = (iy + kRowOut - 1) / kRowOut;
  const int nbx = (ix + kRows - 1) / kRows;
  const long long items = (long long)((iz + kRows - 1) / kRows) * 2 * nbx * segs;
  const int axy = nx * apitch;
  unsigned long long my_fallbacks = 0, my_evals = 0;
  for (long long it = (long long)blockIdx.x * kRescoreWarps + (threadIdx.x >> 5); it < items;
       it += (long long)gridDim.x * kRescoreWarps) {
    RsItem t;
    int zq;
    if (!rs_place2(it, nx, ny, nz, lo, segs, nbx, lane, t, zq)) continue;
    // both planes lie in one tile of the plain kernel (tiles start at even planes from lo), or
    // only the second is owned
    if (tile_flag &&
        tile_flag[((zq - lo) / ts.zt * ts.tiles_x + (t.xb - lo) / ts.xc) * ts.tiles_y + t.seg])
      continue;
    const int yc = min(t.y, ny - lo);
    const RowProp &rp = props[((long long)((zq - lo) / kRows) * nbx + t.bx) * segs + t.seg];
    int top[3][4];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int r = 0; r < 4; ++r) top[a][r] = rp.top[a * 4 + r];
    {
      const int code = kRankTriples[lane];
      const int dw = pick4(top[0], code & 3) - 5, du = pick4(top[1], (code >> 2) & 3) - 5,
                dv = pick4(top[2], code >> 4) - 5;
      __syncwarp();
      w_off[lane] = dw * axy + du * apitch + dv;
      __syncwarp();
    }
    const bool full = t.out && conf_thr > 0.f && rp.conf[lane - 1] < conf_thr;
    const unsigned any_full = __ballot_sync(0xffffffffu, full);
    if (full) my_fallbacks += __popc(t.take);
    float2 in[4][(kRows + 2) / 2];
    rs_inputs2(img, nx, ny, t, yc, scale, in);
    const float2 s2 = make_float2(scale, scale);
    const float *ab = atl + ((long long)(t.z - 1) * axy + (long long)(t.x0 - 1) * apitch + yc);
    const float *lb = lab + ((long long)t.z * axy + (long long)t.x0 * apitch + yc);
    float P[2 * kRows], W[2 * kRows];
#pragma unroll
    for (int r = 0; r < 2 * kRows; ++r) P[r] = W[r] = 0.f;
    if (!any_full) {
      constexpr int kept = LEVEL <= 2 ? 10 : LEVEL == 3 ? 20 : 32;
#pragma unroll kRsUnroll8
      for (int c = 0; c < kept; ++c) {
        const int off = w_off[c];
        eval_offset8<false>(ab + off, lb + off, in, axy, apitch, t.take, s2, P, W);
      }
      my_evals += (unsigned long long)kept * __popc(t.owned);
    } else {
      unsigned long long rank[3];
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        rank[a] = 0x77777777777ULL;
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          rank[a] &= ~(0xFULL << (4 * top[a][r]));
          rank[a] |= (unsigned long long)r << (4 * top[a][r]);
        }
      }
      for (int jw = 5 - hw; jw <= 5 + hw; ++jw) {
        const int rw = (int)((rank[0] >> (4 * jw)) & 0xF);
        for (int ju = 5 - hw; ju <= 5 + hw; ++ju) {
          const int ru = rw + (int)((rank[1] >> (4 * ju)) & 0xF);
          for (int jv = 5 - hw; jv <= 5 + hw; ++jv) {
            const bool mine = full || (ru + (int)((rank[2] >> (4 * jv)) & 0xF) <= LEVEL);
            const int off = (jw - 5) * axy + (ju - 5) * apitch + (jv - 5);
            eval_offset8<true>(ab + off, lb + off, in, axy, apitch, mine ? t.take : 0u, s2, P, W);
          }
        }
      }
      const unsigned long long nw = 2 * hw + 1;
      my_evals += nw * nw * nw * __popc(t.owned);
    }
    rs_store2(t, nx, ny, P, W, pacc, wacc);
  }
  if (my_fallbacks) atomicAdd(fallbacks, my_fallbacks);
  if (lane == 0 && my_evals) atomicAdd(evaluated, my_evals);
}

// The proposal baseline without a network: every voxel rescores the same k offsets, the ones of
// the window nearest its centre. Same items, taps and arithmetic as the proposal rescoring.
__device__ __forceinline__ void rescore_prior_body(
    const PriorList &pl, const float *__restrict__ img, const float *__restrict__ atl,
    const float *__restrict__ lab, int nx, int ny, int nz, int apitch, float scale,
    float *__restrict__ pacc, float *__restrict__ wacc, unsigned long long *__restrict__ evaluated,
    int hw) {
#ifdef PCT_RS_NX
  nx = PCT_RS_NX;
#endif
#ifdef PCT_RS_PITCH
  apitch = PCT_RS_PITCH;
#endif
#ifdef PCT_RS_HW
  hw = PCT_RS_HW;
#endif
  const int lane = threadIdx.x & 31;
  const int lo = hw + 1;
  const int ix = nx - 2 * lo, iz = nz - 2 * lo, iy = ny - 2 * lo;
  if (ix < kRows || iy <= 0 || iz <= 0) return;
  const int segs = (iy + kRowOut - 1) / kRowOut;
  const int nbx = (ix + kRows - 1) / kRows;
  const long long items = (long long)((iz + kRows - 1) / kRows) * kRows * nbx * segs;
  const int axy = nx * apitch;
  unsigned long long my_evals = 0;
  for (long long it = (long long)blockIdx.x * kRescoreWarps + (threadIdx.x >> 5); it < items;
       it += (long long)gridDim.x * kRescoreWarps) {
    RsItem t;
    if (!rs_place(it, nx, ny, nz, lo, segs, nbx, lane, t)) continue;
    const int yc = min(t.y, ny - lo);
    float2 in[3][(kRows + 2) / 2];
    rs_inputs(img, nx, ny, t, yc, scale, in);
    const float2 s2 = make_float2(scale, scale);
    const float *ab = atl + ((long long)(t.z - 1) * axy + (long long)(t.x0 - 1) * apitch + yc);
    const float *lb = lab + ((long long)t.z * axy + (long long)t.x0 * apitch + yc);
    float P[kRows], W[kRows];
#pragma unroll
    for (int r = 0; r < kRows; ++r) P[r] = W[r] = 0.f;
#pragma unroll kRsUnroll
    for (int c = 0; c < pl.n; ++c) {
      const int off = pl.off[c];
      eval_offset4<false>(ab + off, lb + off, in, axy, apitch, t.take, s2, P, W);
    }
    my_evals += (unsigned long long)pl.n * __popc(t.owned);
    rs_store(t, nx, ny, P, W, pacc, wacc);
  }
  if (lane == 0 && my_evals) atomicAdd(evaluated, my_evals);
}

// rescore_prior_body over z-pair items (2 or more interior planes).
__device__ __forceinline__ void rescore_prior8_body(
    const PriorList &pl, const float *__restrict__ img, const float *__restrict__ atl,
    const float *__restrict__ lab, int nx, int ny, int nz, int apitch, float scale,
    float *__restrict__ pacc, float *__restrict__ wacc, unsigned long long *__restrict__ evaluated,
    int hw) {
#ifdef PCT_RS_NX
  nx = PCT_RS_NX;
#endif
#ifdef PCT_RS_PITCH
  apitch = PCT_RS_PITCH;
#endif
#ifdef PCT_RS_HW
  hw = PCT_RS_HW;
#endif
  const int lane = threadIdx.x & 31;
  const int lo = hw + 1;
  const int ix = nx - 2 * lo, iz = nz - 2 * lo, iy = ny - 2 * lo;
  if (ix < kRows || iy <= 0 || iz < 2) return;
  const int segs = (iy + kRowOut - 1) / kRowOut;
  const int nbx = (ix + kRows - 1) / kRows;
  const long long items = (long long)((iz + kRows - 1) / kRows) * 2 * nbx * segs;
  const int axy = nx * apitch;
  unsigned long long my_evals = 0;
  for (long long it = (long long)blockIdx.x * kRescoreWarps + (threadIdx.x >> 5); it < items;
       it += (long long)gridDim.x * kRescoreWarps) {
    RsItem t;
    int zq;
    if (!rs_place2(it, nx, ny, nz, lo, segs, nbx, lane, t, zq)) continue;
    const int yc = min(t.y, ny - lo);
    float2 in[4][(kRows + 2) / 2];
    rs_inputs2(img, nx, ny, t, yc, scale, in);
    const float2 s2 = make_float2(scale, scale);
    const float *ab = atl + ((long long)(t.z - 1) * axy + (long long)(t.x0 - 1) * apitch + yc);
    const float *lb = lab + ((long long)t.z * axy + (long long)t.x0 * apitch + yc);
    float P[2 * kRows], W[2 * kRows];
#pragma unroll
    for (int r = 0; r < 2 * kRows; ++r) P[r] = W[r] = 0.f;
#pragma unroll kRsUnroll8
    for (int c = 0; c < pl.n; ++c) {
      const int off = pl.off[c];
      eval_offset8<false>(ab + off, lb + off, in, axy, apitch, t.take, s2, P, W);
    }
    my_evals += (unsigned long long)pl.n * __popc(t.owned);
    rs_store2(t, nx, ny, P, W, pacc, wacc);
  }
  if (lane == 0 && my_evals) atomicAdd(evaluated, my_evals);
}

#ifdef PCT_RS_JIT
// Entry points of the run-time compiled module (same parameters as the library's kernels).
#define PCT_RS_ENTRY(NAME, LEVEL)                                                                 \
  extern "C" __global__ void __launch_bounds__(kRescoreWarps * 32, PCT_RS_MIN_CTAS) NAME(         \
      const RowProp *__restrict__ props, const float *__restrict__ img,                           \
      const float *__restrict__ atl, const float *__restrict__ lab, int nx, int ny, int nz,       \
      int apitch, float scale, float conf_thr, float *__restrict__ pacc,                          \
      float *__restrict__ wacc, unsigned long long *__restrict__ fallbacks,                       \
      unsigned long long *__restrict__ evaluated, const unsigned char *__restrict__ tile_flag,    \
      const RescoreTiles ts, int hw) {                                                            \
    rescore4_body<LEVEL>(props, img, atl, lab, nx, ny, nz, apitch, scale, conf_thr, pacc, wacc,   \
                         fallbacks, evaluated, tile_flag, ts, hw);                                \
  }
PCT_RS_ENTRY(pct_rescore4_l2, 2)
PCT_RS_ENTRY(pct_rescore4_l3, 3)
PCT_RS_ENTRY(pct_rescore4_l4, 4)
#undef PCT_RS_ENTRY
#define PCT_RS_ENTRY8(NAME, LEVEL)                                                                \
  extern "C" __global__ void __launch_bounds__(kRescoreWarps * 32, PCT_RS_MIN_CTAS8) NAME(        \
      const RowProp *__restrict__ props, const float *__restrict__ img,                           \
      const float *__restrict__ atl, const float *__restrict__ lab, int nx, int ny, int nz,       \
      int apitch, float scale, float conf_thr, float *__restrict__ pacc,                          \
      float *__restrict__ wacc, unsigned long long *__restrict__ fallbacks,                       \
      unsigned long long *__restrict__ evaluated, const unsigned char *__restrict__ tile_flag,    \
      const RescoreTiles ts, int hw) {                                                            \
    rescore8_body<LEVEL>(props, img, atl, lab, nx, ny, nz, apitch, scale, conf_thr, pacc, wacc,   \
                         fallbacks, evaluated, tile_flag, ts, hw);                                \
  }
PCT_RS_ENTRY8(pct_rescore8_l2, 2)
PCT_RS_ENTRY8(pct_rescore8_l3, 3)
PCT_RS_ENTRY8(pct_rescore8_l4, 4)
#undef PCT_RS_ENTRY8

extern "C" __global__ void __launch_bounds__(kRescoreWarps * 32, PCT_RS_MIN_CTAS)
    pct_rescore_prior(const __grid_constant__ PriorList pl, const float *__restrict__ img,
                      const float *__restrict__ atl, const float *__restrict__ lab, int nx, int ny,
                      int nz, int apitch, float scale, float *__restrict__ pacc,
                      float *__restrict__ wacc, unsigned long long *__restrict__ evaluated, int hw) {
  rescore_prior_body(pl, img, atl, lab, nx, ny, nz, apitch, scale, pacc, wacc, evaluated, hw);
}

extern "C" __global__ void __launch_bounds__(kRescoreWarps * 32, PCT_RS_MIN_CTAS8)
    pct_rescore_prior8(const __grid_constant__ PriorList pl, const float *__restrict__ img,
                       const float *__restrict__ atl, const float *__restrict__ lab, int nx, int ny,
                       int nz, int apitch, float scale, float *__restrict__ pacc,
                       float *__restrict__ wacc, unsigned long long *__restrict__ evaluated,
                       int hw) {
  rescore_prior8_body(pl, img, atl, lab, nx, ny, nz, apitch, scale, pacc, wacc, evaluated, hw);
}
#endif
