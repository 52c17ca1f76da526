// Plain FP32 patch-based multi-atlas fusion for sm_100a, atlas slabs staged by TMA.
//
// Same arithmetic contract as the reference (MultiAtlasPatchBasedSegmentationOpenMP +
// PatchSimilarity, NewPatchedBrainPureC.cpp:1184-1212,1350-1449), in FP32:
//     SSD(x,d) = sum_{p in 3x3x3} (I(x+p) - A_a(x+d+p))^2,   w = exp(-SSD/div)
//     out(x)   = sum_{a,d} w*L_a(x+d) / sum_{a,d} w            (NaN rule of :1325-1331)
//
// Work decomposition
//  * A warp owns 30 (y) x RX (x) x 2*TZ (z) output voxels. Lanes run along the contiguous y
//    axis (lanes 1..30 own outputs, lanes 0/31 carry the y-halo). For one offset d the SSD of
//    all voxels is a 3x3x3 box sum of D_d = (I - A_d)^2: each lane box-sums its RX+2 rows x
//    TZ+2 planes in registers along x and z, and the y-box is two warp shuffles.
//  * The thread's two z-halves are packed into float2 and run on the paired FP32 instructions
//    (add/mul/fma .f32x2): same lane throughput as scalar FP32, half the issue slots.
//  * dw is the innermost offset loop: stepping dw shifts the atlas planes by one, so the atlas
//    window (TZ+2 planes x RX+2 rows per half) lives in registers as a ring and each step reads
//    one new plane. The step loop is unrolled one ring period at a time (not the whole window)
//    to keep the kernel inside the instruction cache.
//  * A CTA is 4 warps stacked along x. Its atlas MRI and atlas CT rows (one x-row = a z x y
//    slab) sit in two shared-memory rings indexed by x. Each du step needs one new row of each;
//    one thread issues it with cp.async.bulk.tensor (TMA, no multicast) one step ahead, and the
//    step's readers wait on an mbarrier (transaction-count completion, ping-pong pair). Every
//    per-thread shared-memory read is one LDS with an immediate offset.
//  * TMA zero-fills coordinates outside the volume, so tiles need no clamping: out-of-volume
//    rows/planes/lanes only ever feed voxels outside the interior, which are never stored.
//  * CTAs are persistent over the tile list.
//  * Every mbarrier wait is bounded (globaltimer); on timeout the CTA records an error code,
//    stops at the next CTA barrier, drains its own in-flight copies (bounded) and returns.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "pct_internal.h"
#include "pct_ptx.cuh"

namespace pct {
namespace {

using namespace ptx;

constexpr int kOutY = 30;
constexpr int kWarps = 4;
constexpr int kThreads = kWarps * 32;
constexpr float kDblEpsilonF = 2.220446049250313080847e-16f;

__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

__device__ __forceinline__ float fuse_result(float product, float sum_weight) {
  return (fabsf(product) > kDblEpsilonF && fabsf(sum_weight) > kDblEpsilonF)
             ? __fdiv_rn(product, sum_weight)
             : __int_as_float(0x7fc00000);
}

// ---------------------------------------------------------------- geometry of one variant

template <int HW, int RX, int TZ>
struct Cfg {
  static constexpr int NQ = TZ + 2;          // D planes per half
  static constexpr int NR = RX + 2;          // D rows per warp
  static constexpr int NS = 2 * HW + 1;      // offsets per axis
  static constexpr int XC = kWarps * RX;     // output rows per CTA
  // y extent of a slab row: lanes span 32 positions, +-HW for dv, +2 for the 16-byte
  // alignment of the TMA start coordinate (tile starts are 30*ty, i.e. 0 or 2 mod 4).
  static constexpr int YB = (34 + 2 * HW + 3) / 4 * 4;
  static constexpr int ZA = 2 * TZ + 2 + 2 * HW;  // atlas MRI planes per slab row
  static constexpr int ZL = 2 * TZ + 2 * HW;      // atlas CT planes per slab row
  static constexpr int RA = XC + 3;               // MRI ring: XC+2 rows in use + 1 prefetch
  static constexpr int RL = XC + 1;               // CT ring: XC rows in use + 1 prefetch
  static constexpr uint32_t ROW_A = ZA * YB * 4;  // TMA transaction bytes per row
  static constexpr uint32_t ROW_L = ZL * YB * 4;
  static constexpr uint32_t SLOT_A = (ROW_A + 127) / 128 * 128;
  static constexpr uint32_t SLOT_L = (ROW_L + 127) / 128 * 128;
  static constexpr uint32_t PLANE = YB * 4;       // bytes between planes of a slab row
  static constexpr int SMEM = 128 + 128 + RA * SLOT_A + RL * SLOT_L;  // + alignment slack
  static constexpr int NCH = (NS + NQ - 1) / NQ;  // ring periods per dw sweep
  static constexpr int OFF = NCH * NQ - NS;       // virtual steps skipped in the first period
};

// One subject as the kernels see it.
struct SubjectView {
  const float *img;   // input MRI, reference layout
  float *out;         // fused output, reference layout (interior written)
  float *partial;     // groups > 1: [groups][2][nvox] partial (product, sum_weight) sums
  const CUtensorMap *tmA, *tmL;  // atlas MRI / CT slab maps (param or global space)
  int nx, ny, nz, nxy;
  long long nvox;
  float scale;        // sqrt(log2(e)/div): taps are scaled so that the box sum is SSD*log2(e)/div
  int tiles_y, tiles_x, ntiles;
  int groups, atlases_per_group;  // items = groups * ntiles (group-major)
  int hw;             // half window of this subject (batched kernel dispatch)
  int item_begin;     // first global item of this subject (batched kernel)
  int atlas_base;     // first atlas of group 0 (a single-atlas launch over a tile list)
  float *acc_p, *acc_w;  // non-null: add each voxel's (product, sum_weight) into these instead
  // non-null (masked items): item = pair << 24 | tile, over the atlases atlas_base + i for the
  // set bits i of atlas_mask[tile], two per pair in bit order; pair k's sums go to partial slot k
  const uint32_t *atlas_mask;
};

struct TmaParams {
  SubjectView sv;
  int item_begin, item_end;  // the work items this launch covers (group-major numbering)
  int *err;           // device status word (0 = ok)
  unsigned long long timeout_ns;
  int withhold_cta;   // testing hook: this CTA withholds its first copies (-1 = none)
};

// One dw sweep (all dw for fixed atlas, du, dv) of the thread's voxels.
template <int HW, int RX, int TZ>
__device__ __forceinline__ void sweep_dw(const float2 (&In)[TZ + 2][RX + 2], float2 (&P)[TZ][RX],
                                         float2 (&W)[TZ][RX], const uint32_t (&rowA)[RX + 2],
                                         const uint32_t (&rowL)[RX], const float2 scale2) {
  using C = Cfg<HW, RX, TZ>;
  constexpr int NQ = C::NQ, NR = C::NR;
  float2 Aw[NQ][NR];  // logical plane q at virtual step v lives in slot (q + v) % NQ
#pragma unroll
  for (int q = 0; q < NQ - 1; ++q)
#pragma unroll
    for (int r = 0; r < NR; ++r)
      Aw[(q + C::OFF) % NQ][r] = make_float2(lds_f32(rowA[r] + q * C::PLANE),
                                             lds_f32(rowA[r] + (TZ + q) * C::PLANE));
#pragma unroll 1
  for (int c = 0; c < C::NCH; ++c) {
#pragma unroll
    for (int jj = 0; jj < NQ; ++jj) {
      if (jj < C::OFF && c == 0) continue;
      const uint32_t so = (uint32_t)(c * NQ + jj - C::OFF) * C::PLANE;  // real step s = dw + HW
      {
        constexpr int qn = NQ - 1;
        const int sn = (qn + jj) % NQ;
#pragma unroll
        for (int r = 0; r < NR; ++r)
          Aw[sn][r] = make_float2(lds_f32(rowA[r] + so + qn * C::PLANE),
                                  lds_f32(rowA[r] + so + (TZ + qn) * C::PLANE));
      }
      // x-box of D = s^2 (A - I)^2 per plane
      float2 g[NQ][RX];
#pragma unroll
      for (int q = 0; q < NQ; ++q) {
        const int sq = (q + jj) % NQ;
        float2 D[NR];
#pragma unroll
        for (int r = 0; r < NR; ++r) {
          const float2 d = fma2(Aw[sq][r], scale2, In[q][r]);  // s * (A - I)
          D[r] = mul2(d, d);
        }
#pragma unroll
        for (int x = 0; x < RX; x += 2) {
          if (x + 1 < RX) {
            const float2 mid = add2(D[x + 1], D[x + 2]);
            g[q][x] = add2(D[x], mid);
            g[q][x + 1] = add2(mid, D[x + 3]);
          } else {
            g[q][x] = add2(add2(D[x], D[x + 1]), D[x + 2]);
          }
        }
      }
      // z-box, y-box (warp shuffles), weight, accumulate
#pragma unroll
      for (int x = 0; x < RX; ++x) {
#pragma unroll
        for (int q = 0; q < TZ; q += 2) {
          float2 S[2];
          if (q + 1 < TZ) {
            const float2 mid = add2(g[q + 1][x], g[q + 2][x]);
            S[0] = add2(g[q][x], mid);
            S[1] = add2(mid, g[q + 3][x]);
          } else {
            S[0] = add2(add2(g[q][x], g[q + 1][x]), g[q + 2][x]);
          }
#pragma unroll
          for (int k = 0; k < 2; ++k) {
            if (q + k >= TZ) break;
            const float2 cc = S[k];
            const float2 lft = make_float2(__shfl_up_sync(0xffffffffu, cc.x, 1),
                                           __shfl_up_sync(0xffffffffu, cc.y, 1));
            const float2 rgt = make_float2(__shfl_down_sync(0xffffffffu, cc.x, 1),
                                           __shfl_down_sync(0xffffffffu, cc.y, 1));
            const float2 e = add2(add2(cc, lft), rgt);  // SSD * log2(e) / div
            const float2 w = make_float2(ex2_approx(-e.x), ex2_approx(-e.y));
            const float2 lab = make_float2(lds_f32(rowL[x] + so + (q + k) * C::PLANE),
                                           lds_f32(rowL[x] + so + (TZ + q + k) * C::PLANE));
            P[q + k][x] = fma2(w, lab, P[q + k][x]);
            W[q + k][x] = add2(W[q + k][x], w);
          }
        }
      }
    }
  }
}

// ------------------------------------------------------------- y-pair layout (LY = 1)
//
// Same warp tile (30 y x RX x x 2*TZ z) and the same shared-memory slabs as above, mapped
// differently: half-warp h = lane / 16 owns the z planes [z0 + h*TZ, z0 + h*TZ + TZ), and lane
// j = lane % 16 owns the two adjacent y positions (y0 - 1 + 2j, y0 + 2j), packed in a float2.
//  * y-box: each output needs one neighbour value from each side (the left lane's .y, the right
//    lane's .x): 2 shuffles per voxel pair instead of 4.
//  * x-box: the squares are folded into the first additions as FMAs
//    (g = d0*d0 + (d1*d1 + d2*d2) with the inner pair shared by two outputs), 6 instructions per
//    plane of 3 outputs instead of 5 multiplies + 5 adds.
//  * labels ride a register ring like the atlas planes: one new plane per dw step.
//  * a pair's shared-memory address is 8-byte aligned for every other dv (the parity of
//    dv + HW): those sweeps load pairs with one 64-bit LDS, the others with two 32-bit LDS.

template <bool AL>
__device__ __forceinline__ float2 lds_pair(uint32_t addr) {
  if constexpr (AL) {
    return lds_f32x2(addr);
  } else {
    return make_float2(lds_f32(addr), lds_f32(addr + 4));
  }
}

// g[x] = d[x]^2 + d[x+1]^2 + d[x+2]^2 for x < RX, two outputs at a time sharing d[x+1]^2 + d[x+2]^2.
template <int RX>
__device__ __forceinline__ void xbox_squares(const float2 (&d)[RX + 2], float2 (&g)[RX]) {
  float2 u = make_float2(0.f, 0.f);
#pragma unroll
  for (int x = 0; x < RX; x += 2) {
    if (x + 1 < RX) {
      u = mul2(d[x + 2], d[x + 2]);
      const float2 m = fma2(d[x + 1], d[x + 1], u);
      g[x] = fma2(d[x], d[x], m);
      g[x + 1] = fma2(d[x + 3], d[x + 3], m);
    } else if (x >= 2) {  // odd RX: u holds d[x]^2 from the previous pair
      g[x] = fma2(d[x + 2], d[x + 2], fma2(d[x + 1], d[x + 1], u));
    } else {
      g[x] = fma2(d[x], d[x], fma2(d[x + 1], d[x + 1], mul2(d[x + 2], d[x + 2])));
    }
  }
}

// One dw sweep (all dw for fixed atlas, du, dv) of the lane's voxels, y-pair layout.
// rowA[r] / rowL[r]: the lane's pair in plane 0 of its half's slab rows, at this dv.
template <int HW, int RX, int TZ, bool AL, bool LR>
__device__ __forceinline__ void sweep_dw_yp(const float2 (&In)[TZ + 2][RX + 2],
                                            float2 (&P)[TZ][RX], float2 (&W)[TZ][RX],
                                            const uint32_t (&rowA)[RX + 2],
                                            const uint32_t (&rowL)[RX], const float2 scale2) {
  using C = Cfg<HW, RX, TZ>;
  constexpr int NQ = C::NQ, NR = C::NR;
  // Atlas plane t (= step + D plane) and label plane t (= step + output plane) live in slot
  // (t + OFF) % NQ; at virtual step v = c*NQ + jj that is slot (jj + plane) % NQ.
  float2 Aw[NQ][NR];
  float2 Lw[NQ][RX];
#pragma unroll
  for (int t = 0; t < NQ - 1; ++t)
#pragma unroll
    for (int r = 0; r < NR; ++r) Aw[(t + C::OFF) % NQ][r] = lds_pair<AL>(rowA[r] + t * C::PLANE);
  if constexpr (LR) {
#pragma unroll
    for (int t = 0; t < TZ - 1; ++t)
#pragma unroll
      for (int r = 0; r < RX; ++r)
        Lw[(t + C::OFF) % NQ][r] = lds_pair<AL>(rowL[r] + t * C::PLANE);
  }
#pragma unroll 1
  for (int c = 0; c < C::NCH; ++c) {
#pragma unroll
    for (int jj = 0; jj < NQ; ++jj) {
      if (jj < C::OFF && c == 0) continue;
      const uint32_t so = (uint32_t)(c * NQ + jj - C::OFF) * C::PLANE;  // real step s = dw + HW
      {
        const int sa = (jj + NQ - 1) % NQ;
#pragma unroll
        for (int r = 0; r < NR; ++r)
          Aw[sa][r] = lds_pair<AL>(rowA[r] + so + (NQ - 1) * C::PLANE);
        if constexpr (LR) {
          const int sl = (jj + TZ - 1) % NQ;
#pragma unroll
          for (int r = 0; r < RX; ++r)
            Lw[sl][r] = lds_pair<AL>(rowL[r] + so + (TZ - 1) * C::PLANE);
        }
      }
      // Output planes two at a time: the x-box of D = (s A - s I)^2 for the planes they need
      // (computed once, as late as possible, to keep few x-box sums live), then the z-box, the
      // y-box (half-warp shuffles), the weight and the accumulators.
      float2 g[NQ][RX];
#pragma unroll
      for (int q = 0; q < TZ; q += 2) {
#pragma unroll
        for (int pq = (q == 0 ? 0 : q + 2); pq < (q + 4 < NQ ? q + 4 : NQ); ++pq) {
          const int sq = (pq + jj) % NQ;
          float2 d[NR];
#pragma unroll
          for (int r = 0; r < NR; ++r) d[r] = fma2(Aw[sq][r], scale2, In[pq][r]);  // s * (A - I)
          xbox_squares<RX>(d, g[pq]);
        }
#pragma unroll
        for (int x = 0; x < RX; ++x) {
          float2 S[2];
          if (q + 1 < TZ) {
            const float2 mid = add2(g[q + 1][x], g[q + 2][x]);
            S[0] = add2(g[q][x], mid);
            S[1] = add2(mid, g[q + 3][x]);
          } else {
            S[0] = add2(add2(g[q][x], g[q + 1][x]), g[q + 2][x]);
          }
#pragma unroll
          for (int k = 0; k < 2; ++k) {
            if (q + k >= TZ) break;
            const float2 cc = S[k];
            const float lft = __shfl_up_sync(0xffffffffu, cc.y, 1, 16);
            const float rgt = __shfl_down_sync(0xffffffffu, cc.x, 1, 16);
            const float m = cc.x + cc.y;
            const float2 w = make_float2(ex2_approx(-(m + lft)), ex2_approx(-(m + rgt)));
            const float2 lab = LR ? Lw[(q + k + jj) % NQ][x]
                                  : lds_pair<AL>(rowL[x] + so + (q + k) * C::PLANE);
            P[q + k][x] = fma2(w, lab, P[q + k][x]);
            W[q + k][x] = add2(W[q + k][x], w);
          }
        }
      }
    }
  }
}

// Pipeline state of one CTA, carried across its work items.
struct Pipe {
  uint32_t base;              // 128-byte aligned start of the dynamic shared memory
  uint32_t gstep;             // steps taken: barrier gstep&1, phase (gstep>>1)&1
  bool armed_next;            // thread 0: a prefetch is in flight on barrier (gstep+1)&1
  volatile int *abort_flag;
};

// Processes work item `item` (tile x atlas group) of subject `sv` with register tile (RX, TZ) in
// layout LY (0: z-halves packed; 1: y-pairs, labels read per use; 2: y-pairs, labels in a
// register ring). Returns false when a bounded wait gave up (the CTA must stop).
template <int HW, int RX, int TZ, int LY, bool MASKED = false>
__device__ __forceinline__ bool run_item(const SubjectView &sv, int item, Pipe &pp, int *err,
                                         unsigned long long timeout_ns, int withhold_cta) {
  using C = Cfg<HW, RX, TZ>;
  constexpr int NQ = C::NQ, NR = C::NR, NS = C::NS;
  const uint32_t bar0 = pp.base, bar1 = pp.base + 8;
  const uint32_t ringA = pp.base + 128;
  const uint32_t ringL = ringA + C::RA * C::SLOT_A;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int lo = HW + 1;
  const float2 scale2 = make_float2(sv.scale, sv.scale);
  int grp, t, a_first, natl;
  uint32_t later = 0;  // masked items: the pair's atlases after the current one (bits)
  if constexpr (MASKED) {
    grp = (int)((uint32_t)item >> 24);
    t = item & 0xffffff;
    uint32_t m = sv.atlas_mask[t];
    for (int k = 0; k < 2 * grp; ++k) m &= m - 1;  // drop the earlier pairs' atlases
    natl = min(2, __popc(m));
    a_first = sv.atlas_base + __ffs(m) - 1;
    later = m & (m - 1);
  } else {
    grp = item / sv.ntiles;
    t = item - grp * sv.ntiles;
    a_first = sv.atlas_base + grp * sv.atlases_per_group;
    natl = sv.atlases_per_group;
  }
  const int T = natl * NS;  // du steps per item (atlas-major)
  const int ty = t % sv.tiles_y;
  t /= sv.tiles_y;
  const int txc = t % sv.tiles_x;
  const int tz = t / sv.tiles_x;
  const int y0 = lo + ty * kOutY, X0 = lo + txc * C::XC, z0 = lo + tz * (2 * TZ);
  const int y = y0 - 1 + lane;
  const int yb = y0 - 1 - HW;      // first y of the slab (>= 0)
  const int e = yb & 3;
  const int ybox = yb - e;         // TMA start, 16-byte aligned
  const int xw = X0 + warp * RX;   // this warp's first output row
  const int xA = X0 - 1 - HW, zA = z0 - 1 - HW;  // MRI slab origin (row k=0)
  const int xL = X0 - HW, zL = z0 - HW;          // CT slab origin
  // y-pair layout: half-warp hh stacks in z, lane jj owns y positions yp, yp + 1.
  const int hh = lane >> 4, jj = lane & 15;
  const int yp = y0 - 1 + 2 * jj;
  const uint32_t lane_off = LY == 0 ? (uint32_t)(lane + HW + e) * 4u
                                    : (uint32_t)(2 * jj + HW + e) * 4u + hh * TZ * C::PLANE;

  // Input patch values, negated and scaled (D = (s A + In)^2 = s^2 (A - I)^2), zero outside.
  float2 In[NQ][NR];
#pragma unroll
  for (int q = 0; q < NQ; ++q)
#pragma unroll
    for (int r = 0; r < NR; ++r) {
      float v[2];
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        const int zz = (LY == 0 ? z0 + k * TZ : z0 + hh * TZ) - 1 + q, xx = xw - 1 + r;
        const int yy = LY == 0 ? y : yp + k;
        v[k] = (zz < sv.nz && xx < sv.nx && yy < sv.ny)
                   ? -__ldg(sv.img + (long long)zz * sv.nxy + (long long)xx * sv.ny + yy) * sv.scale
                   : 0.f;
      }
      In[q][r] = make_float2(v[0], v[1]);
    }
  float2 P[TZ][RX], W[TZ][RX];
#pragma unroll
  for (int q = 0; q < TZ; ++q)
#pragma unroll
    for (int r = 0; r < RX; ++r) {
      P[q][r] = make_float2(0.f, 0.f);
      W[q][r] = make_float2(0.f, 0.f);
    }

  int a = a_first;
  for (int i = 0; i < T; ++i, ++pp.gstep) {
    const int ai = i / NS, j = i - ai * NS;
    if constexpr (MASKED) {
      if (j == 0 && i > 0) {  // the pair's second atlas
        a = sv.atlas_base + __ffs(later) - 1;
        later &= later - 1;
      }
    } else {
      a = a_first + ai;
    }
    __syncthreads();  // every warp is done with step i-1: its ring rows may be refilled
    if (*pp.abort_flag) return false;
    const uint32_t gstep = pp.gstep;
    if (tid == 0) {
      fence_proxy_async_smem();
      // Testing hook: withhold the first window of this CTA so that the wait below runs out.
      const bool withhold = (int)blockIdx.x == withhold_cta && gstep == 0;
      if (j == 0 && !withhold) {  // atlas start: the whole window for this step
        const uint32_t b = (gstep & 1) ? bar1 : bar0;
        mbar_arrive_expect_tx(b, (C::XC + 2) * C::ROW_A + C::XC * C::ROW_L);
        for (int k = 0; k < C::XC + 2; ++k)
          tma_load_4d(ringA + (k % C::RA) * C::SLOT_A, sv.tmA, b, ybox, xA + k, zA, a);
        for (int k = 0; k < C::XC; ++k)
          tma_load_4d(ringL + (k % C::RL) * C::SLOT_L, sv.tmL, b, ybox, xL + k, zL, a);
      }
      pp.armed_next = false;
      if (j + 1 < NS) {  // prefetch the one new row of each ring for step i+1
        const uint32_t b = ((gstep + 1) & 1) ? bar1 : bar0;
        mbar_arrive_expect_tx(b, C::ROW_A + C::ROW_L);
        const int ka = j + C::XC + 2, kl = j + C::XC;
        tma_load_4d(ringA + (ka % C::RA) * C::SLOT_A, sv.tmA, b, ybox, xA + ka, zA, a);
        tma_load_4d(ringL + (kl % C::RL) * C::SLOT_L, sv.tmL, b, ybox, xL + kl, zL, a);
        pp.armed_next = true;
      }
    }
    const bool ok = mbar_wait_bounded((gstep & 1) ? bar1 : bar0, (gstep >> 1) & 1, timeout_ns);
    if (!__all_sync(0xffffffffu, ok)) {
      if (lane == 0) {
        atomicExch(err, 1);
        *pp.abort_flag = 1;
      }
      continue;  // the next CTA barrier sees the flag
    }
    // Ring rows of this thread for step (a, du = j - HW).
    uint32_t rowA[NR], rowL[RX];
#pragma unroll
    for (int r = 0; r < NR; ++r)
      rowA[r] = ringA + (uint32_t)((warp * RX + r + j) % C::RA) * C::SLOT_A + lane_off;
#pragma unroll
    for (int r = 0; r < RX; ++r)
      rowL[r] = ringL + (uint32_t)((warp * RX + r + j) % C::RL) * C::SLOT_L + lane_off;
    if constexpr (LY == 0) {
#pragma unroll 1
      for (int dv = -HW; dv <= HW; ++dv) {
        uint32_t ra[NR], rl[RX];
#pragma unroll
        for (int r = 0; r < NR; ++r) ra[r] = rowA[r] + (uint32_t)(dv * 4);
#pragma unroll
        for (int r = 0; r < RX; ++r) rl[r] = rowL[r] + (uint32_t)(dv * 4);
        sweep_dw<HW, RX, TZ>(In, P, W, ra, rl, scale2);
      }
    } else {
      // Pairs are 8-byte aligned when dv + HW is even: those sweeps first, then the others (the
      // order of the offsets only changes the FP32 summation order).
#pragma unroll 1
      for (int sv2 = 0; sv2 < NS; sv2 += 2) {
        uint32_t ra[NR], rl[RX];
#pragma unroll
        for (int r = 0; r < NR; ++r) ra[r] = rowA[r] + (uint32_t)((sv2 - HW) * 4);
#pragma unroll
        for (int r = 0; r < RX; ++r) rl[r] = rowL[r] + (uint32_t)((sv2 - HW) * 4);
        sweep_dw_yp<HW, RX, TZ, true, LY == 2>(In, P, W, ra, rl, scale2);
      }
#pragma unroll 1
      for (int sv2 = 1; sv2 < NS; sv2 += 2) {
        uint32_t ra[NR], rl[RX];
#pragma unroll
        for (int r = 0; r < NR; ++r) ra[r] = rowA[r] + (uint32_t)((sv2 - HW) * 4);
#pragma unroll
        for (int r = 0; r < RX; ++r) rl[r] = rowL[r] + (uint32_t)((sv2 - HW) * 4);
        sweep_dw_yp<HW, RX, TZ, false, LY == 2>(In, P, W, ra, rl, scale2);
      }
    }
  }
  __syncthreads();  // a timeout in the item's last step is seen here
  if (*pp.abort_flag) return false;

#pragma unroll
  for (int k = 0; k < 2; ++k) {
    // LY 0: k is the z half, the lane's y is y; LY 1: k is the y of the pair, the half is hh.
    const int yy = LY == 0 ? y : yp + k;
    if (yy < y0 || yy >= y0 + kOutY || yy >= sv.ny - lo) continue;
#pragma unroll
    for (int q = 0; q < TZ; ++q) {
      const int z = (LY == 0 ? z0 + k * TZ : z0 + hh * TZ) + q;
      if (z >= sv.nz - lo) continue;
#pragma unroll
      for (int r = 0; r < RX; ++r) {
        const int x = xw + r;
        if (x >= sv.nx - lo) continue;
        const float pr = k ? P[q][r].y : P[q][r].x;
        const float sw = k ? W[q][r].y : W[q][r].x;
        const long long v = (long long)z * sv.nxy + (long long)x * sv.ny + yy;
        if (sv.acc_p) {
          sv.acc_p[v] += pr;
          sv.acc_w[v] += sw;
        } else if (sv.groups == 1) {
          sv.out[v] = fuse_result(pr, sw);
        } else {
          sv.partial[(2LL * grp) * sv.nvox + v] = pr;
          sv.partial[(2LL * grp + 1) * sv.nvox + v] = sw;
        }
      }
    }
  }
  return true;
}

__device__ __forceinline__ Pipe pipe_init(unsigned char *smem_raw) {
  Pipe pp;
  pp.base = (smem_u32(smem_raw) + 127u) & ~127u;
  pp.gstep = 0;
  pp.armed_next = false;
  pp.abort_flag =
      reinterpret_cast<volatile int *>(smem_raw + (pp.base + 16 - smem_u32(smem_raw)));
  if (threadIdx.x == 0) {
    mbar_init(pp.base, 1);
    mbar_init(pp.base + 8, 1);
    *pp.abort_flag = 0;
    fence_mbarrier_init();
  }
  __syncthreads();
  return pp;
}

// After an abort, let this CTA's own outstanding copies land (bounded) before exiting: those of
// the step whose wait timed out (gstep-1) and the prefetch armed during it, if any.
__device__ __forceinline__ void pipe_drain(const Pipe &pp, unsigned long long timeout_ns) {
  if (threadIdx.x != 0) return;
  const uint32_t bar0 = pp.base, bar1 = pp.base + 8;
  const uint32_t s = pp.gstep - 1;
  mbar_wait_bounded((s & 1) ? bar1 : bar0, (s >> 1) & 1, timeout_ns);
  if (pp.armed_next)
    mbar_wait_bounded((pp.gstep & 1) ? bar1 : bar0, (pp.gstep >> 1) & 1, timeout_ns);
}

// One subject, persistent over its work items. MB = CTAs per SM the register budget is sized for.
template <int HW, int RX, int TZ, int LY, int MB>
__global__ void __launch_bounds__(kThreads, MB)
    fuse_tma_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmL,
                    TmaParams p) {
  extern __shared__ unsigned char smem_raw[];
  Pipe pp = pipe_init(smem_raw);
  p.sv.tmA = &tmA;
  p.sv.tmL = &tmL;
  for (int item = p.item_begin + blockIdx.x; item < p.item_end; item += gridDim.x) {
    if (!run_item<HW, RX, TZ, LY>(p.sv, item, pp, p.err, p.timeout_ns, p.withhold_cta)) {
      pipe_drain(pp, p.timeout_ns);
      return;
    }
  }
}

// The full search over a device-side list of masked items (count on the device, so the launch
// needs no host round trip): each item is up to two flagged atlases of one tile, its sums written
// to the partial slot of its pair.
template <int HW, int RX, int TZ, int LY, int MB>
__global__ void __launch_bounds__(kThreads, MB)
    fuse_list_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmL,
                     TmaParams p, const int *__restrict__ items, const int *__restrict__ count) {
  extern __shared__ unsigned char smem_raw[];
  Pipe pp = pipe_init(smem_raw);
  p.sv.tmA = &tmA;
  p.sv.tmL = &tmL;
  const int n = *count;
  for (int i = blockIdx.x; i < n; i += gridDim.x) {
    if (!run_item<HW, RX, TZ, LY, true>(p.sv, items[i], pp, p.err, p.timeout_ns, -1)) {
      pipe_drain(pp, p.timeout_ns);
      return;
    }
  }
}

// Register tiles (x rows RX, z planes per half TZ, layout LY, CTAs per SM MB) by half window, in
// sets the autotuner chooses between. Set 0 is the fastest measured shape per window on one B200
// (222x222x112, 10 atlases): y-pairs (3,4) for NH 7 and 11, y-pairs with the label ring (3,3)
// for NH 9. Set 1 is the z-pair layout (3,4), set 2 the z-pair (3,3)/(4,2) tiles, set 3 y-pairs
// with the label ring (3,4), set 4 y-pairs (2,3) at three CTAs per SM (168 registers).
template <int SET, int HW> struct TileOf { static constexpr int RX = 3, TZ = 4, LY = 1, MB = 1; };
template <> struct TileOf<0, 4> { static constexpr int RX = 3, TZ = 3, LY = 2, MB = 1; };
template <> struct TileOf<0, 2> { static constexpr int RX = 3, TZ = 3, LY = 1, MB = 1; };
template <> struct TileOf<0, 1> { static constexpr int RX = 4, TZ = 2, LY = 1, MB = 1; };
template <int HW> struct TileOf<1, HW> { static constexpr int RX = 3, TZ = 4, LY = 0, MB = 1; };
template <> struct TileOf<1, 2> { static constexpr int RX = 3, TZ = 3, LY = 0, MB = 1; };
template <> struct TileOf<1, 1> { static constexpr int RX = 4, TZ = 2, LY = 0, MB = 1; };
template <int HW> struct TileOf<2, HW> { static constexpr int RX = 4, TZ = 2, LY = 0, MB = 1; };
template <> struct TileOf<2, 5> { static constexpr int RX = 3, TZ = 3, LY = 0, MB = 1; };
template <> struct TileOf<2, 2> { static constexpr int RX = 3, TZ = 3, LY = 0, MB = 1; };
template <int HW> struct TileOf<3, HW> { static constexpr int RX = 3, TZ = 4, LY = 2, MB = 1; };
template <> struct TileOf<3, 1> { static constexpr int RX = 4, TZ = 2, LY = 2, MB = 1; };
template <int HW> struct TileOf<4, HW> { static constexpr int RX = 2, TZ = 3, LY = 1, MB = 3; };
template <int SET, int HW>
constexpr int smem_of() {
  return Cfg<HW, TileOf<SET, HW>::RX, TileOf<SET, HW>::TZ>::SMEM;
}
template <int SET>
constexpr int batch_smem() {
  return smem_of<SET, 5>() > smem_of<SET, 4>()
             ? (smem_of<SET, 5>() > smem_of<SET, 3>() ? smem_of<SET, 5>() : smem_of<SET, 3>())
             : (smem_of<SET, 4>() > smem_of<SET, 3>() ? smem_of<SET, 4>() : smem_of<SET, 3>());
}

struct BatchParams {
  const SubjectView *subjects;  // device array, sorted by half window (largest first)
  int nsub;
  int total_items;
  int *err;
  unsigned long long timeout_ns;
};

// Many subjects (uneven sizes, atlas counts and NH in {7, 9, 11}), one persistent launch: work
// items of all subjects are numbered consecutively; each CTA walks the list with a grid stride
// and dispatches every item to the tile code of its subject's window.
template <int SET>
__global__ void __launch_bounds__(kThreads, TileOf<SET, 5>::MB) fuse_batch_kernel(const BatchParams bp) {
  extern __shared__ unsigned char smem_raw[];
  // The current subject's view, copied into shared memory when the subject changes: the tile
  // code then reads its fields from there as it needs them instead of keeping the values it
  // loaded from global memory in registers (the single-subject kernel reads them from its
  // parameters).
  __shared__ __align__(16) SubjectView s_sv;
  static_assert(sizeof(SubjectView) % 4 == 0 && sizeof(SubjectView) <= 4 * kThreads, "copy");
  Pipe pp = pipe_init(smem_raw);
  int s = 0, cur = -1;
  for (int item = blockIdx.x; item < bp.total_items; item += gridDim.x) {
    while (s + 1 < bp.nsub && bp.subjects[s + 1].item_begin <= item) ++s;
    if (s != cur) {  // uniform over the CTA
      __syncthreads();  // every thread is done with the previous subject's view
      if (threadIdx.x < sizeof(SubjectView) / 4)
        reinterpret_cast<int *>(&s_sv)[threadIdx.x] =
            reinterpret_cast<const int *>(bp.subjects + s)[threadIdx.x];
      __syncthreads();
      cur = s;
    }
    const SubjectView &sv = s_sv;
    const int local = item - sv.item_begin;
    bool ok = true;
    switch (sv.hw) {
      case 5: ok = run_item<5, TileOf<SET, 5>::RX, TileOf<SET, 5>::TZ, TileOf<SET, 5>::LY>(sv, local, pp, bp.err, bp.timeout_ns, -1); break;
      case 4: ok = run_item<4, TileOf<SET, 4>::RX, TileOf<SET, 4>::TZ, TileOf<SET, 4>::LY>(sv, local, pp, bp.err, bp.timeout_ns, -1); break;
      default: ok = run_item<3, TileOf<SET, 3>::RX, TileOf<SET, 3>::TZ, TileOf<SET, 3>::LY>(sv, local, pp, bp.err, bp.timeout_ns, -1); break;
    }
    if (!ok) {
      pipe_drain(pp, bp.timeout_ns);
      return;
    }
  }
}

// ---------------------------------------------------------------- host side

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void *ptr = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(ptr);
  }
  return fn;
}

}  // namespace

void *tensor_map_encoder() { return reinterpret_cast<void *>(encode_fn()); }

namespace {

// 4-D map over a pitched volume stack [num][nz][nx][pitch], box = one x-row slab of
// `box_z` planes x `box_y` columns. Out-of-volume elements read as zero.
cudaError_t make_slab_map(CUtensorMap *map, const float *base, int nx, int ny, int nz, int num,
                          int pitch, int box_y, int box_z) {
  auto fn = encode_fn();
  if (!fn) return cudaErrorNotSupported;
  const cuuint64_t dims[4] = {(cuuint64_t)ny, (cuuint64_t)nx, (cuuint64_t)nz, (cuuint64_t)num};
  const cuuint64_t strides[3] = {(cuuint64_t)pitch * 4, (cuuint64_t)pitch * 4 * nx,
                                 (cuuint64_t)pitch * 4 * nx * nz};
  const cuuint32_t box[4] = {(cuuint32_t)box_y, 1u, (cuuint32_t)box_z, 1u};
  const cuuint32_t estr[4] = {1u, 1u, 1u, 1u};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<float *>(base), dims, strides,
                  box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

// Sums the per-group partial (product, sum_weight) of every interior voxel of planes [z0, z1) in
// group order and applies the output rule, so the result does not depend on which CTA ran which
// group.
__global__ void combine_groups_kernel(const float *__restrict__ partial, int groups, int nx, int ny,
                                      int z0, int z1, int lo, long long nvox,
                                      float *__restrict__ out) {
  const int ix = nx - 2 * lo, iy = ny - 2 * lo;
  const long long total = (long long)ix * iy * (z1 - z0);
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int y = (int)(i % iy) + lo;
    const long long r = i / iy;
    const int x = (int)(r % ix) + lo;
    const int z = (int)(r / ix) + z0;
    const long long v = (long long)z * nx * ny + (long long)x * ny + y;
    float pr = 0.f, sw = 0.f;
    for (int g = 0; g < groups; ++g) {
      pr += partial[(2LL * g) * nvox + v];
      sw += partial[(2LL * g + 1) * nvox + v];
    }
    out[v] = fuse_result(pr, sw);
  }
}

// The combine over the interior planes [z0, z1) (clipped to the interior).
cudaError_t launch_combine_groups(const Geometry &g, const float *partial, int groups, float *out,
                                  int z0, int z1, cudaStream_t stream) {
  z0 = std::max(z0, g.lo);
  z1 = std::min(z1, g.nz - g.lo);
  if (z1 <= z0 || g.ix <= 0 || g.iy <= 0) return cudaSuccess;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  combine_groups_kernel<<<sms * 8, 256, 0, stream>>>(partial, groups, g.nx, g.ny, z0, z1, g.lo,
                                                     g.nvox(), out);
  return cudaGetLastError();
}

cudaError_t launch_combine_groups(const Geometry &g, const float *partial, int groups, float *out,
                                  cudaStream_t stream) {
  return launch_combine_groups(g, partial, groups, out, 0, g.nz, stream);
}

// Picks the number of atlas groups (a divisor of num) so that the work items fill the
// persistent grid's rounds: the first group count reaching 97% round occupancy, else the best.
int choose_groups(int ntiles, int num, int slots) {
  int best = 1;
  double best_eff = 0.0;
  for (int g = 1; g <= num; ++g) {
    if (num % g) continue;
    const double rounds = (double)ntiles * g / slots;
    const double eff = rounds / std::ceil(rounds);
    if (eff >= 0.97) return g;
    if (eff > best_eff + 1e-9) {
      best_eff = eff;
      best = g;
    }
  }
  return best;
}

int sm_count() {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms;
}

struct Plan {
  int blocks, groups, ntiles, tiles_y, tiles_x, tiles_z, rx, tz;
};

template <int SET, int HW>
cudaError_t plan_hw(const Geometry &g, Plan *pl) {
  constexpr int RX = TileOf<SET, HW>::RX, TZ = TileOf<SET, HW>::TZ, LY = TileOf<SET, HW>::LY;
  using C = Cfg<HW, RX, TZ>;
  auto kern = fuse_tma_kernel<HW, RX, TZ, LY, TileOf<SET, HW>::MB>;
  cudaError_t e;
  if ((e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM)) !=
      cudaSuccess)
    return e;
  int per_sm = 1;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, C::SMEM)) !=
      cudaSuccess)
    return e;
  if (per_sm < 1) return cudaErrorLaunchOutOfResources;
  pl->rx = RX;
  pl->tz = TZ;
  pl->tiles_y = (g.iy + kOutY - 1) / kOutY;
  pl->tiles_x = (g.ix + C::XC - 1) / C::XC;
  pl->tiles_z = (g.iz + 2 * TZ - 1) / (2 * TZ);
  pl->ntiles = pl->tiles_y * pl->tiles_x * pl->tiles_z;
  const int slots = sm_count() * per_sm;
  pl->groups = choose_groups(pl->ntiles, g.num, slots);
  const long long items = (long long)pl->ntiles * pl->groups;
  pl->blocks = (int)(items < slots ? items : slots);
  return cudaSuccess;
}

SubjectView subject_view(const Geometry &g, const SlabInputs &in, float *out, double div,
                         float *partial, const Plan &pl) {
  SubjectView sv{};
  sv.img = in.img;
  sv.out = out;
  sv.partial = partial;
  sv.nx = g.nx;
  sv.ny = g.ny;
  sv.nz = g.nz;
  sv.nxy = g.nx * g.ny;
  sv.nvox = g.nvox();
  sv.scale = (float)sqrt(1.4426950408889634 / div);
  sv.tiles_y = pl.tiles_y;
  sv.tiles_x = pl.tiles_x;
  sv.ntiles = pl.ntiles;
  sv.groups = pl.groups;
  sv.atlases_per_group = g.num / pl.groups;
  sv.hw = g.hw;
  return sv;
}

template <int SET, int HW>
cudaError_t launch_hw(const Geometry &g, const SlabInputs &in, float *out, double div,
                      float *partial, int *err, const LaunchHooks &wt, int item_begin, int item_end,
                      cudaStream_t stream) {
  constexpr int RX = TileOf<SET, HW>::RX, TZ = TileOf<SET, HW>::TZ;
  using C = Cfg<HW, RX, TZ>;
  Plan pl;
  cudaError_t e = plan_hw<SET, HW>(g, &pl);
  if (e != cudaSuccess) return e;
  if (pl.groups > 1 && !partial) return cudaErrorInvalidValue;
  const bool whole = item_begin < 0;  // every item, then the combine
  if (whole) {
    item_begin = 0;
    item_end = pl.groups * pl.ntiles;
  } else if (pl.groups < 2 || item_begin >= item_end || item_end > pl.groups * pl.ntiles) {
    return cudaErrorInvalidValue;  // an item range needs partial sums and a later combine
  }
  CUtensorMap tmA, tmL;
  if ((e = make_slab_map(&tmA, in.atlas, g.nx, g.ny, g.nz, g.num, in.pitch, C::YB, C::ZA)) !=
      cudaSuccess)
    return e;
  if ((e = make_slab_map(&tmL, in.label, g.nx, g.ny, g.nz, g.num, in.pitch, C::YB, C::ZL)) !=
      cudaSuccess)
    return e;
  TmaParams p{};
  p.sv = subject_view(g, in, out, div, partial, pl);
  p.err = err;
  p.timeout_ns = 2000000000ull;  // 2 s per wait; a step's copies land in microseconds
  p.withhold_cta = -1;
  if (wt.timeout_ns) {
    p.timeout_ns = wt.timeout_ns;
    p.withhold_cta = 0;
  }
  p.item_begin = item_begin;
  p.item_end = item_end;
  const int blocks = std::min(pl.blocks, p.item_end - p.item_begin);
  if (wt.start && (e = cudaEventRecord(wt.start, stream)) != cudaSuccess) return e;
  fuse_tma_kernel<HW, RX, TZ, TileOf<SET, HW>::LY, TileOf<SET, HW>::MB>
      <<<blocks, kThreads, C::SMEM, stream>>>(tmA, tmL, p);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if (wt.stop && (e = cudaEventRecord(wt.stop, stream)) != cudaSuccess) return e;
  if (whole && pl.groups > 1) return launch_combine_groups(g, partial, pl.groups, out, stream);
  return cudaSuccess;
}

template <int SET>
cudaError_t plan_set(const Geometry &g, Plan *pl) {
  switch (g.hw) {
    case 1: return plan_hw<SET, 1>(g, pl);
    case 2: return plan_hw<SET, 2>(g, pl);
    case 3: return plan_hw<SET, 3>(g, pl);
    case 4: return plan_hw<SET, 4>(g, pl);
    case 5: return plan_hw<SET, 5>(g, pl);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t plan_any(const Geometry &g, int set, Plan *pl) {
  switch (set) {
    case 0: return plan_set<0>(g, pl);
    case 1: return plan_set<1>(g, pl);
    case 2: return plan_set<2>(g, pl);
    case 3: return plan_set<3>(g, pl);
    case 4: return plan_set<4>(g, pl);
    default: return cudaErrorInvalidValue;
  }
}

template <int SET>
cudaError_t launch_set(const Geometry &g, const SlabInputs &in, float *out, double div,
                       float *partial, int *err, const LaunchHooks &wt, int ib, int ie,
                       cudaStream_t stream) {
  switch (g.hw) {
    case 1: return launch_hw<SET, 1>(g, in, out, div, partial, err, wt, ib, ie, stream);
    case 2: return launch_hw<SET, 2>(g, in, out, div, partial, err, wt, ib, ie, stream);
    case 3: return launch_hw<SET, 3>(g, in, out, div, partial, err, wt, ib, ie, stream);
    case 4: return launch_hw<SET, 4>(g, in, out, div, partial, err, wt, ib, ie, stream);
    case 5: return launch_hw<SET, 5>(g, in, out, div, partial, err, wt, ib, ie, stream);
    default: return cudaErrorInvalidValue;
  }
}

// Slab box sizes of one subject under a tile set (for its tensor maps in the batch).
template <int SET, int HW>
void boxes_hw(int *yb, int *za, int *zl) {
  using C = Cfg<HW, TileOf<SET, HW>::RX, TileOf<SET, HW>::TZ>;
  *yb = C::YB;
  *za = C::ZA;
  *zl = C::ZL;
}

template <int SET>
cudaError_t batch_plan(int hw, const Geometry &g, Plan *pl, int *yb, int *za, int *zl) {
  cudaError_t e;
  switch (hw) {
    case 5: e = plan_hw<SET, 5>(g, pl); boxes_hw<SET, 5>(yb, za, zl); break;
    case 4: e = plan_hw<SET, 4>(g, pl); boxes_hw<SET, 4>(yb, za, zl); break;
    case 3: e = plan_hw<SET, 3>(g, pl); boxes_hw<SET, 3>(yb, za, zl); break;
    default: return cudaErrorInvalidValue;
  }
  return e;
}

template <int SET>
cudaError_t launch_batch_set(const BatchSubjectIn *subs, int n, void *dev_scratch, int *err,
                             cudaStream_t stream, BatchSetup *setup) {
  // Order subjects by window (largest first), so CTAs working at the same time mostly run the
  // same tile code.
  std::vector<int> order(n);
  for (int i = 0; i < n; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return subs[a].geom.hw > subs[b].geom.hw; });
  std::vector<SubjectView> views(n);
  std::vector<CUtensorMap> maps(2 * (size_t)n);
  int total = 0;
  cudaError_t e;
  for (int k = 0; k < n; ++k) {
    const BatchSubjectIn &b = subs[order[k]];
    Plan pl;
    int yb, za, zl;
    if ((e = batch_plan<SET>(b.geom.hw, b.geom, &pl, &yb, &za, &zl)) != cudaSuccess) return e;
    pl.groups = 1;  // many subjects fill the grid; no partial sums
    if ((e = make_slab_map(&maps[2 * k], b.in.atlas, b.geom.nx, b.geom.ny, b.geom.nz, b.geom.num,
                           b.in.pitch, yb, za)) != cudaSuccess)
      return e;
    if ((e = make_slab_map(&maps[2 * k + 1], b.in.label, b.geom.nx, b.geom.ny, b.geom.nz,
                           b.geom.num, b.in.pitch, yb, zl)) != cudaSuccess)
      return e;
    SubjectView sv = subject_view(b.geom, b.in, b.out, b.div, nullptr, pl);
    sv.item_begin = total;
    total += (b.geom.ix > 0 && b.geom.iy > 0 && b.geom.iz > 0) ? pl.ntiles : 0;
    views[k] = sv;
  }
  // Device copies: maps first (64-byte aligned), then the subject views pointing at them.
  unsigned char *base = static_cast<unsigned char *>(dev_scratch);
  CUtensorMap *d_maps = reinterpret_cast<CUtensorMap *>(base);
  SubjectView *d_views = reinterpret_cast<SubjectView *>(base + maps.size() * sizeof(CUtensorMap));
  for (int k = 0; k < n; ++k) {
    views[k].tmA = d_maps + 2 * k;
    views[k].tmL = d_maps + 2 * k + 1;
  }
  if ((e = cudaMemcpyAsync(d_maps, maps.data(), maps.size() * sizeof(CUtensorMap),
                           cudaMemcpyHostToDevice, stream)) != cudaSuccess)
    return e;
  if ((e = cudaMemcpyAsync(d_views, views.data(), views.size() * sizeof(SubjectView),
                           cudaMemcpyHostToDevice, stream)) != cudaSuccess)
    return e;
  // Host copies must outlive the asynchronous transfers.
  if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) return e;

  constexpr int smem = batch_smem<SET>();
  auto kern = fuse_batch_kernel<SET>;
  if ((e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) !=
      cudaSuccess)
    return e;
  int per_sm = 1;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, smem)) !=
      cudaSuccess)
    return e;
  if (per_sm < 1) return cudaErrorLaunchOutOfResources;
  const int slots = sm_count() * per_sm;
  setup->params_ready = true;
  setup->items = total;
  setup->blocks = total < slots ? total : slots;
  setup->smem = smem;
  setup->set = SET;
  setup->bp_subjects = d_views;
  setup->bp_nsub = n;
  setup->bp_err = err;
  return cudaSuccess;
}

}  // namespace

size_t batch_scratch_bytes(int n) {
  return 2 * (size_t)n * sizeof(CUtensorMap) + (size_t)n * sizeof(SubjectView) + 256;
}

cudaError_t prepare_batch(const BatchSubjectIn *subs, int n, int set, void *dev_scratch, int *err,
                          cudaStream_t stream, BatchSetup *setup) {
  for (int i = 0; i < n; ++i)
    if (subs[i].geom.hw < 3 || subs[i].geom.hw > 5) return cudaErrorInvalidValue;
  switch (set) {
    case 0: return launch_batch_set<0>(subs, n, dev_scratch, err, stream, setup);
    case 1: return launch_batch_set<1>(subs, n, dev_scratch, err, stream, setup);
    case 2: return launch_batch_set<2>(subs, n, dev_scratch, err, stream, setup);
    case 3: return launch_batch_set<3>(subs, n, dev_scratch, err, stream, setup);
    case 4: return launch_batch_set<4>(subs, n, dev_scratch, err, stream, setup);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_prepared_batch(const BatchSetup &setup, cudaStream_t stream) {
  if (!setup.params_ready) return cudaErrorInvalidValue;
  if (setup.items == 0) return cudaSuccess;
  BatchParams bp{static_cast<const SubjectView *>(setup.bp_subjects), setup.bp_nsub, setup.items,
                 setup.bp_err, 2000000000ull};
  switch (setup.set) {
    case 0: fuse_batch_kernel<0><<<setup.blocks, kThreads, setup.smem, stream>>>(bp); break;
    case 1: fuse_batch_kernel<1><<<setup.blocks, kThreads, setup.smem, stream>>>(bp); break;
    case 2: fuse_batch_kernel<2><<<setup.blocks, kThreads, setup.smem, stream>>>(bp); break;
    case 3: fuse_batch_kernel<3><<<setup.blocks, kThreads, setup.smem, stream>>>(bp); break;
    case 4: fuse_batch_kernel<4><<<setup.blocks, kThreads, setup.smem, stream>>>(bp); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

TileShape fuse_tile_shape(const Geometry &g) {
  using T = TileOf<0, 5>;
  TileShape t{};
  t.out_y = kOutY;
  t.xc = kWarps * T::RX;
  t.zt = 2 * T::TZ;
  if (g.ix > 0 && g.iy > 0 && g.iz > 0) {
    t.tiles_y = (g.iy + kOutY - 1) / kOutY;
    t.tiles_x = (g.ix + t.xc - 1) / t.xc;
    t.tiles_z = (g.iz + t.zt - 1) / t.zt;
  }
  return t;
}

namespace {

// One masked item per pair of flagged atlases of every tile with a non-empty mask (any order:
// each item writes its own partial slot).
__global__ void masked_items_kernel(const uint32_t *__restrict__ masks, int ntiles,
                                    int *__restrict__ items, int *__restrict__ count) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntiles; t += gridDim.x * blockDim.x) {
    const uint32_t m = masks[t];
    if (!m) continue;
    const int pairs = (__popc(m) + 1) / 2;
    const int at = atomicAdd(count, pairs);
    for (int k = 0; k < pairs; ++k) items[at + k] = (k << 24) | t;
  }
}

// Adds the pair slots of every interior voxel of a masked tile into acc_p / acc_w, in pair order.
__global__ void masked_combine_kernel(const uint32_t *__restrict__ masks, const TileShape ts,
                                      int nx, int ny, int nz, int lo, long long nvox,
                                      const float *__restrict__ partial, float *__restrict__ acc_p,
                                      float *__restrict__ acc_w) {
  const int ix = nx - 2 * lo, iy = ny - 2 * lo, iz = nz - 2 * lo;
  const long long total = (long long)ix * iy * iz;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int yi = (int)(i % iy);
    const long long r = i / iy;
    const int xi = (int)(r % ix), zi = (int)(r / ix);
    const int t = ((zi / ts.zt) * ts.tiles_x + xi / ts.xc) * ts.tiles_y + yi / ts.out_y;
    const uint32_t m = masks[t];
    if (!m) continue;
    const long long v = (long long)(zi + lo) * nx * ny + (long long)(xi + lo) * ny + (yi + lo);
    float p = acc_p[v], w = acc_w[v];
    for (int k = 0; k < (__popc(m) + 1) / 2; ++k) {
      p += partial[(2LL * k) * nvox + v];
      w += partial[(2LL * k + 1) * nvox + v];
    }
    acc_p[v] = p;
    acc_w[v] = w;
  }
}

}  // namespace

cudaError_t launch_fuse_masked(const Geometry &g, const SlabInputs &in, double div, int atlas_base,
                               const uint32_t *masks, int *items, int *count, float *partial,
                               float *acc_p, float *acc_w, int *err, cudaStream_t stream) {
  if (g.hw != 5 || atlas_base < 0 || atlas_base >= g.num) return cudaErrorInvalidValue;
  if (g.ix <= 0 || g.iy <= 0 || g.iz <= 0) return cudaSuccess;
  using T = TileOf<0, 5>;
  using C = Cfg<5, T::RX, T::TZ>;
  auto kern = fuse_list_kernel<5, T::RX, T::TZ, T::LY, T::MB>;
  cudaError_t e;
  if ((e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM)) !=
      cudaSuccess)
    return e;
  int per_sm = 1;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, C::SMEM)) !=
      cudaSuccess)
    return e;
  if (per_sm < 1) return cudaErrorLaunchOutOfResources;
  CUtensorMap tmA, tmL;
  if ((e = make_slab_map(&tmA, in.atlas, g.nx, g.ny, g.nz, g.num, in.pitch, C::YB, C::ZA)) !=
      cudaSuccess)
    return e;
  if ((e = make_slab_map(&tmL, in.label, g.nx, g.ny, g.nz, g.num, in.pitch, C::YB, C::ZL)) !=
      cudaSuccess)
    return e;
  const TileShape ts = fuse_tile_shape(g);
  const int ntiles = ts.tiles_y * ts.tiles_x * ts.tiles_z;
  if (ntiles >= (1 << 24)) return cudaErrorInvalidValue;  // items pack the tile in 24 bits
  if ((e = cudaMemsetAsync(count, 0, sizeof(int), stream)) != cudaSuccess) return e;
  masked_items_kernel<<<(ntiles + 255) / 256, 256, 0, stream>>>(masks, ntiles, items, count);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  Plan pl{};
  pl.tiles_y = ts.tiles_y;
  pl.tiles_x = ts.tiles_x;
  pl.tiles_z = ts.tiles_z;
  pl.ntiles = ntiles;
  pl.groups = 2;  // partial slots (the pair of each item), not a plan's atlas groups
  TmaParams p{};
  p.sv = subject_view(g, in, nullptr, div, partial, pl);
  p.sv.atlas_base = atlas_base;
  p.sv.atlas_mask = masks;
  p.err = err;
  p.timeout_ns = 2000000000ull;
  p.withhold_cta = -1;
  kern<<<sm_count() * per_sm, kThreads, C::SMEM, stream>>>(tmA, tmL, p, items, count);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  masked_combine_kernel<<<sm_count() * 8, 256, 0, stream>>>(masks, ts, g.nx, g.ny, g.nz, g.lo,
                                                            g.nvox(), partial, acc_p, acc_w);
  return cudaGetLastError();
}

size_t fuse_tma_partial_bytes(const Geometry &g, int set) {
  if (g.ix <= 0 || g.iy <= 0 || g.iz <= 0) return 0;
  Plan pl;
  if (plan_any(g, set, &pl) != cudaSuccess || pl.groups <= 1) return 0;
  return (size_t)pl.groups * 2 * (size_t)g.nvox() * sizeof(float);
}

cudaError_t fuse_tma_plan(const Geometry &g, int set, FusePlanInfo *info) {
  *info = FusePlanInfo{0, 0, 0, 0, 0, 0, 0, 0};
  if (g.ix <= 0 || g.iy <= 0 || g.iz <= 0) return cudaSuccess;
  Plan pl;
  cudaError_t e = plan_any(g, set, &pl);
  if (e != cudaSuccess) return e;
  info->groups = pl.groups;
  info->tiles = pl.ntiles;
  info->ctas = pl.blocks;
  info->rx = pl.rx;
  info->tz = pl.tz;
  info->partial_bytes =
      pl.groups > 1 ? (size_t)pl.groups * 2 * (size_t)g.nvox() * sizeof(float) : 0;
  info->tiles_z = pl.tiles_z;
  info->tiles_xy = pl.tiles_y * pl.tiles_x;
  return cudaSuccess;
}

int fuse_tma_planes_read(const Geometry &g, const FusePlanInfo &info, int ztiles) {
  // z-tile tz reads the atlas MRI slab [2 tz TZ, 2 tz TZ + 2 TZ + 2 + 2 HW) (its first output
  // plane minus the box and window reach), the CT slab and the input taps lie inside it
  const long long n = (long long)ztiles * 2 * info.tz + 2 + 2 * g.hw;
  return ztiles <= 0 ? 0 : (int)(n < g.nz ? n : g.nz);
}

cudaError_t launch_fuse_tma(const Geometry &g, const SlabInputs &in, float *out, double div,
                            float *partial, int *err, const LaunchHooks &wt, int set,
                            cudaStream_t stream) {
  if (g.ix <= 0 || g.iy <= 0 || g.iz <= 0) return cudaSuccess;
  switch (set) {
    case 0: return launch_set<0>(g, in, out, div, partial, err, wt, -1, -1, stream);
    case 1: return launch_set<1>(g, in, out, div, partial, err, wt, -1, -1, stream);
    case 2: return launch_set<2>(g, in, out, div, partial, err, wt, -1, -1, stream);
    case 3: return launch_set<3>(g, in, out, div, partial, err, wt, -1, -1, stream);
    case 4: return launch_set<4>(g, in, out, div, partial, err, wt, -1, -1, stream);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_fuse_tma_items(const Geometry &g, const SlabInputs &in, double div,
                                  float *partial, int *err, int set, int item_begin, int item_end,
                                  cudaStream_t stream) {
  if (g.ix <= 0 || g.iy <= 0 || g.iz <= 0) return cudaSuccess;
  if (item_begin < 0) return cudaErrorInvalidValue;
  const LaunchHooks wt{0, nullptr, nullptr};
  switch (set) {
    case 0: return launch_set<0>(g, in, nullptr, div, partial, err, wt, item_begin, item_end, stream);
    case 1: return launch_set<1>(g, in, nullptr, div, partial, err, wt, item_begin, item_end, stream);
    case 2: return launch_set<2>(g, in, nullptr, div, partial, err, wt, item_begin, item_end, stream);
    case 3: return launch_set<3>(g, in, nullptr, div, partial, err, wt, item_begin, item_end, stream);
    case 4: return launch_set<4>(g, in, nullptr, div, partial, err, wt, item_begin, item_end, stream);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_fuse_tma_combine(const Geometry &g, const float *partial, int set, float *out,
                                    int z_begin, int z_end, cudaStream_t stream) {
  if (g.ix <= 0 || g.iy <= 0 || g.iz <= 0) return cudaSuccess;
  Plan pl;
  cudaError_t e = plan_any(g, set, &pl);
  if (e != cudaSuccess) return e;
  if (pl.groups < 2) return cudaErrorInvalidValue;
  return launch_combine_groups(g, partial, pl.groups, out, z_begin, z_end, stream);
}

namespace {
// One warp per row (grid-stride over rows), so that no element index is divided by the row
// length; PAIRS copies 8-byte pairs (even ny and an 8-byte aligned source; the destination's
// pitch is a multiple of 4 floats).
template <bool PAIRS>
__global__ void pitch_copy_kernel(const float *__restrict__ src, float *__restrict__ dst,
                                  long long rows, int ny, int pitch) {
  const int lane = threadIdx.x & 31;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long r = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < rows;
       r += nwarps) {
    const float *s = src + r * ny;
    float *d = dst + r * pitch;
    if constexpr (PAIRS) {
      const float2 *s2 = reinterpret_cast<const float2 *>(s);
      float2 *d2 = reinterpret_cast<float2 *>(d);
#pragma unroll 4
      for (int c = lane; c < ny / 2; c += 32) d2[c] = s2[c];
    } else {
#pragma unroll 4
      for (int c = lane; c < ny; c += 32) d[c] = s[c];
    }
  }
}
}  // namespace

cudaError_t launch_pitch_copy(const float *src, float *dst, long long rows, int ny, int pitch,
                              cudaStream_t stream) {
  if (rows <= 0) return cudaSuccess;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (ny % 2 == 0 && reinterpret_cast<uintptr_t>(src) % 8 == 0 &&
      reinterpret_cast<uintptr_t>(dst) % 16 == 0 && pitch % 4 == 0)
    pitch_copy_kernel<true><<<sms * 8, 256, 0, stream>>>(src, dst, rows, ny, pitch);
  else
    pitch_copy_kernel<false><<<sms * 8, 256, 0, stream>>>(src, dst, rows, ny, pitch);
  return cudaGetLastError();
}

}  // namespace pct
