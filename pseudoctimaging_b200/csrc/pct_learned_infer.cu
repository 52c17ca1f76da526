// Inference side of the learned proposal (EXEC_CHOICE 7).
//
// Per atlas, over the whole volume:
//   conv1 (2 -> 16 channels)            tcgen05: FP16 operands (y taps folded into K), FP32 in TMEM
//   conv2..conv4 (16 -> 16 channels)    tcgen05: BF16 implicit GEMM, FP32 in TMEM
//   heads, proposal and rescoring       row segments of 30 voxels along y: per voxel the 33
//                                       logits and a softmax per axis; the summed probabilities of
//                                       a block's anchor segment pick 4 offsets per axis and the
//                                       rank triples with i + j + k <= L (L = 4, 3, 2: 32, 20 or
//                                       10 offsets); the exact FP32 SSD of those candidates ->
//                                       weights exp(-SSD/div) -> product and weight sums. A voxel
//                                       whose own probability mass on the kept set is below the
//                                       confidence threshold takes all 11^3.
// The sums are kept per voxel across atlases and turned into the output with the reference's
// NaN rule at the end. Out-of-volume inputs of the convolutions read as zero; interior voxels
// (6 or more voxels from every face) only see in-volume values.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdlib.h>
#include <stdint.h>

#include <cuda.h>
#include <cudaTypedefs.h>

#include <array>
#include <algorithm>
#include <vector>

#include "pct_internal.h"
#include "pct_learned.h"
#include "pct_ptx.cuh"

namespace pct {
namespace learned {
namespace {

constexpr float kDblEpsilonF = 2.220446049250313080847e-16f;
constexpr int kFallbackAtlases = 32;  // atlases per full-search launch of the fallback (mask bits)


// ---------------------------------------------------------------- conv1 (tensor cores)

// ---------------------------------------------------------------- conv 16 -> 16 (tcgen05)

// Feature volumes are BF16 with the 16 channels split in two halves of 8: half h of voxel v at
// element (h * nvox + v) * 8, so that a run of voxels of one half is a run of 16-byte rows.
//
// conv 16 -> 16 is an implicit GEMM on tcgen05: M = 128 consecutive y of one output x-row (126
// stored), K = 16 input channels per tap. A CTA work item is a column of 4 x-rows x 126 y over a
// run of consecutive output z-planes; its input planes z0 - 1 .. z0 + planes stream through a
// 2-slot ring of shared memory, one TMA box per plane ([half][x][y][8 channels], 6 x-rows of 128
// y from y0 - 1; each (half, x) row is one 2 KB line read as 256 8-byte elements), which is the
// canonical K-major no-swizzle operand layout (8-row core matrices of 16-byte rows, the two
// halves LBO apart). The A operand for input row ix at y shift ky is a descriptor start address
// in the plane's slot (its rows 126 and 127 run into the next row and feed only the MMA rows 126
// and 127, which are not stored).
//
// An input row (plane p, row ix, shift ky) feeds the output rows o = ix - kx (kx = 0..2) of the
// three output planes p + 1 - kz (kz = 0..2). The accumulators of three consecutive output planes
// live in TMEM as a ring of plane slots r = z mod 3, column 16 (3 o + r) + channel, so the nine
// (kz, kx) blocks an input row feeds are adjacent columns: one MMA with N = 48 x (rows fed) <= 144
// covers them. Its B operand is a weight sequence ordered the same way, W(kz = (rho - r) mod 3,
// kx, ky) for kx = 2, 1, 0 and r = 0, 1, 2, stored for each ky and rotation rho = (p + 1) mod 3.
// 18 MMAs per input plane; after the MMAs of plane p the output plane p - 1 is complete, and the
// epilogue reads it, zeroes its slot for plane p + 2 and then stores it. The first two and last
// two outputs of an item are the run's halo and are only zeroed; an item of one plane reuses no
// slot, so its three input planes run back to back and it is finalised once.
//
// Warp roles: warps 0-3 epilogue (TMEM lane quarter = warp, one voxel per thread: bias, ReLU,
// BF16 store, zeroing), warp 4 the TMA producer, warp 5 the MMA issuer (the whole warp computes
// the operands, one elected lane issues). Two CTAs share each SM, so one CTA's MMAs overlap the
// other's epilogue; every wait is bounded.
constexpr int kCvTX = 4, kCvTY = 126;  // output x-rows and stored y per item column (M = 128)
constexpr int kCvSX = kCvTX + 2, kCvSY = 128;
constexpr int kCvHalf = kCvSX * kCvSY * 16;                          // 12,288 B
constexpr int kCvPlane = 2 * kCvHalf;                                // 24,576 B per ring slot
constexpr int kCvRing = 2;                                           // input-plane slots
constexpr int kCvChunk = 13;                                         // max output planes per item
constexpr int kCvSeqRows = 144;                                      // 9 blocks of 16 channels
constexpr int kCvSeq = 2 * kCvSeqRows * 16;                          // 4,608 B per (ky, rho)
constexpr int kCvWBytes = 9 * kCvSeq;                                // 41,472 B
constexpr int kCvCols = 256;                                         // 3 plane slots x 64 used
constexpr int kCvThreads = 192;
constexpr size_t kConvSmem = 128 + kCvRing * kCvPlane + kCvWBytes + 128;  // 2 CTAs per SM
constexpr int kFragWords = kCvWBytes / 4;  // per layer: the weight sequences as stored in smem
constexpr unsigned long long kConvTimeoutNs = 2000000000ULL;

// Upper bound of one layer's work items: x tiles x y tiles x planes.
long long conv_items_bound(const Geometry &g) {
  return (long long)g.nx * ((g.ny + kCvTY - 1) / kCvTY) * g.nz;
}

size_t conv_list_bytes(const Geometry &g) {
  return (4 * (size_t)g.nx + 2 * 4 * (size_t)conv_items_bound(g) + 8) * sizeof(int);
}

// Weight sequences of one layer: sequence q = 3 ky + rho, byte offset q * 4608 + h * 2304 +
// n * 16 + 2 c8 holds W[co][8h + c8][kz * 9 + kx * 3 + ky] for row n = 16 (3 kxi + r) + co,
// kx = 2 - kxi, kz = (rho - r) mod 3.
__global__ void pack_frags_kernel(const __nv_bfloat16 *__restrict__ wbf, int woff,
                                  uint32_t *__restrict__ frag) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kFragWords) return;
  const int off = 4 * i;
  const int q = off / kCvSeq, h = (off % kCvSeq) / (kCvSeqRows * 16);
  const int n = (off % (kCvSeqRows * 16)) / 16, c8 = (off % 16) / 2;
  const int ky = q / 3, rho = q % 3, blk = n / 16, co = n % 16, ci = 8 * h + c8;
  const int kx = 2 - blk / 3, r = blk % 3, kz = (rho - r + 3) % 3;
  const int t = kz * 9 + kx * 3 + ky;
  const __nv_bfloat16 lo = wbf[woff + (co * kC + ci) * 27 + t];
  const __nv_bfloat16 hi = wbf[woff + (co * kC + ci + 1) * 27 + t];
  frag[i] = (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

// The output region of one layer: work items {x tile | y tile << 16, first plane | planes << 16}
// over x tiles of 4 rows (first row | mask of the rows to compute << 16; NULL: 4i, all rows) and
// y tiles of 126 from y_lo.
struct ConvGrid {
  int nx, ny, nz;
  int y_lo, y_hi, tile_y;
  int n_items;
  long long nvox;
  const int2 *items;
  const int *xlist;
};

struct ConvItem {
  int x0, y0, z0, planes;
  unsigned mask;
};

__device__ __forceinline__ ConvItem conv_item(const ConvGrid &g, int i) {
  const int2 e = g.items[i];
  ConvItem r;
  const int xi = e.x & 0xFFFF, ty = (int)((unsigned)e.x >> 16);
  if (g.xlist) {
    const int xe = g.xlist[xi];
    r.x0 = xe & 0xFFFF;
    r.mask = (unsigned)xe >> 16;
  } else {
    r.x0 = xi * kCvTX;
    r.mask = 0xFu;
  }
  r.y0 = g.y_lo + ty * g.tile_y;
  r.z0 = e.y & 0xFFFF;
  r.planes = (int)((unsigned)e.y >> 16);
  return r;
}

namespace tc5 {

__device__ __forceinline__ uint64_t desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  // K-major, no swizzle: start >> 4 | LBO >> 4 | SBO >> 4 | descriptor version 1
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ uint32_t idesc_bf16(int n) {
  // D FP32, A and B BF16 (K-major), N, M = 128
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((128u >> 4) << 24);
}

// MMA (accumulating) and commit, issued by one elected lane of a converged warp: the warp
// computes the operands together, which keeps them warp-uniform.
__device__ __forceinline__ void mma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc) {
  asm volatile(
      "{\n\t.reg .pred e, p;\n\telect.sync _|e, 0xffffffff;\n\t"
      "setp.ne.b32 p, 1, 0;\n\t"
      "@e tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc)
      : "memory");
}

__device__ __forceinline__ void commit(uint32_t bar) {
  asm volatile(
      "{\n\t.reg .pred e;\n\telect.sync _|e, 0xffffffff;\n\t"
      "@e tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n\t}" ::"r"(bar)
      : "memory");
}

__device__ __forceinline__ void fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}

__device__ __forceinline__ void st16_zero(uint32_t taddr) {
  const uint32_t z = 0u;
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, "
      "%1, %1, %1, %1, %1};" ::"r"(taddr),
      "r"(z)
      : "memory");
}

__device__ __forceinline__ void wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

}  // namespace tc5

__global__ void __launch_bounds__(kCvThreads, 2)
    conv16_kernel(const __grid_constant__ CUtensorMap tm, const uint32_t *__restrict__ frag,
                  const __nv_bfloat16 *__restrict__ wbf, int boff, __nv_bfloat16 *__restrict__ out,
                  ConvGrid g, int *__restrict__ err) {
  extern __shared__ unsigned char smem_raw[];
  const uint32_t raw = ptx::smem_u32(smem_raw);
  const uint32_t base = (raw + 127u) & ~127u;
  const uint32_t wtab = base + kCvRing * kCvPlane;
  // barriers: full[ring], empty[ring], mdone (MMAs of an input plane complete), zeroed[3]
  const uint32_t full0 = wtab + kCvWBytes, empty0 = full0 + 8 * kCvRing;
  const uint32_t mdone = empty0 + 8 * kCvRing, zeroed0 = mdone + 8;
  unsigned char *gen = smem_raw + (zeroed0 + 24 - raw);
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(gen);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(gen + 4);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

  // weight sequences into shared memory (visible to the tensor core through the async proxy)
  {
    uint32_t *w = reinterpret_cast<uint32_t *>(smem_raw + (wtab - raw));
    for (int i = threadIdx.x; i < kFragWords; i += kCvThreads) w[i] = __ldg(frag + i);
    ptx::fence_proxy_async_smem();
  }
  if (threadIdx.x == 0) {
    for (int i = 0; i < kCvRing; ++i) {
      ptx::mbar_init(full0 + 8 * i, 1);
      ptx::mbar_init(empty0 + 8 * i, 1);
    }
    ptx::mbar_init(mdone, 1);
    for (int i = 0; i < 3; ++i) ptx::mbar_init(zeroed0 + 8 * i, 4);
    *abort_flag = 0;
    ptx::fence_mbarrier_init();
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     ptx::smem_u32(tmem_slot)),
                 "r"(kCvCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc5::fence_before();
  __syncthreads();
  tc5::fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 4) {
    // TMA producer: the input planes z0 - 1 .. z0 + planes of every item, in order, into the ring
    if (lane == 0) {
      uint32_t j = 0;  // planes issued
      for (int it = blockIdx.x; it < g.n_items && !*abort_flag; it += gridDim.x) {
        const ConvItem c = conv_item(g, it);
        for (int p = 0; p < c.planes + 2; ++p, ++j) {
          const uint32_t slot = j % kCvRing;
          if (j >= kCvRing &&
              !ptx::mbar_wait_bounded(empty0 + 8 * slot, ((j / kCvRing) - 1) & 1, kConvTimeoutNs)) {
            *abort_flag = 1;
            break;
          }
          ptx::mbar_arrive_expect_tx(full0 + 8 * slot, kCvPlane);
          ptx::tma_load_4d(base + slot * kCvPlane, &tm, full0 + 8 * slot, 2 * (c.y0 - 1), c.x0 - 1,
                           c.z0 - 1 + p, 0);
        }
      }
      // planes still landing: wait for the last ring's worth (bounded)
      for (uint32_t q = j > kCvRing ? j - kCvRing : 0; q < j; ++q)
        if (!ptx::mbar_wait_bounded(full0 + 8 * (q % kCvRing), (q / kCvRing) & 1, kConvTimeoutNs))
          *abort_flag = 1;  // reported as a timeout
    }
  } else if (warp == 5) {
    // MMA issuer: the whole warp runs the loop, one elected lane issues
    uint32_t j = 0;              // input planes consumed
    uint32_t nz[3] = {1, 1, 1};  // completed zeroings each plane slot must reach (initial one)
    const uint64_t db0 = tc5::desc(wtab, kCvSeqRows * 16, 128);
    for (int it = blockIdx.x; it < g.n_items && !*abort_flag; it += gridDim.x) {
      const ConvItem c = conv_item(g, it);
      bool ok = true;
      for (int p = 0; p < c.planes + 2 && ok; ++p, ++j) {
        const int zin = c.z0 - 1 + p;  // input plane; feeds output planes zin - 1 .. zin + 1
        // the slots of the outputs this plane feeds must be zeroed: all three at the first plane
        // of an item, else the one that output zin + 1 takes over (an item of one plane reuses
        // no slot and waits only at its start)
        for (int r = 0; r < 3 && ok; ++r)
          if (p == 0 || (c.planes > 1 && r == (zin + 1 + 3) % 3))
            ok = ptx::mbar_wait_bounded(zeroed0 + 8 * r, (nz[r] - 1) & 1, kConvTimeoutNs);
        ok = ok && ptx::mbar_wait_bounded(full0 + 8 * (j % kCvRing), (j / kCvRing) & 1,
                                          kConvTimeoutNs);
        if (!ok) {
          *abort_flag = 1;
          break;
        }
        tc5::fence_after();
        const uint64_t da = tc5::desc(base + (j % kCvRing) * kCvPlane, kCvHalf, 128);
        const int rho = (zin + 1 + 3) % 3;
#pragma unroll 1
        for (int ix = 0; ix < kCvSX; ++ix) {
          int o_lo = ix - 2 < 0 ? 0 : ix - 2, o_hi = ix < kCvTX - 1 ? ix : kCvTX - 1;
          while (o_lo <= o_hi && !((c.mask >> o_lo) & 1u)) ++o_lo;
          while (o_hi >= o_lo && !((c.mask >> o_hi) & 1u)) --o_hi;
          if (o_lo > o_hi) continue;
          const uint32_t id = tc5::idesc_bf16(48 * (o_hi - o_lo + 1));
          const uint32_t d = tmem + 48 * o_lo;
          // descriptor start fields count 16-byte units: sequence (ky, rho), block 3 (2 - ix + o_lo)
          const uint64_t db = db0 + (uint64_t)(rho * (kCvSeq / 16) + 3 * (2 - ix + o_lo) * 16);
#pragma unroll
          for (int ky = 0; ky < 3; ++ky)
            tc5::mma(d, da + (uint64_t)(ix * kCvSY + ky), db + (uint64_t)(ky * 3 * (kCvSeq / 16)),
                     id);
        }
        tc5::commit(empty0 + 8 * (j % kCvRing));
        tc5::commit(mdone);
        // output zin - 1 completes with this plane; its slot is zeroed next (and, at the end of
        // the item, the two halo outputs after it); a one-plane item zeroes all three at its end
        if (c.planes > 1 || p == c.planes + 1) nz[(zin - 1 + 3) % 3] += 1;
        if (p == c.planes + 1) {
          nz[(zin + 3) % 3] += 1;
          nz[(zin + 1 + 3) % 3] += 1;
        }
      }
    }
    // let every issued MMA finish before the accumulators are released (bounded)
    if (j > 0 && !ptx::mbar_wait_bounded(mdone, (j - 1) & 1, kConvTimeoutNs))
      *abort_flag = 1;  // reported as a timeout
  } else {
    // epilogue: warp w reads TMEM lanes 32w..32w+31 = output y0 + 32w + lane
    const uint32_t lane_addr = tmem + ((uint32_t)(32 * warp) << 16);
    float bias[kC];
#pragma unroll
    for (int c = 0; c < kC; ++c) bias[c] = __bfloat162float(wbf[boff + c]);
    // every plane slot starts at zero
#pragma unroll
    for (int q = 0; q < 12; ++q) tc5::st16_zero(lane_addr + 16 * q);
    tc5::wait_st();
    tc5::fence_before();
    __syncwarp();
    if (lane == 0)
      for (int r = 0; r < 3; ++r) ptx::mbar_arrive(zeroed0 + 8 * r);
    uint32_t j = 0;  // input planes whose MMAs were waited for
    bool stop = false;
    for (int it = blockIdx.x; it < g.n_items && !stop; it += gridDim.x) {
      const ConvItem c = conv_item(g, it);
      const int y = c.y0 + 32 * warp + lane;
      const bool y_ok = y < g.y_hi && 32 * warp + lane < kCvTY;
      // outputs z0 - 2 .. z0 + planes + 1: after input plane z0 - 1 + i for i <= planes + 1
      for (int i = 0; i < c.planes + 4; ++i) {
        if (i < c.planes + 2) {
          if (!ptx::mbar_wait_bounded(mdone, j & 1, kConvTimeoutNs)) {
            *abort_flag = 1;
            stop = true;
            break;
          }
          ++j;
          tc5::fence_after();
        }
        const bool single = c.planes == 1;
        if (single && i != 2) continue;  // one-plane item: finalised once, after its last plane
        const int z = c.z0 - 2 + i;
        const int r = (z + 3) % 3;
        const uint32_t acc = lane_addr + 16 * r;
        const bool real = i >= 2 && i < c.planes + 2;
        // read the plane slot, zero it (all three for a one-plane item) and release it to the MMA
        // warp, then store
        uint32_t v[kCvTX][16];
        if (real) {
#pragma unroll
          for (int o = 0; o < kCvTX; ++o) tc5::ld16(acc + 48 * o, v[o]);
          tc5::wait_ld();
        }
        if (single) {
#pragma unroll
          for (int q = 0; q < 12; ++q) tc5::st16_zero(lane_addr + 16 * q);
        } else {
#pragma unroll
          for (int o = 0; o < kCvTX; ++o) tc5::st16_zero(acc + 48 * o);
        }
        tc5::wait_st();
        tc5::fence_before();
        __syncwarp();
        if (lane == 0) {
          if (single)
            for (int q = 0; q < 3; ++q) ptx::mbar_arrive(zeroed0 + 8 * q);
          else
            ptx::mbar_arrive(zeroed0 + 8 * r);
        }
        if (real) {
#pragma unroll
          for (int o = 0; o < kCvTX; ++o) {
            const int x = c.x0 + o;
            if (((c.mask >> o) & 1u) && x < g.nx && y_ok) {
              uint32_t h[8];
#pragma unroll
              for (int q = 0; q < 8; ++q) {
                const float v0 = fmaxf(__uint_as_float(v[o][2 * q]) + bias[2 * q], 0.f);
                const float v1 = fmaxf(__uint_as_float(v[o][2 * q + 1]) + bias[2 * q + 1], 0.f);
                const __nv_bfloat162 pr = __floats2bfloat162_rn(v0, v1);
                h[q] = *reinterpret_cast<const uint32_t *>(&pr);
              }
              const long long vx = ((long long)z * g.nx + x) * g.ny + y;
              *reinterpret_cast<uint4 *>(out + vx * 8) = make_uint4(h[0], h[1], h[2], h[3]);
              *reinterpret_cast<uint4 *>(out + (g.nvox + vx) * 8) =
                  make_uint4(h[4], h[5], h[6], h[7]);
            }
          }
        }
      }
    }
  }
  tc5::fence_before();
  __syncthreads();
  if (*abort_flag && threadIdx.x == 0) atomicExch(err, 3);
  if (warp == 0) {
    tc5::fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCvCols)
                 : "memory");
  }
}

// Variant for layers whose planes are needed in short runs (isolated anchor planes, or 3 around
// them): the accumulators of two consecutive output planes are double-buffered (64 columns
// each) instead of forming the three-plane ring, so an output plane costs 54 MMAs of N <= 48 (an
// input row at one y shift feeds up to 3 output rows of one plane through one MMA, weights stored
// per (kz, ky) as W(kx = 2) | W(kx = 1) | W(kx = 0)) but no output waits for another's epilogue;
// input planes stream through a 4-slot ring, so an item's three planes are all in flight; an item
// with one output row loads only the 3 input rows it needs (a second TMA map, half the bytes).
constexpr int kRwRing = 4;
constexpr int kRwSeq = 2 * 48 * 16;                     // one (kz, ky) weight sequence
constexpr int kRwWBytes = 9 * kRwSeq;                   // 13,824 B
constexpr int kRwCols = 2 * kCvTX * 16;                 // two accumulators
constexpr size_t kRwSmem = 128 + kRwRing * kCvPlane + kRwWBytes + 128;  // 2 CTAs per SM
constexpr int kRwFragWords = kRwWBytes / 4;

// conv16_rows_kernel weight sequences of one layer, byte offset ((kz * 3 + ky) * 2 + h) * 768 + n * 16 + 2 c8 holds
// W[co][8h + c8][kz * 9 + kx * 3 + ky] for n = 16 (2 - kx) + co.
__global__ void pack_rows_kernel(const __nv_bfloat16 *__restrict__ wbf, int woff,
                                  uint32_t *__restrict__ frag) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kRwFragWords) return;
  const int off = 4 * i;
  const int sq = off / kRwSeq, h = (off % kRwSeq) / 768, n = (off % 768) / 16, c8 = (off % 16) / 2;
  const int kz = sq / 3, ky = sq % 3, kx = 2 - n / 16, co = n % 16, ci = 8 * h + c8;
  const int t = kz * 9 + kx * 3 + ky;
  const __nv_bfloat16 lo = wbf[woff + (co * kC + ci) * 27 + t];
  const __nv_bfloat16 hi = wbf[woff + (co * kC + ci + 1) * 27 + t];
  frag[i] = (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

// The output region of one layer: work items {x tile | y tile << 16, first plane | planes << 16}

__global__ void __launch_bounds__(kCvThreads, 2)
    conv16_rows_kernel(const __grid_constant__ CUtensorMap tm, const __grid_constant__ CUtensorMap tm3,
                       const uint32_t *__restrict__ frag, const __nv_bfloat16 *__restrict__ wbf,
                       int boff, __nv_bfloat16 *__restrict__ out, ConvGrid g,
                       int *__restrict__ err) {
  extern __shared__ unsigned char smem_raw[];
  const uint32_t raw = ptx::smem_u32(smem_raw);
  const uint32_t base = (raw + 127u) & ~127u;
  const uint32_t wtab = base + kRwRing * kCvPlane;
  // barriers: full[kRwRing], empty[kRwRing], dfull[2], dempty[2]
  const uint32_t full0 = wtab + kRwWBytes, empty0 = full0 + 8 * kRwRing;
  const uint32_t dfull0 = empty0 + 8 * kRwRing, dempty0 = dfull0 + 16;
  unsigned char *gen = smem_raw + (dempty0 + 16 - raw);
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(gen);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(gen + 4);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

  // weight sequences into shared memory (visible to the tensor core through the async proxy)
  {
    uint32_t *w = reinterpret_cast<uint32_t *>(smem_raw + (wtab - raw));
    for (int i = threadIdx.x; i < kRwFragWords; i += kCvThreads) w[i] = __ldg(frag + i);
    ptx::fence_proxy_async_smem();
  }
  if (threadIdx.x == 0) {
    for (int i = 0; i < kRwRing; ++i) {
      ptx::mbar_init(full0 + 8 * i, 1);
      ptx::mbar_init(empty0 + 8 * i, 1);
    }
    for (int i = 0; i < 2; ++i) {
      ptx::mbar_init(dfull0 + 8 * i, 1);
      ptx::mbar_init(dempty0 + 8 * i, 4);
    }
    *abort_flag = 0;
    ptx::fence_mbarrier_init();
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     ptx::smem_u32(tmem_slot)),
                 "r"(kRwCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc5::fence_before();
  __syncthreads();
  tc5::fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 4) {
    // TMA producer: the input planes z0 - 1 .. z0 + planes of every item, in order, into the ring
    if (lane == 0) {
      uint32_t j = 0;  // planes issued
      for (int it = blockIdx.x; it < g.n_items && !*abort_flag; it += gridDim.x) {
        const ConvItem c = conv_item(g, it);
        for (int p = 0; p < c.planes + 2; ++p, ++j) {
          const uint32_t slot = j % kRwRing;
          if (j >= kRwRing &&
              !ptx::mbar_wait_bounded(empty0 + 8 * slot, ((j / kRwRing) - 1) & 1, kConvTimeoutNs)) {
            *abort_flag = 1;
            break;
          }
          // an item of one output row needs 3 input rows: the narrow box
          const bool narrow = c.mask == 1u;
          ptx::mbar_arrive_expect_tx(full0 + 8 * slot, narrow ? kCvPlane / 2 : kCvPlane);
          ptx::tma_load_4d(base + slot * kCvPlane, narrow ? &tm3 : &tm, full0 + 8 * slot,
                           2 * (c.y0 - 1), c.x0 - 1, c.z0 - 1 + p, 0);
        }
      }
      // planes still landing: wait for the last ring's worth (bounded)
      for (uint32_t q = j > kRwRing ? j - kRwRing : 0; q < j; ++q)
        if (!ptx::mbar_wait_bounded(full0 + 8 * (q % kRwRing), (q / kRwRing) & 1, kConvTimeoutNs))
          *abort_flag = 1;  // reported as a timeout
    }
  } else if (warp == 5) {
    // MMA issuer: the whole warp runs the loop, one elected lane issues
    {
      uint32_t j0 = 0, t = 0;  // first ring load of the item, output planes issued
      const uint64_t db0 = tc5::desc(wtab, 768, 128);
      for (int it = blockIdx.x; it < g.n_items && !*abort_flag; it += gridDim.x) {
        const ConvItem c = conv_item(g, it);
        for (int i = 0; i < c.planes; ++i, ++t) {
          const int b = t & 1;
          bool ok = ptx::mbar_wait_bounded(dempty0 + 8 * b, (t >> 1) & 1, kConvTimeoutNs);
          uint64_t da[3];
#pragma unroll
          for (int kz = 0; kz < 3; ++kz) {
            const uint32_t q = j0 + i + kz;
            ok = ok && ptx::mbar_wait_bounded(full0 + 8 * (q % kRwRing), (q / kRwRing) & 1,
                                               kConvTimeoutNs);
            da[kz] = tc5::desc(base + (q % kRwRing) * kCvPlane,
                               c.mask == 1u ? kCvHalf / 2 : kCvHalf, 128);
          }
          if (!ok) {
            *abort_flag = 1;
            break;
          }
          tc5::fence_after();
          const uint32_t dcol = tmem + b * (kCvTX * 16);
#pragma unroll 1
          for (int ix = 0; ix < kCvSX; ++ix) {
            // output rows fed by input row ix: o = ix - kx, kx = 2..0, within the item's mask
            int o_lo = ix - 2 < 0 ? 0 : ix - 2, o_hi = ix < kCvTX - 1 ? ix : kCvTX - 1;
            while (o_lo <= o_hi && !((c.mask >> o_lo) & 1u)) ++o_lo;
            while (o_hi >= o_lo && !((c.mask >> o_hi) & 1u)) --o_hi;
            if (o_lo > o_hi) continue;
            const uint32_t id = tc5::idesc_bf16(16 * (o_hi - o_lo + 1));
            const uint32_t d = dcol + 16 * o_lo;
            // descriptor start fields count 16-byte units
            const uint64_t db = db0 + (uint64_t)((o_lo - ix + 2) * 16);
#pragma unroll
            for (int sq = 0; sq < 9; ++sq) {
              const int kz = sq / 3, ky = sq % 3;
              tc5::mma(d, da[kz] + (uint64_t)(ix * kCvSY + ky), db + (uint64_t)(sq * kRwSeq / 16),
                       id);
            }
          }
          tc5::commit(dfull0 + 8 * b);
          // plane j0 + i feeds no later output of the item; the last output frees all three
          tc5::commit(empty0 + 8 * ((j0 + i) % kRwRing));
          if (i == c.planes - 1) {
            tc5::commit(empty0 + 8 * ((j0 + i + 1) % kRwRing));
            tc5::commit(empty0 + 8 * ((j0 + i + 2) % kRwRing));
          }
        }
        j0 += c.planes + 2;
      }
      // let every issued MMA finish before the accumulators are released (bounded)
      if (t > 0 &&
          !ptx::mbar_wait_bounded(dfull0 + 8 * ((t - 1) & 1), ((t - 1) >> 1) & 1, kConvTimeoutNs))
        *abort_flag = 1;  // reported as a timeout
    }
  } else {
    // epilogue: warp w reads TMEM lanes 32w..32w+31 = output y0 + 32w + lane
    const uint32_t lane_addr = tmem + ((uint32_t)(32 * warp) << 16);
    float bias[kC];
#pragma unroll
    for (int c = 0; c < kC; ++c) bias[c] = __bfloat162float(wbf[boff + c]);
    // both accumulators start at zero
#pragma unroll
    for (int q = 0; q < kRwCols / 16; ++q) tc5::st16_zero(lane_addr + 16 * q);
    tc5::wait_st();
    tc5::fence_before();
    __syncwarp();
    if (lane == 0) {
      ptx::mbar_arrive(dempty0);
      ptx::mbar_arrive(dempty0 + 8);
    }
    uint32_t t = 0;
    bool stop = false;
    for (int it = blockIdx.x; it < g.n_items && !stop; it += gridDim.x) {
      const ConvItem c = conv_item(g, it);
      const int y = c.y0 + 32 * warp + lane;
      const bool y_ok = y < g.y_hi && 32 * warp + lane < kCvTY;
      for (int i = 0; i < c.planes; ++i, ++t) {
        const int b = t & 1;
        if (!ptx::mbar_wait_bounded(dfull0 + 8 * b, (t >> 1) & 1, kConvTimeoutNs)) {
          *abort_flag = 1;
          stop = true;
          break;
        }
        tc5::fence_after();
        const int z = c.z0 + i;
        const uint32_t acc = lane_addr + b * (kCvTX * 16);
        uint32_t r[kCvTX][16];
#pragma unroll
        for (int o = 0; o < kCvTX; ++o) tc5::ld16(acc + 16 * o, r[o]);
        tc5::wait_ld();
#pragma unroll
        for (int o = 0; o < kCvTX; ++o) {
          const int x = c.x0 + o;
          if (((c.mask >> o) & 1u) && x < g.nx && y_ok) {
            uint32_t h[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
              const float v0 = fmaxf(__uint_as_float(r[o][2 * q]) + bias[2 * q], 0.f);
              const float v1 = fmaxf(__uint_as_float(r[o][2 * q + 1]) + bias[2 * q + 1], 0.f);
              const __nv_bfloat162 pr = __floats2bfloat162_rn(v0, v1);
              h[q] = *reinterpret_cast<const uint32_t *>(&pr);
            }
            const long long v = ((long long)z * g.nx + x) * g.ny + y;
            *reinterpret_cast<uint4 *>(out + v * 8) = make_uint4(h[0], h[1], h[2], h[3]);
            *reinterpret_cast<uint4 *>(out + (g.nvox + v) * 8) =
                make_uint4(h[4], h[5], h[6], h[7]);
          }
        }
#pragma unroll
        for (int o = 0; o < kCvTX; ++o) tc5::st16_zero(acc + 16 * o);
        tc5::wait_st();
        tc5::fence_before();
        __syncwarp();
        if (lane == 0) ptx::mbar_arrive(dempty0 + 8 * b);
      }
    }
  }
  tc5::fence_before();
  __syncthreads();
  if (*abort_flag && threadIdx.x == 0) atomicExch(err, 3);
  if (warp == 0) {
    tc5::fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kRwCols)
                 : "memory");
  }
}

// ---------------------------------------------------------------- conv 2 -> 16 (tcgen05)

// conv1 on tcgen05, as a 3 x 3 (z, x) convolution over 16 "channels" per voxel: for input MRI
// and atlas MRI c, the raw intensities at y - 1, y, y + 1 (FP16) and five zeros, so the y taps
// are folded into K and both input channels fill one K = 16 MMA. Items, the TMEM ring of three
// output-plane accumulators, the weight-sequence rotations and the warp roles follow
// conv16_kernel, except that the producer warps build each input plane's operand slot in shared
// memory from the FP32 volumes (the y expansion has no TMA form) and that an item column covers
// 128 y: 6 MMAs (N = 48 x rows fed) per input plane. The epilogue applies the network's input
// scale 1/512 to the FP32 sums (the layer is linear before its bias), the bias and ReLU.
constexpr int kC1Y = 128;                    // output y per item column (M = 128, all stored)
constexpr int kC1Seq = 2 * kCvSeqRows * 16;  // one rotation: 144 rows x 16 FP16 channels
constexpr int kC1WBytes = 3 * kC1Seq;        // 13,824 B
constexpr int kC1Ring = 3;
constexpr int kC1Threads = 288;  // warps 0-3 epilogue, 4 MMA, 5-8 producers
constexpr size_t kC1Smem = 128 + kC1Ring * kCvPlane + kC1WBytes + 128;  // 2 CTAs per SM
constexpr int kC1FragWords = kC1WBytes / 4;

// conv1 weight sequences: rotation rho, byte offset rho * 4608 + h * 2304 + n * 16 + 2 c holds
// (c < 3) W1[co][h][kz * 9 + kx * 3 + c] as FP16 (c = y tap, h = input channel) for row
// n = 16 (3 kxi + r) + co, kx = 2 - kxi, kz = (rho - r) mod 3.
__global__ void pack_c1_kernel(const __nv_bfloat16 *__restrict__ wbf, uint32_t *__restrict__ frag) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kC1FragWords) return;
  const int off = 4 * i;
  const int rho = off / kC1Seq, h = (off % kC1Seq) / (kCvSeqRows * 16);
  const int n = (off % (kCvSeqRows * 16)) / 16, c = (off % 16) / 2;
  const int blk = n / 16, co = n % 16;
  const int kx = 2 - blk / 3, r = blk % 3, kz = (rho - r + 3) % 3;
  const int wb = kW1 + (co * kCin + h) * 27 + kz * 9 + kx * 3;
  const float w0 = c < 3 ? __bfloat162float(wbf[wb + c]) : 0.f;
  const float w1 = c + 1 < 3 ? __bfloat162float(wbf[wb + c + 1]) : 0.f;
  const __half2 hw = __floats2half2_rn(w0, w1);
  frag[i] = *reinterpret_cast<const uint32_t *>(&hw);
}

__device__ __forceinline__ uint32_t idesc_f16(int n) {
  // D FP32, A and B FP16 (K-major), N, M = 128
  return (1u << 4) | ((uint32_t)(n >> 3) << 17) | ((128u >> 4) << 24);
}

__global__ void __launch_bounds__(kC1Threads, 2)
    conv1_tc_kernel(const float *__restrict__ img, const float *__restrict__ atl, int apitch,
                    const uint32_t *__restrict__ frag, const __nv_bfloat16 *__restrict__ wbf,
                    __nv_bfloat16 *__restrict__ out, ConvGrid g, int *__restrict__ err) {
  extern __shared__ unsigned char smem_raw[];
  const uint32_t raw = ptx::smem_u32(smem_raw);
  const uint32_t base = (raw + 127u) & ~127u;
  const uint32_t wtab = base + kC1Ring * kCvPlane;
  // barriers: full[ring] (4 producer warps), empty[ring], mdone, zeroed[3]
  const uint32_t full0 = wtab + kC1WBytes, empty0 = full0 + 8 * kC1Ring;
  const uint32_t mdone = empty0 + 8 * kC1Ring, zeroed0 = mdone + 8;
  unsigned char *gen = smem_raw + (zeroed0 + 24 - raw);
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(gen);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(gen + 4);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

  {
    uint32_t *w = reinterpret_cast<uint32_t *>(smem_raw + (wtab - raw));
    for (int i = threadIdx.x; i < kC1FragWords; i += kC1Threads) w[i] = __ldg(frag + i);
    ptx::fence_proxy_async_smem();
  }
  if (threadIdx.x == 0) {
    for (int i = 0; i < kC1Ring; ++i) {
      ptx::mbar_init(full0 + 8 * i, 4);
      ptx::mbar_init(empty0 + 8 * i, 1);
    }
    ptx::mbar_init(mdone, 1);
    for (int i = 0; i < 3; ++i) ptx::mbar_init(zeroed0 + 8 * i, 4);
    *abort_flag = 0;
    ptx::fence_mbarrier_init();
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     ptx::smem_u32(tmem_slot)),
                 "r"(kCvCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc5::fence_before();
  __syncthreads();
  tc5::fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp >= 5) {
    // producers: thread tp builds the operand rows of y = y0 + tp for the 6 x-rows of a plane
    const int tp = threadIdx.x - 160;
    unsigned char *slots = smem_raw + (base - raw);
    uint32_t j = 0;
    bool stop = false;
    for (int it = blockIdx.x; it < g.n_items && !stop && !*abort_flag; it += gridDim.x) {
      const ConvItem c = conv_item(g, it);
      const int y = c.y0 + tp;
      for (int p = 0; p < c.planes + 2; ++p, ++j) {
        const uint32_t slot = j % kC1Ring;
        if (j >= kC1Ring &&
            !ptx::mbar_wait_bounded(empty0 + 8 * slot, ((j / kC1Ring) - 1) & 1, kConvTimeoutNs)) {
          *abort_flag = 1;
          stop = true;
          break;
        }
        const int z = c.z0 - 1 + p;
        unsigned char *dst = slots + slot * kCvPlane + tp * 16;
        // each lane loads its own y of the 6 rows of both volumes (all loads in flight at once);
        // y - 1 and y + 1 come from the neighbouring lanes, the warp's edge lanes load theirs
        const bool zin_ok = z >= 0 && z < g.nz;
        const int ye = lane == 0 ? y - 1 : y + 1;  // the edge neighbour this lane may need
        float ci[kCvSX], ca[kCvSX], ei[kCvSX], ea[kCvSX];
#pragma unroll
        for (int xr = 0; xr < kCvSX; ++xr) {
          const int x = c.x0 - 1 + xr;
          const bool row_ok = zin_ok && x >= 0 && x < g.nx;
          const long long ro = (long long)z * g.nx + x;
          ci[xr] = ca[xr] = ei[xr] = ea[xr] = 0.f;
          if (row_ok && y < g.ny) {
            ci[xr] = __ldg(img + ro * g.ny + y);
            ca[xr] = __ldg(atl + ro * apitch + y);
          }
          if (row_ok && (lane == 0 || lane == 31) && ye >= 0 && ye < g.ny) {
            ei[xr] = __ldg(img + ro * g.ny + ye);
            ea[xr] = __ldg(atl + ro * apitch + ye);
          }
        }
#pragma unroll
        for (int xr = 0; xr < kCvSX; ++xr) {
          float im = __shfl_up_sync(0xffffffffu, ci[xr], 1), ip = __shfl_down_sync(0xffffffffu, ci[xr], 1);
          float am = __shfl_up_sync(0xffffffffu, ca[xr], 1), ap = __shfl_down_sync(0xffffffffu, ca[xr], 1);
          if (lane == 0) {
            im = ei[xr];
            am = ea[xr];
          }
          if (lane == 31) {
            ip = ei[xr];
            ap = ea[xr];
          }
          const __half2 i01 = __floats2half2_rn(im, ci[xr]), a01 = __floats2half2_rn(am, ca[xr]);
          const __half2 i2 = __floats2half2_rn(ip, 0.f), a2 = __floats2half2_rn(ap, 0.f);
          *reinterpret_cast<uint4 *>(dst + xr * kCvSY * 16) =
              make_uint4(*reinterpret_cast<const uint32_t *>(&i01),
                         *reinterpret_cast<const uint32_t *>(&i2), 0u, 0u);
          *reinterpret_cast<uint4 *>(dst + kCvHalf + xr * kCvSY * 16) =
              make_uint4(*reinterpret_cast<const uint32_t *>(&a01),
                         *reinterpret_cast<const uint32_t *>(&a2), 0u, 0u);
        }
        ptx::fence_proxy_async_smem();  // the tensor core reads the slot through the async proxy
        __syncwarp();
        if (lane == 0) ptx::mbar_arrive(full0 + 8 * slot);
      }
    }
  } else if (warp == 4) {
    // MMA issuer: the whole warp runs the loop, one elected lane issues
    uint32_t j = 0;
    uint32_t nz[3] = {1, 1, 1};
    const uint64_t db0 = tc5::desc(wtab, kCvSeqRows * 16, 128);
    for (int it = blockIdx.x; it < g.n_items && !*abort_flag; it += gridDim.x) {
      const ConvItem c = conv_item(g, it);
      bool ok = true;
      for (int p = 0; p < c.planes + 2 && ok; ++p, ++j) {
        const int zin = c.z0 - 1 + p;
        for (int r = 0; r < 3 && ok; ++r)
          if (p == 0 || (c.planes > 1 && r == (zin + 1 + 3) % 3))
            ok = ptx::mbar_wait_bounded(zeroed0 + 8 * r, (nz[r] - 1) & 1, kConvTimeoutNs);
        ok = ok && ptx::mbar_wait_bounded(full0 + 8 * (j % kC1Ring), (j / kC1Ring) & 1,
                                          kConvTimeoutNs);
        if (!ok) {
          *abort_flag = 1;
          break;
        }
        tc5::fence_after();
        const uint64_t da = tc5::desc(base + (j % kC1Ring) * kCvPlane, kCvHalf, 128);
        const int rho = (zin + 1 + 3) % 3;
#pragma unroll 1
        for (int ix = 0; ix < kCvSX; ++ix) {
          int o_lo = ix - 2 < 0 ? 0 : ix - 2, o_hi = ix < kCvTX - 1 ? ix : kCvTX - 1;
          while (o_lo <= o_hi && !((c.mask >> o_lo) & 1u)) ++o_lo;
          while (o_hi >= o_lo && !((c.mask >> o_hi) & 1u)) --o_hi;
          if (o_lo > o_hi) continue;
          tc5::mma(tmem + 48 * o_lo, da + (uint64_t)(ix * kCvSY),
                   db0 + (uint64_t)(rho * (kC1Seq / 16) + 3 * (2 - ix + o_lo) * 16),
                   idesc_f16(48 * (o_hi - o_lo + 1)));
        }
        tc5::commit(empty0 + 8 * (j % kC1Ring));
        tc5::commit(mdone);
        if (c.planes > 1 || p == c.planes + 1) nz[(zin - 1 + 3) % 3] += 1;
        if (p == c.planes + 1) {
          nz[(zin + 3) % 3] += 1;
          nz[(zin + 1 + 3) % 3] += 1;
        }
      }
    }
    if (j > 0 && !ptx::mbar_wait_bounded(mdone, (j - 1) & 1, kConvTimeoutNs))
      *abort_flag = 1;  // reported as a timeout
  } else {
    // epilogue: warp w reads TMEM lanes 32w..32w+31 = output y0 + 32w + lane
    const uint32_t lane_addr = tmem + ((uint32_t)(32 * warp) << 16);
    float bias[kC];
#pragma unroll
    for (int q = 0; q < kC; ++q) bias[q] = __bfloat162float(wbf[kB1 + q]);
#pragma unroll
    for (int q = 0; q < 12; ++q) tc5::st16_zero(lane_addr + 16 * q);
    tc5::wait_st();
    tc5::fence_before();
    __syncwarp();
    if (lane == 0)
      for (int r = 0; r < 3; ++r) ptx::mbar_arrive(zeroed0 + 8 * r);
    uint32_t j = 0;
    bool stop = false;
    for (int it = blockIdx.x; it < g.n_items && !stop; it += gridDim.x) {
      const ConvItem c = conv_item(g, it);
      const int y = c.y0 + 32 * warp + lane;
      const bool y_ok = y < g.y_hi;
      for (int i = 0; i < c.planes + 4; ++i) {
        if (i < c.planes + 2) {
          if (!ptx::mbar_wait_bounded(mdone, j & 1, kConvTimeoutNs)) {
            *abort_flag = 1;
            stop = true;
            break;
          }
          ++j;
          tc5::fence_after();
        }
        const bool single = c.planes == 1;
        if (single && i != 2) continue;
        const int z = c.z0 - 2 + i;
        const int r = (z + 3) % 3;
        const uint32_t acc = lane_addr + 16 * r;
        const bool real = i >= 2 && i < c.planes + 2;
        uint32_t v[kCvTX][16];
        if (real) {
#pragma unroll
          for (int o = 0; o < kCvTX; ++o) tc5::ld16(acc + 48 * o, v[o]);
          tc5::wait_ld();
        }
        if (single) {
#pragma unroll
          for (int q = 0; q < 12; ++q) tc5::st16_zero(lane_addr + 16 * q);
        } else {
#pragma unroll
          for (int o = 0; o < kCvTX; ++o) tc5::st16_zero(acc + 48 * o);
        }
        tc5::wait_st();
        tc5::fence_before();
        __syncwarp();
        if (lane == 0) {
          if (single)
            for (int q = 0; q < 3; ++q) ptx::mbar_arrive(zeroed0 + 8 * q);
          else
            ptx::mbar_arrive(zeroed0 + 8 * r);
        }
        if (real) {
#pragma unroll
          for (int o = 0; o < kCvTX; ++o) {
            const int x = c.x0 + o;
            if (((c.mask >> o) & 1u) && x < g.nx && y_ok) {
              uint32_t h[8];
#pragma unroll
              for (int q = 0; q < 8; ++q) {
                const float v0 = fmaxf(fmaf(__uint_as_float(v[o][2 * q]), kInScale, bias[2 * q]), 0.f);
                const float v1 =
                    fmaxf(fmaf(__uint_as_float(v[o][2 * q + 1]), kInScale, bias[2 * q + 1]), 0.f);
                const __nv_bfloat162 pr = __floats2bfloat162_rn(v0, v1);
                h[q] = *reinterpret_cast<const uint32_t *>(&pr);
              }
              const long long vx = ((long long)z * g.nx + x) * g.ny + y;
              *reinterpret_cast<uint4 *>(out + vx * 8) = make_uint4(h[0], h[1], h[2], h[3]);
              *reinterpret_cast<uint4 *>(out + (g.nvox + vx) * 8) =
                  make_uint4(h[4], h[5], h[6], h[7]);
            }
          }
        }
      }
    }
  }
  tc5::fence_before();
  __syncthreads();
  if (*abort_flag && threadIdx.x == 0) atomicExch(err, 3);
  if (warp == 0) {
    tc5::fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCvCols)
                 : "memory");
  }
}

// ---------------------------------------------------------------- proposal + rescoring

// Head weights staged in shared memory by every kernel that proposes, transposed and padded for
// packed FP32 FMAs: [16 channels][34 outputs] (output 33 is a zero pad), then 34 biases.
constexpr int kHeadPad = kHeads + 1;
constexpr int kHeadFloats = kC * kHeadPad + kHeadPad;

__device__ __forceinline__ void stage_heads(const __nv_bfloat16 *__restrict__ wbf, float *hwt) {
  for (int i = threadIdx.x; i < kHeadFloats; i += blockDim.x) {
    float v = 0.f;
    if (i < kC * kHeadPad) {
      const int c = i / kHeadPad, o = i % kHeadPad;
      if (o < kHeads) v = __bfloat162float(wbf[kH + o * kC + c]);
    } else if (i - kC * kHeadPad < kHeads) {
      v = __bfloat162float(wbf[kHB + i - kC * kHeadPad]);
    }
    hwt[i] = v;
  }
}

// Per-axis offset probabilities of one (voxel, atlas) pair from its 16 conv4 features: the three
// softmaxes over dw, du, dv of the heads' logits, p[a * 11 + j] for offset j - 5 on axis a. For a
// window NH = 2 half + 1 below 11 each softmax runs over the window's offsets only
// (|j - 5| <= half) and the others get probability 0; at NH = 11 every offset takes part.
__device__ __forceinline__ bool in_window(int j, int half) { return (unsigned)(j - 5 + half) <= 2u * half; }

__device__ __forceinline__ void axis_probs(const __nv_bfloat16 *__restrict__ f4, long long v,
                                           long long nvox, const float *__restrict__ hw,
                                           float (&p)[kHeads], int half) {
  float f[kC];
  {
    __align__(16) __nv_bfloat16 fb[kC];
    reinterpret_cast<uint4 *>(fb)[0] = *reinterpret_cast<const uint4 *>(f4 + v * 8);
    reinterpret_cast<uint4 *>(fb)[1] = *reinterpret_cast<const uint4 *>(f4 + (nvox + v) * 8);
#pragma unroll
    for (int c = 0; c < kC; ++c) f[c] = __bfloat162float(fb[c]);
  }
  // logits: for each pair of outputs one packed FMA per channel, in channel order
  float2 acc[kHeadPad / 2];
#pragma unroll
  for (int o2 = 0; o2 < kHeadPad / 2; ++o2)
    acc[o2] = *reinterpret_cast<const float2 *>(hw + kC * kHeadPad + 2 * o2);
#pragma unroll
  for (int c = 0; c < kC; ++c) {
    const float2 fc = make_float2(f[c], f[c]);
#pragma unroll
    for (int o2 = 0; o2 < kHeadPad / 2; ++o2)
      acc[o2] = __ffma2_rn(*reinterpret_cast<const float2 *>(hw + c * kHeadPad + 2 * o2), fc,
                           acc[o2]);
  }
#pragma unroll
  for (int o = 0; o < kHeads; ++o) p[o] = (o & 1) ? acc[o / 2].y : acc[o / 2].x;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    float m = -INFINITY;
#pragma unroll
    for (int j = 0; j < kAxis; ++j)
      if (in_window(j, half)) m = fmaxf(m, p[a * kAxis + j]);
    float sum = 0.f;
#pragma unroll
    for (int j = 0; j < kAxis; ++j) {
      p[a * kAxis + j] = in_window(j, half) ? __expf(p[a * kAxis + j] - m) : 0.f;
      sum += p[a * kAxis + j];
    }
    const float inv = 1.f / sum;
#pragma unroll
    for (int j = 0; j < kAxis; ++j) p[a * kAxis + j] *= inv;
  }
}

// The 4 largest of p[a * 11 .. a * 11 + 10] within the window in order, ties to the lower
// offset: indices 0..10.
__device__ __forceinline__ void top4(const float (&p)[kHeads], int a, int (&idx)[4], int half) {
  unsigned used = 0;
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    int bi = 5;
    float bp = -1.f;
#pragma unroll
    for (int j = 0; j < kAxis; ++j)
      if (in_window(j, half) && !((used >> j) & 1u) && p[a * kAxis + j] > bp) {
        bp = p[a * kAxis + j];
        bi = j;
      }
    used |= 1u << bi;
    idx[r] = bi;
  }
}

// p[a * 11 + idx] for a run-time idx, without local memory.
__device__ __forceinline__ float pick(const float (&p)[kHeads], int a, int idx) {
  float v = 0.f;
#pragma unroll
  for (int j = 0; j < kAxis; ++j) v = (j == idx) ? p[a * kAxis + j] : v;
  return v;
}

// Probability mass p_w * p_u * p_v of the kept set, the rank triples (i, j, k) with
// i + j + k <= level (2, 3 or 4), from the per-axis probabilities of ranks 0..3, tp[a][r].
__device__ __forceinline__ float mass_of(const float (&tp)[3][4], int level) {
  float t[5];
#pragma unroll
  for (int s2 = 0; s2 <= 4; ++s2) {
    float acc = 0.f;
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int k = 0; k < 4; ++k)
        if (j + k <= s2) acc = fmaf(tp[1][j], tp[2][k], acc);
    t[s2] = acc;
  }
  float m = 0.f;
#pragma unroll
  for (int i = 0; i < 4; ++i)
    if (i <= level) m += tp[0][i] * (level - i == 4 ? t[4] : level - i == 3 ? t[3]
                                     : level - i == 2 ? t[2] : level - i == 1 ? t[1] : t[0]);
  return m;
}

// The same mass from a voxel's own probabilities and per-axis lists top[a][0..3].
__device__ __forceinline__ float kept_mass(const float (&p)[kHeads], const int (&top)[3][4]) {
  float tp[3][4];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int r = 0; r < 4; ++r) tp[a][r] = pick(p, a, top[a][r]);
  return mass_of(tp, 4);
}

// The proposal of one voxel on its own (the testing hook reports it): its 4 most probable
// offsets per axis (as -5..5) and the mass of its kept set.
struct Proposal {
  signed char top[3][4];
  float conf;
};

__device__ __forceinline__ void propose(const __nv_bfloat16 *__restrict__ f4, long long v,
                                        long long nvox, const float *__restrict__ hw,
                                        Proposal &pr, int half) {
  float p[kHeads];
  axis_probs(f4, v, nvox, hw, p, half);
  int top[3][4];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    top4(p, a, top[a], half);
#pragma unroll
    for (int r = 0; r < 4; ++r) pr.top[a][r] = (signed char)(top[a][r] - 5);
  }
  pr.conf = kept_mass(p, top);
}

// Testing hook: the proposal of given voxels.
__global__ void proposal_hook_kernel(const __nv_bfloat16 *__restrict__ f4,
                                     const __nv_bfloat16 *__restrict__ wbf,
                                     const int64_t *__restrict__ voxels, int n, long long nvox,
                                     signed char *__restrict__ top, float *__restrict__ conf,
                                     int half) {
  __shared__ __align__(16) float hw[kHeadFloats];
  stage_heads(wbf, hw);
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  Proposal pr;
  propose(f4, voxels[i], nvox, hw, pr, half);
  for (int a = 0; a < 3; ++a)
    for (int r = 0; r < 4; ++r) top[i * 12 + a * 4 + r] = pr.top[a][r];
  conf[i] = pr.conf;
}

// Rescoring device code (RowProp, the kept rank triples, the tap evaluation and both rescoring
// kernels' bodies); the same text is compiled again per geometry at run time.
#include "pct_rescore.cuh"
static_assert(kRsAxis == kAxis && kRsTopK == kTopK, "rescoring constants follow the network's");

constexpr int kProbStride = kHeads;  // 33 floats per lane row: column reads are conflict-free

__device__ __forceinline__ int anchor_of(int b, int block, int extent) {
  const int a = b * block + block / 2;
  return a < extent ? a : extent - 1;
}

// HALF: the window's half width (5, 4, 3), a template so that NH = 11 compiles without the
// window tests.
template <int HALF>
__global__ void __launch_bounds__(kRescoreWarps * 32)
    propose_rows_kernel(const __nv_bfloat16 *__restrict__ f4, const __nv_bfloat16 *__restrict__ wbf,
                        int nx, int ny, int nz, int block, int level,
                        RowProp *__restrict__ props) {
  constexpr int half = HALF;
  __shared__ __align__(16) float hw[kHeadFloats];
  __shared__ float s_prob[kRescoreWarps * 32 * kProbStride];
  __shared__ float s_sum[kRescoreWarps * 36];
  __shared__ int s_top[kRescoreWarps * 12];
  stage_heads(wbf, hw);
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int lo = half + 1;
  const int ix = nx - 2 * lo, iz = nz - 2 * lo, iy = ny - 2 * lo;
  if (ix <= 0 || iy <= 0 || iz <= 0) return;
  const int segs = (iy + kRowOut - 1) / kRowOut;
  const int nbx = (ix + block - 1) / block, nbz = (iz + block - 1) / block;
  const long long items = (long long)nbz * nbx * segs;
  const int nxy = nx * ny;
  for (long long it = (long long)blockIdx.x * kRescoreWarps + (threadIdx.x >> 5); it < items;
       it += (long long)gridDim.x * kRescoreWarps) {
    const int seg = (int)(it % segs);
    const long long r0 = it / segs;
    const int bx = (int)(r0 % nbx), bz = (int)(r0 / nbx);
    const int x = lo + anchor_of(bx, block, ix), z = lo + anchor_of(bz, block, iz);
    const int y = lo + seg * kRowOut - 1 + lane;
    const bool out_lane = lane >= 1 && lane <= kRowOut && y < ny - lo;
    float p[kHeads];
    if (out_lane) {
      axis_probs(f4, (long long)z * nxy + (long long)x * ny + y, (long long)nz * nxy, hw, p, half);
    } else {
#pragma unroll
      for (int o = 0; o < kHeads; ++o) p[o] = 0.f;
    }
    // row sums through shared memory: lane l sums column l (and column 32) of the segment's
    // probabilities; lanes 0..2 pick the top 4 of axis 0..2
    float *wp = s_prob + (threadIdx.x >> 5) * 32 * kProbStride;
    float *wsum = s_sum + (threadIdx.x >> 5) * 36;
    int *wtop = s_top + (threadIdx.x >> 5) * 12;
#pragma unroll
    for (int o = 0; o < kHeads; ++o) wp[lane * kProbStride + o] = p[o];
    __syncwarp();
    {
      float c0 = 0.f, c1 = 0.f;
#pragma unroll 8
      for (int r = 0; r < 32; ++r) {
        c0 += wp[r * kProbStride + lane];
        c1 += wp[r * kProbStride + 32];
      }
      wsum[lane] = c0;
      if (lane == 0) wsum[32] = c1;
    }
    __syncwarp();
    if (lane < 3) {
      float q[kAxis];
#pragma unroll
      for (int j = 0; j < kAxis; ++j) q[j] = wsum[lane * kAxis + j];
      unsigned used = 0;
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        int bi = 5;
        float bp = -1.f;
#pragma unroll
        for (int j = 0; j < kAxis; ++j)
          if (in_window(j, half) && !((used >> j) & 1u) && q[j] > bp) {
            bp = q[j];
            bi = j;
          }
        used |= 1u << bi;
        wtop[lane * 4 + r] = bi;
      }
    }
    __syncwarp();
    RowProp &rp = props[r0 * segs + seg];
    if (lane < 12) rp.top[lane] = (signed char)wtop[lane];
    if (out_lane) {
      float tp[3][4];
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int r = 0; r < 4; ++r) tp[a][r] = wp[lane * kProbStride + a * kAxis + wtop[a * 4 + r]];
      rp.conf[lane - 1] = mass_of(tp, level);
    } else if (lane >= 1 && lane <= kRowOut) {
      rp.conf[lane - 1] = 0.f;
    }
    __syncwarp();  // the warp's shared rows are rewritten by its next segment
  }
}

// Exact FP32 rescoring of one atlas. A warp owns a row segment (z, x, y0 .. y0+29) of interior
// voxels; lane l sits at y = y0 - 1 + l (lanes 0 and 31 are the y halo). Every voxel of the
// segment computes its per-axis probabilities; their sums over the segment give the row's
// proposal: per axis the 4 most probable offsets, and the rank triples with i + j + k <= level.
// A voxel whose own probability mass on those is below conf_thr falls back to all 11^3
// offsets. Each offset is evaluated once for all 32 lanes: D(y) = sum over the 3x3 (dz, dx) taps
// of the squared differences at y, then SSD(y) = D(y-1) + D(y) + D(y+1) by warp shuffles; a lane
// adds the weight exp(-SSD/div) and the weighted CT value for the offsets it keeps.
__device__ __forceinline__ void eval_offset(const float *__restrict__ atl,
                                            const float *__restrict__ lab, const float (&in)[9],
                                            long long vz, long long axy, int apitch, int yc,
                                            int dw, int du, int dv, bool take, float &P,
                                            float &W, float neg_k) {
  const float *a = atl + vz + (long long)(dw - 1) * axy + (long long)(du - 1) * apitch + yc + dv;
  float d = 0.f;
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    const float t = in[k] - __ldg(a + (long long)(k / 3) * axy + (long long)(k % 3) * apitch);
    d = fmaf(t, t, d);
  }
  const float ssd =
      __shfl_up_sync(0xffffffffu, d, 1) + d + __shfl_down_sync(0xffffffffu, d, 1);
  if (take) {
    const float w = ptx::ex2_approx(ssd * neg_k);
    P = fmaf(w, __ldg(lab + vz + (long long)dw * axy + (long long)du * apitch + yc + dv), P);
    W += w;
  }
}

__global__ void __launch_bounds__(kRescoreWarps * 32, 3)
    rescore_kernel(const RowProp *__restrict__ props, int block, int level,
                   const float *__restrict__ img,
                   const float *__restrict__ atl, const float *__restrict__ lab, int nx, int ny,
                   int nz, int apitch, float neg_k, float conf_thr, float *__restrict__ pacc,
                   float *__restrict__ wacc, unsigned long long *__restrict__ fallbacks,
                   unsigned long long *__restrict__ evaluated, int half) {
  const int lane = threadIdx.x & 31;
  const int lo = half + 1;
  const int ix = nx - 2 * lo, iz = nz - 2 * lo, iy = ny - 2 * lo;
  if (ix <= 0 || iy <= 0 || iz <= 0) return;
  const int segs = (iy + kRowOut - 1) / kRowOut;
  const int nbx = (ix + block - 1) / block;
  const long long items = (long long)iz * ix * segs;
  const int nxy = nx * ny;
  const long long axy = (long long)nx * apitch;
  unsigned long long my_fallbacks = 0, my_evals = 0;
  for (long long it = (long long)blockIdx.x * kRescoreWarps + (threadIdx.x >> 5); it < items;
       it += (long long)gridDim.x * kRescoreWarps) {
    const int seg = (int)(it % segs);
    const long long r0 = it / segs;
    const int x = (int)(r0 % ix) + lo, z = (int)(r0 / ix) + lo;
    const int y0 = lo + seg * kRowOut;
    const int y = y0 - 1 + lane;
    const bool out_lane = lane >= 1 && lane <= kRowOut && y < ny - lo;
    const int yc = min(y, ny - lo);  // halo lanes past the interior load clamped (unused) values
    // the proposal of this row's block (its anchor row's 4 offsets per axis) and this voxel's
    // confidence, measured on the anchor row's voxel at the same y
    const RowProp &rp = props[(((long long)((z - lo) / block) * nbx) + (x - lo) / block) * segs + seg];
    int top[3][4];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int r = 0; r < 4; ++r) top[a][r] = rp.top[a * 4 + r];
    const bool full = out_lane && conf_thr > 0.f && rp.conf[lane - 1] < conf_thr;
    const unsigned any_full = __ballot_sync(0xffffffffu, full);
    if (full) ++my_fallbacks;
    // input taps of this lane: I(z+dz, x+dx, y), 3x3 (dz, dx)
    float in[9];
#pragma unroll
    for (int k = 0; k < 9; ++k)
      in[k] = __ldg(img + (long long)(z + k / 3 - 1) * nxy + (long long)(x + k % 3 - 1) * ny + yc);
    const long long vz = (long long)(z - 1) * axy + (long long)(x - 1) * apitch;  // (dz,dx)=(-1,-1)
    float P = 0.f, W = 0.f;
    if (!any_full) {
      // the kept offsets, in rank-triple order
      int kept = 0;
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j + i < 5 && j < 4; ++j)
#pragma unroll
          for (int k = 0; k + j + i < 5 && k < 4; ++k)
            if (i + j + k <= level) {
              eval_offset(atl, lab, in, vz + axy + apitch, axy, apitch, yc, top[0][i] - 5,
                          top[1][j] - 5, top[2][k] - 5, out_lane, P, W, neg_k);
              ++kept;
            }
      my_evals += kept;
    } else {
      // the full window; lanes that did not fall back keep only their row's kept set
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
      for (int jw = 5 - half; jw <= 5 + half; ++jw) {
        const int rw = (int)((rank[0] >> (4 * jw)) & 0xF);
        for (int ju = 5 - half; ju <= 5 + half; ++ju) {
          const int ru = rw + (int)((rank[1] >> (4 * ju)) & 0xF);
          for (int jv = 5 - half; jv <= 5 + half; ++jv) {
            const bool mine = full || (ru + (int)((rank[2] >> (4 * jv)) & 0xF) <= level);
            eval_offset(atl, lab, in, vz + axy + apitch, axy, apitch, yc, jw - 5, ju - 5, jv - 5,
                        mine && out_lane, P, W, neg_k);
          }
        }
      }
      my_evals += (unsigned long long)(2 * half + 1) * (2 * half + 1) * (2 * half + 1);
    }
    if (out_lane) {
      const long long v = (long long)z * nxy + (long long)x * ny + y;
      pacc[v] += P;
      wacc[v] += W;
    }
  }
  if (my_fallbacks) atomicAdd(fallbacks, my_fallbacks);
  if (lane == 0 && my_evals) atomicAdd(evaluated, my_evals);
}

// Proposal rescoring, library build (run-time strides); launch_rescore4 prefers the per-geometry
// run-time compiled module of the same code.
template <int LEVEL>
__global__ void __launch_bounds__(kRescoreWarps * 32, 4)
    rescore4_kernel(const RowProp *__restrict__ props, const float *__restrict__ img,
                    const float *__restrict__ atl, const float *__restrict__ lab, int nx, int ny,
                    int nz, int apitch, float scale, float conf_thr, float *__restrict__ pacc,
                    float *__restrict__ wacc, unsigned long long *__restrict__ fallbacks,
                    unsigned long long *__restrict__ evaluated,
                    const unsigned char *__restrict__ tile_flag, const RescoreTiles ts, int hw) {
  rescore4_body<LEVEL>(props, img, atl, lab, nx, ny, nz, apitch, scale, conf_thr, pacc, wacc,
                       fallbacks, evaluated, tile_flag, ts, hw);
}

// The confidence fallback at the plain kernel's tile granularity (blocks of 4 x 4 rows share a
// proposal and its per-voxel confidences): a tile falls back for this atlas when any of its
// interior voxels has a confidence below the threshold. The rescoring skips flagged tiles; bit
// `bit` of the tile's mask records the atlas for the plain kernel's full search, which runs once
// for a block of up to 32 atlases. Counts the fallback (voxel, atlas) pairs and the offsets
// evaluated by their rows.
__global__ void flag_tiles_kernel(const RowProp *__restrict__ props, int nx, int ny, int nz,
                                  float conf_thr, const TileShape ts,
                                  unsigned char *__restrict__ flag, uint32_t *__restrict__ masks,
                                  int bit, unsigned long long *__restrict__ fallbacks,
                                  unsigned long long *__restrict__ evaluated) {
  const int lo = 6;  // NH = 11 only: the plain kernel's tiles of that window
  const int ix = nx - 2 * lo, iy = ny - 2 * lo, iz = nz - 2 * lo;
  const int nbx = (ix + kRows - 1) / kRows, segs = (iy + kRowOut - 1) / kRowOut;
  const int ntiles = ts.tiles_y * ts.tiles_x * ts.tiles_z;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntiles; t += gridDim.x * blockDim.x) {
    const int ty = t % ts.tiles_y, r = t / ts.tiles_y;
    const int tx = r % ts.tiles_x, tz = r / ts.tiles_x;
    const int x0 = tx * ts.xc, x1 = min(x0 + ts.xc, ix);  // interior-relative
    const int z0 = tz * ts.zt, z1 = min(z0 + ts.zt, iz);
    const int nyv = min(kRowOut, iy - ty * kRowOut);
    bool any = false;
    for (int zb = z0 / kRows; zb <= (z1 - 1) / kRows && !any; ++zb)
      for (int bx = x0 / kRows; bx <= (x1 - 1) / kRows && !any; ++bx) {
        const RowProp &rp = props[((long long)zb * nbx + bx) * segs + ty];
        for (int l = 0; l < nyv; ++l)
          if (rp.conf[l] < conf_thr) {
            any = true;
            break;
          }
      }
    flag[t] = any ? 1 : 0;
    if (any) {
      masks[t] |= 1u << bit;  // one thread per tile; the atlases' launches are ordered
      const unsigned long long rows = (unsigned long long)(z1 - z0) * (x1 - x0);
      atomicAdd(fallbacks, rows * nyv);
      atomicAdd(evaluated, rows * kAxis * kAxis * kAxis);
    }
  }
}

// The no-network centre prior, library build (run-time strides).
__global__ void __launch_bounds__(kRescoreWarps * 32, 4)
    rescore_prior_kernel(const __grid_constant__ PriorList pl, const float *__restrict__ img,
                         const float *__restrict__ atl, const float *__restrict__ lab, int nx,
                         int ny, int nz, int apitch, float scale, float *__restrict__ pacc,
                         float *__restrict__ wacc, unsigned long long *__restrict__ evaluated,
                         int hw) {
  rescore_prior_body(pl, img, atl, lab, nx, ny, nz, apitch, scale, pacc, wacc, evaluated, hw);
}

__global__ void finalize_kernel(const float *__restrict__ pacc, const float *__restrict__ wacc,
                                float *__restrict__ out, int nx, int ny, int nz, int lo) {
  const int ix = nx - 2 * lo, iy = ny - 2 * lo, iz = nz - 2 * lo;
  const long long total = (ix > 0 && iy > 0 && iz > 0) ? (long long)ix * iy * iz : 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int y = (int)(i % iy) + lo;
    const long long r0 = i / iy;
    const int x = (int)(r0 % ix) + lo;
    const int z = (int)(r0 / ix) + lo;
    const long long v = (long long)z * nx * ny + (long long)x * ny + y;
    const float pr = pacc[v], sw = wacc[v];
    out[v] = (fabsf(pr) > kDblEpsilonF && fabsf(sw) > kDblEpsilonF) ? __fdiv_rn(pr, sw)
                                                                    : __int_as_float(0x7fc00000);
  }
}

int sms() {
  int dev = 0, n = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  return n;
}

int anchor_of_host(int b, int block, int extent) {
  const int a = b * block + block / 2;
  return a < extent ? a : extent - 1;
}

// Scratch layout: two BF16 channel-last feature volumes, the product and weight sums, the three
// packed fragment tables and the fallback counter.
struct InferScratch {
  __nv_bfloat16 *fa, *fb;
  float *pacc, *wacc;
  uint32_t *frag;
  unsigned long long *fallbacks;  // (voxel, atlas) pairs that took the full search
  unsigned long long *evaluated;  // offsets evaluated by warp rows, summed over rows
  int *err;                       // bounded-wait status of the probe hook
  RowProp *props;                 // row-segment proposals of the block anchor rows (two tables)
  int *lists;                     // the convolutions' x tiles and work items
};

// Bytes before the proposal table (features, sums, fragments, counters), 256-aligned.
size_t infer_base_bytes(long long nvox) {
  const size_t b = (size_t)nvox * kC * 2 * 2 + (size_t)nvox * 4 * 2 +
                   (3 * (size_t)(kFragWords + kRwFragWords) + kC1FragWords) * 4 + 256;
  return (b + 255) / 256 * 256;
}

InferScratch carve(void *scratch, long long nvox) {
  InferScratch r;
  unsigned char *p = static_cast<unsigned char *>(scratch);
  r.fa = reinterpret_cast<__nv_bfloat16 *>(p);
  r.fb = r.fa + nvox * kC;
  r.pacc = reinterpret_cast<float *>(r.fb + nvox * kC);
  r.wacc = r.pacc + nvox;
  r.frag = reinterpret_cast<uint32_t *>(r.wacc + nvox);
  r.fallbacks = reinterpret_cast<unsigned long long *>(
      r.frag + 3 * (kFragWords + kRwFragWords) + kC1FragWords);
  r.evaluated = r.fallbacks + 1;
  r.err = reinterpret_cast<int *>(r.fallbacks + 2);
  r.props = reinterpret_cast<RowProp *>(static_cast<unsigned char *>(scratch) +
                                        infer_base_bytes(nvox));
  r.lists = nullptr;  // placed by the launch, which knows the geometry
  return r;
}

}  // namespace

size_t prop_table_bytes(const Geometry &g) {
  const size_t rows = (size_t)g.nz * g.nx * (size_t)((g.ny + kRowOut - 1) / kRowOut + 1);
  return (rows * sizeof(RowProp) + 255) / 256 * 256;
}

// The confidence fallback's item count, items (up to 16 per tile), atlas masks and per-atlas tile
// flags (after the convolutions' lists).
size_t fallback_bytes(const Geometry &g) {
  const TileShape ts = fuse_tile_shape(g);
  const size_t ntiles = (size_t)ts.tiles_y * ts.tiles_x * ts.tiles_z;
  return 16 + 16 * ntiles * sizeof(int) + ntiles * sizeof(uint32_t) + ntiles + 256;
}

size_t fallback_partial_bytes(const Geometry &g) {
  const int slots = (std::min(g.num, kFallbackAtlases) + 1) / 2;
  return (size_t)2 * slots * (size_t)g.nvox() * sizeof(float);
}

size_t infer_scratch_bytes(const Geometry &g) {
  return infer_base_bytes(g.nvox()) + 2 * prop_table_bytes(g) + conv_list_bytes(g) +
         fallback_bytes(g) + 256;
}

unsigned long long *infer_counters(void *scratch, long long nvox) {
  return carve(scratch, nvox).fallbacks;
}

namespace {

// TMA map over a channel-last BF16 feature volume [nz][nx][ny][16]: one box is a conv16 slab
// (3 z x 6 x x 66 y voxels), 32-byte swizzled, out-of-volume voxels zero.
cudaError_t make_feature_map(CUtensorMap *map, const __nv_bfloat16 *base, const Geometry &g,
                             int rows = kCvSX) {
  auto fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(tensor_map_encoder());
  if (!fn) return cudaErrorNotSupported;
  // [half][z][x][y, 8 channels] with each (half, z, x) row as 2 ny 8-byte elements; one box = a
  // conv16 ring slot (one plane, `rows` x-rows of 128 y), out-of-volume voxels zero
  const cuuint64_t dims[4] = {2 * (cuuint64_t)g.ny, (cuuint64_t)g.nx, (cuuint64_t)g.nz, 2};
  const cuuint64_t strides[3] = {16 * (cuuint64_t)g.ny, 16 * (cuuint64_t)g.ny * g.nx,
                                 16 * (cuuint64_t)g.nvox()};
  const cuuint32_t box[4] = {2 * kCvSY, (cuuint32_t)rows, 1, 2};
  const cuuint32_t estr[4] = {1u, 1u, 1u, 1u};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, const_cast<__nv_bfloat16 *>(base), dims,
                  strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

// What each convolution must produce. The proposals read conv4 features on the anchor rows
// (z, x) of the row blocks, at the interior y; layer conv(4 - r) is needed r voxels around them.
// Every needed output's receptive field lies inside the volume (interior margin 6 > 4 layers), so
// the zero padding of the volume edge never reaches a needed value and skipped outputs are never
// read. Dense plans compute every voxel. `lists` (uploaded to the device) holds the 3 nx x-tile
// entries of the sparse plans (first row | row mask << 16), then each layer's work items.
struct ConvPlan {
  int c1_z, c1_nz, c1_x, c1_nx;  // conv1 box (z, x; every y)
  int y_lo[4], y_hi[4];          // [0..2]: conv2..conv4, [3]: conv1
  int n_items[4], item_off[4];   // work items (offset in ints into the lists)
  bool ring[4];                  // conv16_kernel (plane-slot ring) or conv16_rows_kernel
  bool dense;
};

// Work items of a layer: every (x tile, y tile) column over each run of consecutive planes of
// `zs`, cut into the fewest pieces of at most kCvChunk planes, of nearly equal length (a 101-plane
// run: 8 pieces of 12 or 13, which spreads evenly over the persistent grid).
void add_items(ConvPlan &p, int l, const std::vector<int> &zs, int x_tiles, std::vector<int> &lists,
               int tile_y = kCvTY) {
  const int tiles_y = (p.y_hi[l] - p.y_lo[l] + tile_y - 1) / tile_y;
  if (lists.size() & 1) lists.push_back(0);  // items are read as 8-byte int2
  p.item_off[l] = (int)lists.size();
  for (int xi = 0; xi < x_tiles; ++xi)
    for (int ty = 0; ty < tiles_y; ++ty)
      for (size_t i = 0; i < zs.size();) {
        size_t e = i + 1;
        while (e < zs.size() && zs[e] == zs[e - 1] + 1) ++e;  // the run [i, e)
        const int len = (int)(e - i), pieces = (len + kCvChunk - 1) / kCvChunk;
        for (int q = 0, at = 0; q < pieces; ++q) {
          const int n = len / pieces + (q < len % pieces ? 1 : 0);
          lists.push_back(xi | (ty << 16));
          lists.push_back(zs[i + at] | (n << 16));
          at += n;
        }
        i = e;
      }
  p.n_items[l] = (int)((lists.size() - p.item_off[l]) / 2);
  // the plane-slot ring pays off when items hold runs of planes; short runs (isolated anchor
  // planes, or 3 around them) take the double-buffered variant
  long long planes = 0;
  for (size_t i = p.item_off[l] + 1; i < lists.size(); i += 2) planes += (unsigned)lists[i] >> 16;
  p.ring[l] = planes >= 4LL * p.n_items[l];
}

ConvPlan dense_plan(const Geometry &g, std::vector<int> &lists) {
  ConvPlan p{};
  lists.assign(4 * (size_t)g.nx, 0);
  p.c1_nz = g.nz;
  p.c1_nx = g.nx;
  std::vector<int> zs(g.nz);
  for (int z = 0; z < g.nz; ++z) zs[z] = z;
  for (int l = 0; l < 4; ++l) {
    p.y_hi[l] = g.ny;
    add_items(p, l, zs, (g.nx + kCvTX - 1) / kCvTX, lists, l == 3 ? kC1Y : kCvTY);
  }
  p.dense = true;
  return p;
}

// Anchor rows of blocks of `block` rows along an axis with `extent` interior rows from row 6.
std::vector<int> anchors(int extent, int block, int lo) {
  std::vector<int> a;
  for (int b = 0; b * block < extent; ++b) a.push_back(lo + anchor_of_host(b, block, extent));
  return a;
}

// The rows within `radius` of an anchor, in order.
std::vector<int> rows_near(const std::vector<int> &anc, int radius, int n) {
  std::vector<char> need(n, 0);
  for (int a : anc)
    for (int d = -radius; d <= radius; ++d)
      if (a + d >= 0 && a + d < n) need[a + d] = 1;
  std::vector<int> r;
  for (int i = 0; i < n; ++i)
    if (need[i]) r.push_back(i);
  return r;
}

// Sparse plan for row blocks of `block`: greedy 4-row x tiles starting at the first uncovered
// needed row, items over the needed planes.
ConvPlan sparse_plan(const Geometry &g, int block, std::vector<int> &lists) {
  ConvPlan p{};
  lists.assign(4 * (size_t)g.nx, 0);
  const int iz = g.iz, ix = g.ix, iy = g.iy;
  if (iz <= 0 || ix <= 0 || iy <= 0) return p;  // no interior: nothing to compute
  const std::vector<int> az = anchors(iz, block, g.lo), ax = anchors(ix, block, g.lo);
  p.c1_z = az.front() - 3;
  p.c1_nz = az.back() + 4 - p.c1_z;
  p.c1_x = ax.front() - 3;
  p.c1_nx = ax.back() + 4 - p.c1_x;
  for (int l = 0; l < 3; ++l) {
    const int radius = 2 - l;
    const std::vector<int> zs = rows_near(az, radius, g.nz), xs = rows_near(ax, radius, g.nx);
    int nt = 0;
    for (size_t i = 0; i < xs.size();) {
      const int x0 = xs[i];
      unsigned mask = 0;
      while (i < xs.size() && xs[i] < x0 + kCvTX) mask |= 1u << (xs[i++] - x0);
      lists[(size_t)l * g.nx + nt++] = x0 | (int)(mask << 16);
    }
    p.y_lo[l] = g.lo - radius;
    p.y_hi[l] = g.ny - g.lo + radius;
    add_items(p, l, zs, nt, lists);
  }
  // conv1: the box 3 rows and planes around the anchors, y within 3 of the interior
  {
    int nt = 0;
    for (int x0 = p.c1_x; x0 < p.c1_x + p.c1_nx; x0 += kCvTX) {
      const int rows = p.c1_x + p.c1_nx - x0 < kCvTX ? p.c1_x + p.c1_nx - x0 : kCvTX;
      lists[3 * (size_t)g.nx + nt++] = x0 | (int)(((1u << rows) - 1u) << 16);
    }
    std::vector<int> zs(p.c1_nz);
    for (int i = 0; i < p.c1_nz; ++i) zs[i] = p.c1_z + i;
    p.y_lo[3] = g.lo - 3;
    p.y_hi[3] = g.ny - g.lo + 3;
    add_items(p, 3, zs, nt, lists, kC1Y);
  }
  return p;
}

// conv1 .. conv4 of one (input, atlas) pair; returns the buffer holding the conv4 features.
cudaError_t run_convs(const Geometry &g, const __nv_bfloat16 *wbf, const float *img,
                      const float *atlas_a, int apitch, const InferScratch &sc, int *err,
                      const ConvPlan &p, __nv_bfloat16 **features, cudaStream_t s) {
  const int n_sm = sms();
  *features = sc.fb;  // conv1 -> fa, conv2 -> fb, conv3 -> fa, conv4 -> fb
  cudaError_t e;
  ConvGrid cg;
  cg.nx = g.nx;
  cg.ny = g.ny;
  cg.nz = g.nz;
  cg.nvox = g.nvox();
  if (p.n_items[3] > 0) {
    cg.xlist = p.dense ? nullptr : sc.lists + 3 * g.nx;
    cg.items = reinterpret_cast<const int2 *>(sc.lists + p.item_off[3]);
    cg.n_items = p.n_items[3];
    cg.y_lo = p.y_lo[3];
    cg.y_hi = p.y_hi[3];
    cg.tile_y = kC1Y;
    const int blocks = cg.n_items < 2 * n_sm ? cg.n_items : 2 * n_sm;
    conv1_tc_kernel<<<blocks, kC1Threads, kC1Smem, s>>>(
        img, atlas_a, apitch, sc.frag + 3 * (kFragWords + kRwFragWords), wbf, sc.fa, cg, err);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  CUtensorMap maps[2], maps3[2];
  if ((e = make_feature_map(&maps[0], sc.fa, g)) != cudaSuccess) return e;
  if ((e = make_feature_map(&maps[1], sc.fb, g)) != cudaSuccess) return e;
  if ((e = make_feature_map(&maps3[0], sc.fa, g, 3)) != cudaSuccess) return e;
  if ((e = make_feature_map(&maps3[1], sc.fb, g, 3)) != cudaSuccess) return e;
  const int boffs[3] = {kB2, kB3, kB4};
  __nv_bfloat16 *bufs[2] = {sc.fa, sc.fb};
  for (int l = 0; l < 3; ++l) {
    cg.xlist = p.dense ? nullptr : sc.lists + l * g.nx;
    cg.items = reinterpret_cast<const int2 *>(sc.lists + p.item_off[l]);
    cg.n_items = p.n_items[l];
    cg.y_lo = p.y_lo[l];
    cg.y_hi = p.y_hi[l];
    cg.tile_y = kCvTY;
    if (cg.n_items <= 0) continue;
    const int blocks = cg.n_items < 2 * n_sm ? cg.n_items : 2 * n_sm;
    if (!p.ring[l]) {
      conv16_rows_kernel<<<blocks, kCvThreads, kRwSmem, s>>>(
          maps[l & 1], maps3[l & 1], sc.frag + 3 * kFragWords + l * kRwFragWords, wbf, boffs[l],
          bufs[(l + 1) & 1], cg, err);
      if ((e = cudaGetLastError()) != cudaSuccess) return e;
      continue;
    }
    conv16_kernel<<<blocks, kCvThreads, kConvSmem, s>>>(maps[l & 1], sc.frag + l * kFragWords, wbf,
                                                        boffs[l], bufs[(l + 1) & 1], cg, err);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t pack_all(const __nv_bfloat16 *wbf, uint32_t *frag, cudaStream_t s) {
  cudaError_t e0 = cudaFuncSetAttribute(conv16_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)kConvSmem);
  if (e0 != cudaSuccess) return e0;
  e0 = cudaFuncSetAttribute(conv16_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)kRwSmem);
  if (e0 != cudaSuccess) return e0;
  const int woffs[3] = {kW2, kW3, kW4};
  for (int l = 0; l < 3; ++l) {
    pack_frags_kernel<<<(kFragWords + 255) / 256, 256, 0, s>>>(wbf, woffs[l], frag + l * kFragWords);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    pack_rows_kernel<<<(kRwFragWords + 255) / 256, 256, 0, s>>>(
        wbf, woffs[l], frag + 3 * kFragWords + l * kRwFragWords);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  e0 = cudaFuncSetAttribute(conv1_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)kC1Smem);
  if (e0 != cudaSuccess) return e0;
  pack_c1_kernel<<<(kC1FragWords + 255) / 256, 256, 0, s>>>(
      wbf, frag + 3 * (kFragWords + kRwFragWords));
  return cudaSuccess;
}

#include "pct_rescore_src.inc"  // k_pct_rescore_source: the text of pct_rescore.cuh

// Resident CTAs per SM of the run-time compiled z-pair rescoring (its launch bound, 96 registers).
// Its launches are one wave of resident CTAs; the one-plane items keep one CTA per four items
// (as one wave of 7 per SM they measured slower: k = 20 4.80 ms against 4.61, k = 10 4.35
// against 4.02).
constexpr int kRs8CtasPerSm = PCT_RS_MIN_CTAS8;

// An entry point of the rescoring module compiled for this x extent and atlas row pitch, or
// nullptr: the environment variable PCT_RESCORE_JIT=0 keeps the library build, as does a
// missing NVRTC.
void *rescore_jit(const char *entry, int nx, int pitch, int hw, cudaStream_t s) {
  const char *env = getenv("PCT_RESCORE_JIT");
  if (env && env[0] == '0') return nullptr;
  const std::vector<std::string> opts = {"-DPCT_RS_JIT", "-DPCT_RS_NX=" + std::to_string(nx),
                                         "-DPCT_RS_PITCH=" + std::to_string(pitch),
                                         "-DPCT_RS_HW=" + std::to_string(hw)};
  // while `s` is being captured a module is only looked up, never built (loading one is not a
  // stream operation)
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  const bool build = cudaStreamIsCapturing(s, &cap) == cudaSuccess && cap == cudaStreamCaptureStatusNone;
  return jit::kernel(k_pct_rescore_source, "pct_rescore.cuh", opts, entry, build);
}

// One atlas's proposal rescoring: the geometry's compiled module where there is one, else the
// library's kernel (same code, run-time strides).
cudaError_t launch_rescore4(int level, int blocks, const RowProp *props, const float *img,
                            const float *atl, const float *lab, int nx, int ny, int nz,
                            int apitch, float scale, float conf_thr, float *pacc, float *wacc,
                            unsigned long long *fallbacks, unsigned long long *evaluated,
                            const unsigned char *tile_flag, RescoreTiles ts, int hw,
                            cudaStream_t s) {
  // z-pair items (two planes of a block per warp) where there are two or more interior planes
  // and 32 offsets per item (at 10 and 20 the one-plane items' higher occupancy wins: learned
  // step k = 10 4.02 ms against 4.10, k = 20 4.61 against 4.65, k = 32 5.34 against 5.24)
  const int lo = hw + 1, ix = nx - 2 * lo, iy = ny - 2 * lo, iz = nz - 2 * lo;
  const char *pairs_env = getenv("PCT_RS_PAIRS");
  if (level == 4 && iz >= 2 && ix >= kRows && iy > 0 && !(pairs_env && pairs_env[0] == '0')) {
    void *f8 = rescore_jit(level == 2 ? "pct_rescore8_l2" : level == 3 ? "pct_rescore8_l3"
                                                                       : "pct_rescore8_l4",
                           nx, apitch, hw, s);
    if (f8) {
      const long long items = (long long)((iz + kRows - 1) / kRows) * 2 * ((ix + kRows - 1) / kRows) *
                              ((iy + kRowOut - 1) / kRowOut);
      // one wave of resident CTAs (5 per SM) walking the items: 5.155 ms per learned step
      // against 5.199 with one CTA per 4 items
      const long long b8 = (items + kRescoreWarps - 1) / kRescoreWarps;
      int blocks8 = (int)(b8 > kRs8CtasPerSm * (long long)sms() ? kRs8CtasPerSm * (long long)sms()
                                                                : b8);
      void *args[] = {&props, &img,     &atl,  &lab,  &nx,        &ny,        &nz,        &apitch,
                      &scale, &conf_thr, &pacc, &wacc, &fallbacks, &evaluated, &tile_flag, &ts,
                      &hw};
      return jit::launch(f8, blocks8, kRescoreWarps * 32, s, args);
    }
  }
  void *fn = rescore_jit(level == 2 ? "pct_rescore4_l2" : level == 3 ? "pct_rescore4_l3"
                                                                      : "pct_rescore4_l4",
                         nx, apitch, hw, s);
  if (fn) {
    void *args[] = {&props, &img,     &atl,  &lab,  &nx,        &ny,        &nz,        &apitch,
                    &scale, &conf_thr, &pacc, &wacc, &fallbacks, &evaluated, &tile_flag, &ts,
                    &hw};
    return jit::launch(fn, blocks, kRescoreWarps * 32, s, args);
  }
  auto k4 = level == 2 ? rescore4_kernel<2> : level == 3 ? rescore4_kernel<3> : rescore4_kernel<4>;
  k4<<<blocks, kRescoreWarps * 32, 0, s>>>(props, img, atl, lab, nx, ny, nz, apitch, scale,
                                            conf_thr, pacc, wacc, fallbacks, evaluated, tile_flag,
                                            ts, hw);
  return cudaGetLastError();
}

cudaError_t launch_rescore_prior(int blocks, const PriorList &pl, const float *img,
                                 const float *atl, const float *lab, int nx, int ny, int nz,
                                 int apitch, float scale, float *pacc, float *wacc,
                                 unsigned long long *evaluated, int hw, cudaStream_t s) {
  // z-pair items from 32 offsets on, as for the proposals (prior k = 81: 4.54 ms against 4.85,
  // k = 123 6.59 against 7.20)
  const int lo = hw + 1, ix = nx - 2 * lo, iy = ny - 2 * lo, iz = nz - 2 * lo;
  const char *pairs_env = getenv("PCT_RS_PAIRS");
  if (pl.n >= 32 && iz >= 2 && ix >= kRows && iy > 0 && !(pairs_env && pairs_env[0] == '0')) {
    void *f8 = rescore_jit("pct_rescore_prior8", nx, apitch, hw, s);
    if (f8) {
      const long long items = (long long)((iz + kRows - 1) / kRows) * 2 * ((ix + kRows - 1) / kRows) *
                              ((iy + kRowOut - 1) / kRowOut);
      // one wave of resident CTAs (5 per SM) walking the items: 5.155 ms per learned step
      // against 5.199 with one CTA per 4 items
      const long long b8 = (items + kRescoreWarps - 1) / kRescoreWarps;
      int blocks8 = (int)(b8 > kRs8CtasPerSm * (long long)sms() ? kRs8CtasPerSm * (long long)sms()
                                                                : b8);
      PriorList copy = pl;
      void *args[] = {&copy, &img, &atl, &lab, &nx, &ny, &nz, &apitch, &scale, &pacc, &wacc,
                      &evaluated, &hw};
      return jit::launch(f8, blocks8, kRescoreWarps * 32, s, args);
    }
  }
  void *fn = rescore_jit("pct_rescore_prior", nx, apitch, hw, s);
  if (fn) {
    PriorList copy = pl;
    void *args[] = {&copy, &img, &atl, &lab, &nx, &ny, &nz, &apitch, &scale, &pacc, &wacc,
                    &evaluated, &hw};
    return jit::launch(fn, blocks, kRescoreWarps * 32, s, args);
  }
  rescore_prior_kernel<<<blocks, kRescoreWarps * 32, 0, s>>>(pl, img, atl, lab, nx, ny, nz, apitch,
                                                             scale, pacc, wacc, evaluated, hw);
  return cudaGetLastError();
}

}  // namespace

// The learned form over all atlases of `in` (atlas and label rows `in.pitch` floats apart, the
// input MRI contiguous). Writes the interior of `out`; the border is left untouched.
cudaError_t launch_learned(const Geometry &g, const void *weights, const SlabInputs &in, float *out,
                           double div, float conf_thr, int block, int level, bool every_voxel,
                           void *scratch, float *fb_partial, int *err,
                           const LearnedStreams *streams, cudaStream_t s) {
  if (block < 1 || level < 2 || level > 4) return cudaErrorInvalidValue;
  // work items pack x and z coordinates in 16 bits
  if (g.nx >= 65536 || g.nz >= 65536) return cudaErrorInvalidValue;
  const __nv_bfloat16 *wbf = static_cast<const __nv_bfloat16 *>(weights);
  const long long nvox = g.nvox();
  const long long astride = (long long)g.nz * g.nx * in.pitch;
  InferScratch sc = carve(scratch, nvox);
  sc.lists = reinterpret_cast<int *>(reinterpret_cast<unsigned char *>(sc.props) +
                                     2 * prop_table_bytes(g));
  cudaError_t e;
  std::vector<int> lists;
  ConvPlan plan = sparse_plan(g, block, lists);
  if (every_voxel) {
    // whole-volume convolutions with the same kernel per layer as the restricted plan, so that
    // both give the same values
    const ConvPlan restricted = plan;
    plan = dense_plan(g, lists);
    for (int l = 0; l < 3; ++l) plan.ring[l] = restricted.ring[l];
  }
  if (lists.size() * sizeof(int) > conv_list_bytes(g)) return cudaErrorInvalidValue;
  if ((e = cudaMemcpyAsync(sc.lists, lists.data(), lists.size() * sizeof(int),
                           cudaMemcpyHostToDevice, s)) != cudaSuccess)
    return e;
  // Confidence fallback through the plain kernel's tiles, where its TMA maps can read the stacks
  // (16-byte row strides); otherwise the rescoring runs the full window for low-confidence rows.
  const TileShape ts = fuse_tile_shape(g);
  const int ntiles = ts.tiles_y * ts.tiles_x * ts.tiles_z;
  const bool tile_fallback =
      conf_thr > 0.f && fb_partial && block == kRows && g.hw == 5 && ntiles > 0 &&
      in.pitch % 4 == 0 && reinterpret_cast<uintptr_t>(in.atlas) % 16 == 0 &&
      reinterpret_cast<uintptr_t>(in.label) % 16 == 0;
  unsigned char *fb_region = reinterpret_cast<unsigned char *>(sc.lists) + conv_list_bytes(g);
  int *fb_count = reinterpret_cast<int *>(fb_region);
  int *fb_items = reinterpret_cast<int *>(fb_region + 16);
  uint32_t *fb_masks = reinterpret_cast<uint32_t *>(fb_items + 16 * (size_t)ntiles);
  unsigned char *fb_flag = reinterpret_cast<unsigned char *>(fb_masks + ntiles);
  if ((e = cudaMemsetAsync(sc.pacc, 0, (size_t)nvox * 4 * 2, s)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(sc.fallbacks, 0, 2 * sizeof(unsigned long long), s)) != cudaSuccess)
    return e;
  if ((e = pack_all(wbf, sc.frag, s)) != cudaSuccess) return e;
  const float neg_k = (float)(-1.4426950408889634 / div);
  const float scale = (float)sqrt(1.4426950408889634 / div);
  const int nblk = sms() * 8;
  long long rows = 0;
  if (g.ix > 0 && g.iy > 0 && g.iz > 0)
    rows = (long long)g.iz * g.ix * ((g.iy + kRowOut - 1) / kRowOut);
  const long long rblk = (rows + kRescoreWarps - 1) / kRescoreWarps;
  const int rescore_blocks = (int)(rblk < 1 ? 1 : (rblk > 64LL * sms() ? 64LL * sms() : rblk));
  long long prows = 0;
  if (g.ix > 0 && g.iy > 0 && g.iz > 0)
    prows = (long long)((g.iz + block - 1) / block) * ((g.ix + block - 1) / block) *
            ((g.iy + kRowOut - 1) / kRowOut);
  const long long pblk = (prows + kRescoreWarps - 1) / kRescoreWarps;
  const int propose_blocks = (int)(pblk < 1 ? 1 : (pblk > 64LL * sms() ? 64LL * sms() : pblk));
  // two streams: atlas a's convolutions and proposal (stream cs) run while atlas a - 1 is
  // rescored (stream s); the proposal tables alternate, the sums are touched by s only
  const bool two = streams && streams->aux && g.num > 1;
  const cudaStream_t cs = two ? streams->aux : s;
  RowProp *tables[2] = {sc.props, reinterpret_cast<RowProp *>(
                                      reinterpret_cast<unsigned char *>(sc.props) +
                                      prop_table_bytes(g))};
  if (two) {
    if ((e = cudaEventRecord(streams->ev[0], s)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(cs, streams->ev[0], 0)) != cudaSuccess) return e;
  }
  // Every exit after the fork joins the auxiliary stream back into s (the last atlas's wait for
  // its proposal already does on success; on an error the work queued on cs must not outlive
  // the call unordered).
  auto join = [&](cudaError_t status) {
    if (two && cudaEventRecord(streams->ev[0], cs) == cudaSuccess)
      cudaStreamWaitEvent(s, streams->ev[0], 0);
    return status;
  };
  for (int a = 0; a < g.num; ++a) {
    const float *A = in.atlas + a * astride, *L = in.label + a * astride;
    RowProp *props = two ? tables[a & 1] : tables[0];
    __nv_bfloat16 *f4 = nullptr;
    if ((e = run_convs(g, wbf, in.img, A, in.pitch, sc, err, plan, &f4, cs)) != cudaSuccess)
      return join(e);
    // the table is free once the rescoring of atlas a - 2 has read it
    if (two && a >= 2 && (e = cudaStreamWaitEvent(cs, streams->ev[3 + (a & 1)], 0)) != cudaSuccess)
      return join(e);
    auto kp = g.hw == 5 ? propose_rows_kernel<5> : g.hw == 4 ? propose_rows_kernel<4>
                                                              : propose_rows_kernel<3>;
    kp<<<propose_blocks, kRescoreWarps * 32, 0, cs>>>(f4, wbf, g.nx, g.ny, g.nz, block, level,
                                                      props);
    if ((e = cudaGetLastError()) != cudaSuccess) return join(e);
    if (two) {
      if ((e = cudaEventRecord(streams->ev[1 + (a & 1)], cs)) != cudaSuccess) return join(e);
      if ((e = cudaStreamWaitEvent(s, streams->ev[1 + (a & 1)], 0)) != cudaSuccess) return join(e);
    }
    if (block == kRows && g.ix >= kRows &&
        (long long)g.nz * g.nx * in.pitch < (1LL << 31) - 1) {
      if (tile_fallback) {
        // atlases in blocks of 32 (the mask bits); a block's full search runs after its last
        if (a % kFallbackAtlases == 0 &&
            (e = cudaMemsetAsync(fb_masks, 0, (size_t)ntiles * sizeof(uint32_t), s)) != cudaSuccess)
          return join(e);
        flag_tiles_kernel<<<(ntiles + 255) / 256, 256, 0, s>>>(
            props, g.nx, g.ny, g.nz, conf_thr, ts, fb_flag, fb_masks, a % kFallbackAtlases,
            sc.fallbacks, sc.evaluated);
        if ((e = cudaGetLastError()) != cudaSuccess) return join(e);
      }
      if ((e = launch_rescore4(level, rescore_blocks, props, in.img, A, L, g.nx, g.ny, g.nz,
                               in.pitch, scale, tile_fallback ? 0.f : conf_thr, sc.pacc, sc.wacc,
                               sc.fallbacks, sc.evaluated, tile_fallback ? fb_flag : nullptr,
                               RescoreTiles{ts.zt, ts.xc, ts.tiles_x, ts.tiles_y}, g.hw, s)) !=
          cudaSuccess)
        return join(e);
      if (tile_fallback && (a % kFallbackAtlases == kFallbackAtlases - 1 || a == g.num - 1)) {
        if ((e = launch_fuse_masked(g, in, div, a - a % kFallbackAtlases, fb_masks, fb_items,
                                    fb_count, fb_partial, sc.pacc, sc.wacc, err, s)) !=
            cudaSuccess)
          return join(e);
      }
    } else {
      rescore_kernel<<<rescore_blocks, kRescoreWarps * 32, 0, s>>>(
          props, block, level, in.img, A, L, g.nx, g.ny, g.nz, in.pitch, neg_k, conf_thr, sc.pacc,
          sc.wacc, sc.fallbacks, sc.evaluated, g.hw);
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return join(e);
    if (two && (e = cudaEventRecord(streams->ev[3 + (a & 1)], s)) != cudaSuccess) return join(e);
  }
  finalize_kernel<<<nblk, 256, 0, s>>>(sc.pacc, sc.wacc, out, g.nx, g.ny, g.nz, g.lo);
  return cudaGetLastError();
}

// The k offsets (dw, du, dv) of the NH^3 window (half width hw) nearest its centre, by squared
// distance, ties in (dw, du, dv) order.
std::vector<std::array<int, 3>> prior_offsets(int k, int hw) {
  std::vector<std::array<int, 3>> all;
  for (int dw = -hw; dw <= hw; ++dw)
    for (int du = -hw; du <= hw; ++du)
      for (int dv = -hw; dv <= hw; ++dv) all.push_back({dw, du, dv});
  std::stable_sort(all.begin(), all.end(), [](const std::array<int, 3> &a, const std::array<int, 3> &b) {
    return a[0] * a[0] + a[1] * a[1] + a[2] * a[2] < b[0] * b[0] + b[1] * b[1] + b[2] * b[2];
  });
  all.resize(k);
  return all;
}

cudaError_t launch_prior(const Geometry &g, const SlabInputs &in, float *out, double div, int k,
                         void *scratch, cudaStream_t s) {
  const long long window = (2LL * g.hw + 1) * (2 * g.hw + 1) * (2 * g.hw + 1);
  if (k < 1 || k > kMaxPrior || k > window) return cudaErrorInvalidValue;
  if (g.ix < kRows || (long long)g.nz * g.nx * in.pitch >= (1LL << 31) - 1)
    return cudaErrorInvalidValue;
  const long long nvox = g.nvox();
  InferScratch sc = carve(scratch, nvox);
  cudaError_t e;
  if ((e = cudaMemsetAsync(sc.pacc, 0, (size_t)nvox * 4 * 2, s)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(sc.fallbacks, 0, 2 * sizeof(unsigned long long), s)) != cudaSuccess)
    return e;
  PriorList pl{};
  pl.n = k;
  const int axy = g.nx * in.pitch;
  const auto offs = prior_offsets(k, g.hw);
  for (int c = 0; c < k; ++c) pl.off[c] = offs[c][0] * axy + offs[c][1] * in.pitch + offs[c][2];
  const float scale = (float)sqrt(1.4426950408889634 / div);
  long long rows = 0;
  if (g.ix > 0 && g.iy > 0 && g.iz > 0)
    rows = (long long)g.iz * g.ix * ((g.iy + kRowOut - 1) / kRowOut);
  const long long rblk = (rows + kRescoreWarps - 1) / kRescoreWarps;
  const int blocks = (int)(rblk < 1 ? 1 : (rblk > 64LL * sms() ? 64LL * sms() : rblk));
  const long long astride = (long long)g.nz * g.nx * in.pitch;
  for (int a = 0; a < g.num; ++a) {
    if ((e = launch_rescore_prior(blocks, pl, in.img, in.atlas + a * astride,
                                  in.label + a * astride, g.nx, g.ny, g.nz, in.pitch, scale,
                                  sc.pacc, sc.wacc, sc.evaluated, g.hw, s)) != cudaSuccess)
      return e;
  }
  finalize_kernel<<<sms() * 8, 256, 0, s>>>(sc.pacc, sc.wacc, out, g.nx, g.ny, g.nz, g.lo);
  return cudaGetLastError();
}

// Testing hook: conv4 features and proposals of one (input, atlas) pair at given voxels.
cudaError_t learned_probe(const Geometry &g, const void *weights, const float *img,
                          const float *atlas_a, void *scratch, const int64_t *voxels, int n,
                          float *features, signed char *top, float *conf, cudaStream_t s) {
  const __nv_bfloat16 *wbf = static_cast<const __nv_bfloat16 *>(weights);
  if (g.nx >= 65536 || g.nz >= 65536) return cudaErrorInvalidValue;
  InferScratch sc = carve(scratch, g.nvox());
  sc.lists = reinterpret_cast<int *>(reinterpret_cast<unsigned char *>(sc.props) +
                                     2 * prop_table_bytes(g));
  cudaError_t e;
  if ((e = pack_all(wbf, sc.frag, s)) != cudaSuccess) return e;
  __nv_bfloat16 *f4 = nullptr;
  if ((e = cudaMemsetAsync(sc.err, 0, sizeof(int), s)) != cudaSuccess) return e;
  std::vector<int> lists;
  const ConvPlan plan = dense_plan(g, lists);
  if (lists.size() * sizeof(int) > conv_list_bytes(g)) return cudaErrorInvalidValue;
  if ((e = cudaMemcpyAsync(sc.lists, lists.data(), lists.size() * sizeof(int),
                           cudaMemcpyHostToDevice, s)) != cudaSuccess)
    return e;
  if ((e = run_convs(g, wbf, img, atlas_a, g.ny, sc, sc.err, plan, &f4, s)) != cudaSuccess)
    return e;
  // the sums area is free here: voxel list, proposals and confidences go there
  int64_t *d_vox = reinterpret_cast<int64_t *>(sc.pacc);
  signed char *d_top = reinterpret_cast<signed char *>(d_vox + n);
  float *d_conf = reinterpret_cast<float *>(d_top + ((12 * (size_t)n + 15) / 16) * 16);
  if ((size_t)n * (8 + 12 + 4) + 16 > (size_t)g.nvox() * 8) return cudaErrorInvalidValue;
  if ((e = cudaMemcpyAsync(d_vox, voxels, n * sizeof(int64_t), cudaMemcpyHostToDevice, s)) !=
      cudaSuccess)
    return e;
  proposal_hook_kernel<<<(n + 127) / 128, 128, 0, s>>>(f4, wbf, d_vox, n, g.nvox(), d_top, d_conf,
                                                       g.hw);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if (top && (e = cudaMemcpyAsync(top, d_top, 12 * (size_t)n, cudaMemcpyDeviceToHost, s)) !=
                 cudaSuccess)
    return e;
  if (conf && (e = cudaMemcpyAsync(conf, d_conf, 4 * (size_t)n, cudaMemcpyDeviceToHost, s)) !=
                  cudaSuccess)
    return e;
  int status = 0;
  if ((e = cudaMemcpyAsync(&status, sc.err, sizeof(int), cudaMemcpyDeviceToHost, s)) != cudaSuccess)
    return e;
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
  if (status != 0) return cudaErrorLaunchTimeout;
  if (features) {
    for (int i = 0; i < n; ++i) {
      __nv_bfloat16 tmp[kC];
      for (int h = 0; h < 2; ++h)
        if ((e = cudaMemcpy(tmp + 8 * h, f4 + ((long long)h * g.nvox() + voxels[i]) * 8,
                            8 * sizeof(__nv_bfloat16), cudaMemcpyDeviceToHost)) != cudaSuccess)
          return e;
      for (int c = 0; c < kC; ++c) features[i * kC + c] = __bfloat162float(tmp[c]);
    }
  }
  return cudaSuccess;
}

}  // namespace learned
}  // namespace pct
