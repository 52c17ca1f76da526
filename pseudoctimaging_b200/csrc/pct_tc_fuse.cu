// Tensor-core form (EXEC_CHOICE 5 = FP16, 6 = BF16): the SSD's cross term as a dense correlation
// on tcgen05, top-16 selection per (voxel, atlas), exact FP32 rescoring of the survivors
// (reference arithmetic: PatchSimilarity and the window loop, NewPatchedBrainPureC.cpp:1184-1212,
// 1283-1331; the GPU kernel it stands beside computes the SSD directly in FP64,
// PatchBasedPseudoCT.cu:444-641).
//
// Operands (K = 32 per position or voxel, 16-bit, FP32 accumulation in TMEM):
//   B row (position p): its 27 atlas taps b = round16((A - mu) / 64), then -hh, -hl, -ht, 0,
//                       where hh + hl + ht = |b|^2 / 2 (FP32 sum of squares split in 16-bit parts)
//   A row (voxel v)   : its 27 input taps a = round16((I - mu) / 64), then 1, 1, 1, 0
//   D = A B^T = a.b - |b|^2 / 2, plus -|a|^2 / 2 (three 16-bit parts) through the penalty MMA
//   below, so D = -|a - b|^2 / 2: the positions rank by the SSD of the rounded patches up to FP32
//   accumulation, and the cancellation of the expanded form never reaches a subtraction in FP32.
//   mu is one integer per subject (the rounded mean of the input MRI), so every position's row
//   is computed once per atlas, not once per tile that sees it.
//
// Work: one launch per atlas. A CTA owns tiles of 4 (z) x 4 (x) x 8 (y) = 128 voxels (M = 128;
// warp w's TMEM lanes are the voxels of tile plane z = w) and is persistent over the tiles. The
// positions a tile's voxels compare with form a 14 x 14 x 18 box, run as 28 chunks of one plane
// x 7 x-rows x 18 y (126 positions, N = 128), centre planes first so that each voxel's 16th best
// rises early. Per chunk three MMAs (K = 16 each): the two halves of the taps, and a window
// penalty (A: the voxel's x and y one-hot times 60000, B: -60000 where the position is outside
// that x or y window), so out-of-window columns score about -3.6e9 and need no masking.
//
// Warp roles (192 threads): warps 0-3 select, rescore and write; warp 4 issues the TMA loads
// (B chunks through a 6-stage ring, the FP32 atlas region of each tile for the rescoring);
// warp 5 issues the MMAs into two TMEM accumulators of 128 columns, so the tensor core works on
// chunk c + 1 while chunk c is being read.
//
// Selection per warp and group of 32 columns: one tcgen05.ld, the maximum of the lane's 32
// scores (three-input max), a vote; in a group where some lane's maximum beats its 16th best,
// each column is voted on and the lanes it beats insert it into a sorted top-16 held in
// registers, whose keys carry the offset index in their 11 low mantissa bits (ties closer than
// 2^-12 relative are broken by that index).
//
// Every mbarrier wait is bounded (globaltimer); on expiry the CTA sets a status word, the others
// see an abort flag at their next wait, and the kernel reports PCT_ERR_TIMEOUT through the host.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "pct_internal.h"
#include "pct_ptx.cuh"

namespace pct {
namespace tc {
namespace {

constexpr int kTZ = 4, kTX = 4, kTY = 8;       // voxel tile
constexpr int kPZ = 14, kPY = 18;              // position box (14 x 14 x 18)
constexpr int kRZ = 16, kRX = 16, kRY = 20;    // FP32 atlas region (positions + patch halo)
constexpr int kHalfX = 7;                      // x-rows per chunk
constexpr int kChunkPos = kHalfX * kPY;        // 126 positions per chunk
constexpr int kChunks = kPZ * 2;
constexpr int kTop = 16;
constexpr int kEpi = 128;                      // selecting threads (warps 0-3)
constexpr int kThreads = 192;
constexpr int kStages = 6;
constexpr int kKg = kChunkPos * 16;            // bytes per 8-element K group of a chunk (2016)
constexpr int kSlot = 8192;                    // one chunk: 4 K groups (8064 B) + MMA overread
constexpr int kAKg = 128 * 16;                 // bytes per K group of the voxel operand
constexpr int kTmemCols = 256;                 // two accumulators
constexpr float kScale = 1.0f / 64.0f;
constexpr float kPenalty = 60000.0f;
// Below every in-window score (-|a - b|^2/2 of 16-bit patches stays above -1e9 for any MRI
// intensities up to ~10^5) and above every penalised one (about -3.6e9): the initial 16th best.
constexpr float kFloorScore = -1.0e9f;
// A later atlas's selection starts at this multiple of the lowest 16th best score of the voxel
// over the atlases before it (scores are -|a - b|^2/2 <= 0, so the start lies below it): the
// atlases of one subject differ little there, and a voxel whose own 16th best is lower sends its
// tile to the exact redo launch (1.08 of the previous atlas's value alone sent so many tiles
// there that the step took 380 ms instead of 209 ms on config 2; of the running minimum, margins
// 1.10 / 1.15 / 1.25 / 1.40 took 219.5 / 208.3 / 209.0 / 216.5 ms: fewer redos against fewer
// insertions, flat between 1.15 and 1.25).
constexpr float kWarmMargin = 1.25f;
constexpr float kDblEpsilonF = 2.220446049250313080847e-16f;
constexpr unsigned long long kTimeoutNs = 2000000000ULL;

// shared memory map (bytes from the 1024-aligned base)
constexpr int kOffSlots = 0;
constexpr int kOffA = kOffSlots + kStages * kSlot;          // [6 K groups][128 rows][16 B]
constexpr int kOffMask = kOffA + 6 * kAKg;                  // [2 halves][2 K groups][128][16 B]
constexpr int kOffRegion = kOffMask + 4 * kAKg;             // FP32 [16][16][20]
constexpr int kStashStride = 33;
constexpr int kOffStash = kOffRegion + kRZ * kRX * kRY * 4; // [128][33] floats
constexpr int kOffBars = kOffStash + kEpi * kStashStride * 4;
constexpr int kNumBars = 2 * kStages + 4 + 3;               // full, empty, tfull[2], tempty[2],
                                                            // a_ready, reg_full, reg_empty
constexpr int kOffMisc = kOffBars + 8 * kNumBars;           // TMEM slot, abort and redo flags
constexpr int kSmemBytes = kOffMisc + 16 + 1024;            // + alignment slack

struct Params {
  const float *img, *label;
  float *pacc, *wacc;
  int nx, ny, nz, atlas, apitch;
  int tiles_z, tiles_x, tiles_y, ntiles;
  float neg_k;        // -log2(e) / div
  const float *mu;    // device: the subject's offset
  int *err;
  int16_t *dbg_top;   // optional: this atlas's survivors per voxel [nvox][16], best first
  // Warm start: s16[v] holds the lowest 16th-best score of voxel v over the atlases done so far;
  // with `warm`, this atlas's selection starts from kWarmMargin x that value instead of -1e9. A
  // tile
  // where a voxel ends with fewer than 16 candidates above its start is not accumulated; it is
  // listed in redo_list for an exact second launch over that list (`list`, `list_count`).
  float *s16;
  int warm;
  const int *list, *list_count;  // null: every tile; else the tiles list[0 .. *list_count)
  int *redo_list, *redo_count;
};

__device__ __forceinline__ int tiles_of(const Params &p) {
  return p.list ? *p.list_count : p.ntiles;
}

__device__ __forceinline__ int tile_at(const Params &p, int i) { return p.list ? p.list[i] : i; }

// ------------------------------------------------------------------ tcgen05 wrappers

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo) {
  // K-major, no swizzle: start >> 4 | LBO >> 4 | SBO (8 rows x 16 B) >> 4 | version 1
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)(128 >> 4) << 32) | (1ull << 46);
}

template <bool BF16>
__device__ __forceinline__ uint32_t instr_desc() {
  const uint32_t fmt = BF16 ? 1u : 0u;  // D FP32; A, B FP16 or BF16, K-major; N = M = 128
  return (1u << 4) | (fmt << 7) | (fmt << 10) | ((uint32_t)(128 >> 3) << 17) |
         ((uint32_t)(128 >> 4) << 24);
}

// Issued by one elected lane of a converged warp.
__device__ __forceinline__ void mma_f16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                        uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred e, p;\n\telect.sync _|e, 0xffffffff;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "@e tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile(
      "{\n\t.reg .pred e;\n\telect.sync _|e, 0xffffffff;\n\t"
      "@e tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n\t}" ::"r"(
          bar)
      : "memory");
}

__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, "
      "%30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]),
        "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]),
        "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// 3-D tiled TMA load (no multicast) into this CTA's shared memory, completing on `bar`.
__device__ __forceinline__ void tma_load_4d(uint32_t dst, const CUtensorMap *map, uint32_t bar,
                                            int c0, int c1, int c2, int c3) {
  ptx::tma_load_4d(dst, map, bar, c0, c1, c2, c3);
}

// Barrier among the 128 selecting threads only (warps 0-3); the other warps never join it.
__device__ __forceinline__ void named_barrier_epilogue() {
  asm volatile("bar.sync 1, 128;" ::: "memory");
}

// ------------------------------------------------------------------ operand rows

template <bool BF16>
__device__ __forceinline__ uint32_t pack2(float a, float b) {
  if (BF16) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t *>(&h);
  } else {
    const __half2 h = __floats2half2_rn(a, b);
    return *reinterpret_cast<const uint32_t *>(&h);
  }
}

template <bool BF16>
__device__ __forceinline__ float round16(float a) {
  return BF16 ? __bfloat162float(__float2bfloat16_rn(a)) : __half2float(__float2half_rn(a));
}

__device__ __forceinline__ float max3f(float a, float b, float c) {
  float r;
  asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
}

// Maximum of 32 values: 16 three-input maxima, depth 4.
__device__ __forceinline__ float max32(const float (&v)[32]) {
  float t[10];
#pragma unroll
  for (int k = 0; k < 10; ++k) t[k] = max3f(v[3 * k], v[3 * k + 1], v[3 * k + 2]);
  const float u0 = max3f(t[0], t[1], t[2]), u1 = max3f(t[3], t[4], t[5]);
  const float u2 = max3f(t[6], t[7], t[8]), u3 = max3f(t[9], v[30], v[31]);
  return fmaxf(max3f(u0, u1, u2), u3);
}

// Inserts key into a descending top-16 of packed keys (key beats the 16th).
__device__ __forceinline__ void insert_key(float (&tv)[kTop], float key) {
#pragma unroll
  for (int j = 0; j < kTop; ++j) {
    const float hi = fmaxf(tv[j], key);
    key = fminf(tv[j], key);
    tv[j] = hi;
  }
}

__device__ __forceinline__ float pack_key(float score, int offset) {
  return __int_as_float((__float_as_int(score) & ~0x7FF) | offset);
}

// ------------------------------------------------------------------ the features of one atlas

// feat: [4 K groups][nz][nx][ny] x 16 bytes (8 elements): the B rows of every position whose 3^3
// patch lies inside the volume; zero rows elsewhere (never read by a window of an interior voxel).
template <bool BF16>
__global__ void features_kernel(const float *__restrict__ atl, int nx, int ny, int nz, int apitch,
                                const float *__restrict__ mu_ptr, uint4 *__restrict__ feat) {
  const long long nvox = (long long)nx * ny * nz;
  const float mu = *mu_ptr;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nvox;
       i += (long long)gridDim.x * blockDim.x) {
    const int y = (int)(i % ny);
    const long long r = i / ny;
    const int x = (int)(r % nx), z = (int)(r / nx);
    uint32_t w[16];
    if (z >= 1 && z < nz - 1 && x >= 1 && x < nx - 1 && y >= 1 && y < ny - 1) {
      float b[27];
      float s2 = 0.f;
#pragma unroll
      for (int k = 0; k < 27; ++k) {
        const float v = __ldg(atl + ((long long)(z - 1 + k / 9) * nx + (x - 1 + (k / 3) % 3)) *
                                        apitch + (y - 1 + k % 3));
        b[k] = round16<BF16>((v - mu) * kScale);
        s2 = fmaf(b[k], b[k], s2);
      }
      const float h = 0.5f * s2;
      const float hh = round16<BF16>(h);
      const float hl = round16<BF16>(h - hh);
      const float ht = round16<BF16>(h - hh - hl);
#pragma unroll
      for (int k = 0; k < 13; ++k) w[k] = pack2<BF16>(b[2 * k], b[2 * k + 1]);
      w[13] = pack2<BF16>(b[26], -hh);
      w[14] = pack2<BF16>(-hl, -ht);
      w[15] = 0u;
    } else {
#pragma unroll
      for (int k = 0; k < 16; ++k) w[k] = 0u;
    }
#pragma unroll
    for (int j = 0; j < 4; ++j)
      feat[(long long)j * nvox + i] = make_uint4(w[4 * j], w[4 * j + 1], w[4 * j + 2], w[4 * j + 3]);
  }
}

// mu = rint(mean of the input MRI), FP32, fixed summation order (one block of 1024 threads:
// thread t sums elements t, t + 1024, ... in order, then a halving tree in shared memory).
__global__ void __launch_bounds__(1024) mean_kernel(const float *__restrict__ img, long long n,
                                                    float *__restrict__ mu) {
  __shared__ float part[1024];
  float s = 0.f;
  long long i = threadIdx.x;
  for (; i + 7 * 1024 < n; i += 8 * 1024) {  // eight loads in flight, the same summation order
    float v[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) v[j] = __ldg(img + i + j * 1024);
#pragma unroll
    for (int j = 0; j < 8; ++j) s += v[j];
  }
  for (; i < n; i += 1024) s += img[i];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int h = 512; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) part[threadIdx.x] += part[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) *mu = rintf(part[0] / (float)n);
}

__global__ void finalize_kernel(const float *__restrict__ pacc, const float *__restrict__ wacc,
                                float *__restrict__ out, int nx, int ny, int nz) {
  const int lo = 6;
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

// ------------------------------------------------------------------ the correlation kernel

// Chunk c of a tile: plane pz of the box (centre planes first) and half h of its x-rows.
__device__ __forceinline__ void chunk_of(int c, int &pz, int &half) {
  const int dzc = c >> 1;
  pz = (dzc & 1) ? 7 - (dzc + 1) / 2 : 7 + dzc / 2;
  half = c & 1;
}

struct Bars {
  uint32_t full, empty, tfull, tempty, a_ready, reg_full, reg_empty;
};

template <bool BF16>
__global__ void __launch_bounds__(kThreads, 2)
    tc_fuse_kernel(const __grid_constant__ CUtensorMap tm_feat,
                   const __grid_constant__ CUtensorMap tm_atlas, const Params p) {
  extern __shared__ unsigned char smem_raw[];
  const uint32_t raw = ptx::smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  unsigned char *sbase = smem_raw + (base - raw);
  const uint32_t slots = base + kOffSlots, opA = base + kOffA, opM = base + kOffMask;
  float *region = reinterpret_cast<float *>(sbase + kOffRegion);
  Bars bar;
  bar.full = base + kOffBars;
  bar.empty = bar.full + 8 * kStages;
  bar.tfull = bar.empty + 8 * kStages;
  bar.tempty = bar.tfull + 16;
  bar.a_ready = bar.tempty + 16;
  bar.reg_full = bar.a_ready + 8;
  bar.reg_empty = bar.reg_full + 8;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(sbase + kOffMisc);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(sbase + kOffMisc + 4);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int lo = 6;

  if (tid == 0) {
    for (int i = 0; i < kStages; ++i) {
      ptx::mbar_init(bar.full + 8 * i, 1);
      ptx::mbar_init(bar.empty + 8 * i, 1);
    }
    for (int i = 0; i < 2; ++i) {
      ptx::mbar_init(bar.tfull + 8 * i, 1);
      ptx::mbar_init(bar.tempty + 8 * i, kEpi);
    }
    ptx::mbar_init(bar.a_ready, kEpi);
    ptx::mbar_init(bar.reg_full, 1);
    ptx::mbar_init(bar.reg_empty, kEpi);
    *abort_flag = 0;
    abort_flag[1] = 0;  // the redo flag of the tile being selected
    ptx::fence_mbarrier_init();
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     ptx::smem_u32(tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  for (int i = tid; i < kStages * (kSlot - 4 * kKg) / 16; i += kThreads) {
    const int per = (kSlot - 4 * kKg) / 16;
    *reinterpret_cast<uint4 *>(sbase + kOffSlots + (i / per) * kSlot + 4 * kKg + (i % per) * 16) =
        make_uint4(0u, 0u, 0u, 0u);
  }
  // the window penalty operand (constant): half h, row n, columns 0-3 the x one-hots of the
  // voxel operand, 4-11 the y one-hots
  if (tid < kEpi) {
    for (int h = 0; h < 2; ++h) {
      const int n = tid;
      const int px = h * kHalfX + n / kPY, py = n % kPY;
      float m[16];
#pragma unroll
      for (int c = 0; c < 16; ++c) m[c] = c >= 12 && c < 15 ? 1.f : 0.f;  // -|a|^2/2 columns
#pragma unroll
      for (int c = 0; c < 4; ++c)
        if (n >= kChunkPos || (unsigned)(px - c) > 10u) m[c] = -kPenalty;
#pragma unroll
      for (int c = 0; c < 8; ++c)
        if (n >= kChunkPos || (unsigned)(py - c) > 10u) m[4 + c] = -kPenalty;
      for (int j = 0; j < 2; ++j)
        *reinterpret_cast<uint4 *>(sbase + kOffMask + (h * 2 + j) * kAKg + n * 16) =
            make_uint4(pack2<BF16>(m[8 * j], m[8 * j + 1]), pack2<BF16>(m[8 * j + 2], m[8 * j + 3]),
                       pack2<BF16>(m[8 * j + 4], m[8 * j + 5]),
                       pack2<BF16>(m[8 * j + 6], m[8 * j + 7]));
    }
  }
  ptx::fence_proxy_async_smem();
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = *tmem_slot;
  const int nxy = p.nx * p.ny;

  if (warp == 4) {
    // ---------------- TMA producer
    if (lane == 0) {
      uint32_t g = 0;  // chunks issued
      int k = 0;       // tiles started by this CTA
      const int n_tiles = tiles_of(p);
      for (int i = blockIdx.x; i < n_tiles && !*abort_flag; i += gridDim.x, ++k) {
        const int t = tile_at(p, i);
        const int ty = t % p.tiles_y, r = t / p.tiles_y;
        const int tx = r % p.tiles_x, tz = r / p.tiles_x;
        const int oz = lo + tz * kTZ, ox = lo + tx * kTX, oy = lo + ty * kTY;
        for (int c = 0; c < kChunks; ++c, ++g) {
          if (c == kStages) {
            // the FP32 region of this tile, once the previous tile's rescoring released it
            if (k > 0 && !ptx::mbar_wait_bounded(bar.reg_empty, (k - 1) & 1, kTimeoutNs)) {
              *abort_flag = 1;
              atomicExch(p.err, 4);
              break;
            }
            ptx::mbar_arrive_expect_tx(bar.reg_full, kRZ * kRX * kRY * 4);
            tma_load_4d(base + kOffRegion, &tm_atlas, bar.reg_full, oy - 6, ox - 6, oz - 6, p.atlas);
          }
          const uint32_t s = g % kStages;
          if (g >= kStages &&
              !ptx::mbar_wait_bounded(bar.empty + 8 * s, ((g / kStages) - 1) & 1, kTimeoutNs)) {
            *abort_flag = 1;
            atomicExch(p.err, 4);
            break;
          }
          int pz, half;
          chunk_of(c, pz, half);
          ptx::mbar_arrive_expect_tx(bar.full + 8 * s, 4 * kKg);
          tma_load_4d(slots + s * kSlot, &tm_feat, bar.full + 8 * s, 2 * (oy - 5),
                      ox - 5 + half * kHalfX, oz - 5 + pz, 0);
        }
      }
      // copies still landing (only after an abort are any of them unconsumed): wait for the last
      // load of every slot and for the last region, bounded, before the CTA may exit
      for (uint32_t q = g > kStages ? g - kStages : 0; q < g; ++q)
        ptx::mbar_wait_bounded(bar.full + 8 * (q % kStages), (q / kStages) & 1, kTimeoutNs);
      if (k > 0) ptx::mbar_wait_bounded(bar.reg_full, (k - 1) & 1, kTimeoutNs);
    }
  } else if (warp == 5) {
    // ---------------- MMA issuer (the whole warp runs the loop; one elected lane issues)
    const uint32_t idesc = instr_desc<BF16>();
    uint32_t g = 0, u = 0;
    int k = 0;
    bool stop = false;
    const int n_tiles = tiles_of(p);
    for (int i = blockIdx.x; i < n_tiles && !stop; i += gridDim.x, ++k) {
      const bool a_ok = ptx::mbar_wait_bounded(bar.a_ready, k & 1, kTimeoutNs);
      if (!__all_sync(0xffffffffu, a_ok && !*abort_flag)) {
        if (lane == 0) {
          *abort_flag = 1;
          atomicExch(p.err, 4);
        }
        break;
      }
      for (int c = 0; c < kChunks; ++c, ++g, ++u) {
        const uint32_t s = g % kStages, b = u & 1;
        const bool ok =
            ptx::mbar_wait_bounded(bar.full + 8 * s, (g / kStages) & 1, kTimeoutNs) &&
            (u < 2 || ptx::mbar_wait_bounded(bar.tempty + 8 * b, ((u >> 1) - 1) & 1, kTimeoutNs));
        if (!__all_sync(0xffffffffu, ok && !*abort_flag)) {
          if (lane == 0) {
            *abort_flag = 1;
            atomicExch(p.err, 4);
          }
          stop = true;
          break;
        }
        fence_after_sync();
        int pz, half;
        chunk_of(c, pz, half);
        const uint32_t d = tmem + b * 128;
        const uint32_t bs = slots + s * kSlot;
        mma_f16(d, smem_desc(opA, kAKg), smem_desc(bs, kKg), idesc, 0u);
        mma_f16(d, smem_desc(opA + 2 * kAKg, kAKg), smem_desc(bs + 2 * kKg, kKg), idesc, 1u);
        mma_f16(d, smem_desc(opA + 4 * kAKg, kAKg), smem_desc(opM + half * 2 * kAKg, kAKg), idesc,
                1u);
        mma_commit(bar.empty + 8 * s);
        mma_commit(bar.tfull + 8 * b);
      }
    }
    // after an abort: let the MMAs already issued finish before the accumulators are freed
    if (u > 0 && *abort_flag)
      ptx::mbar_wait_bounded(bar.tfull + 8 * ((u - 1) & 1), ((u - 1) >> 1) & 1, kTimeoutNs);
  } else {
    // ---------------- selection, rescoring and output (warps 0-3, voxel m = tid)
    const int m = tid, vz = m >> 5, vx = (m >> 3) & 3, vy = m & 7;
    const float mu = *p.mu;
    const uint32_t my_tmem = tmem + ((uint32_t)(warp * 32) << 16);
    const float *L = p.label + (long long)p.atlas * p.nz * p.nx * p.apitch;
    uint32_t u = 0;
    int k = 0;
    bool stop = false;
    float in[27];
    // the first tile's voxel operand
    auto build_a = [&](int t, float (&taps)[27]) {
      const int ty = t % p.tiles_y, r = t / p.tiles_y;
      const int tx = r % p.tiles_x, tz = r / p.tiles_x;
      const int gz = lo + tz * kTZ + vz, gx = lo + tx * kTX + vx, gy = lo + ty * kTY + vy;
#pragma unroll
      for (int q = 0; q < 27; ++q) {
        const int z = gz - 1 + q / 9, x = gx - 1 + (q / 3) % 3, y = gy - 1 + q % 3;
        taps[q] = (z < p.nz && x < p.nx && y < p.ny)
                      ? __ldg(p.img + (long long)z * nxy + (long long)x * p.ny + y)
                      : 0.f;
      }
      uint32_t w[24];
      float ar[27];
      float s2 = 0.f;
#pragma unroll
      for (int q = 0; q < 27; ++q) {
        ar[q] = round16<BF16>((taps[q] - mu) * kScale);
        s2 = fmaf(ar[q], ar[q], s2);
      }
#pragma unroll
      for (int q = 0; q < 13; ++q) w[q] = pack2<BF16>(ar[2 * q], ar[2 * q + 1]);
      w[13] = pack2<BF16>(ar[26], 1.f);
      w[14] = pack2<BF16>(1.f, 1.f);
      w[15] = 0u;
      // |a|^2/2 in three 16-bit parts, subtracted through the penalty MMA: the accumulated score
      // is then -|a - b|^2/2 itself, small, so that packing offsets into its low bits costs
      // nothing of the ranking
      const float ha = 0.5f * s2;
      const float hh = round16<BF16>(ha);
      const float hl = round16<BF16>(ha - hh);
      const float ht = round16<BF16>(ha - hh - hl);
      float oh[16];
#pragma unroll
      for (int c = 0; c < 16; ++c) oh[c] = 0.f;
      oh[12] = -hh;
      oh[13] = -hl;
      oh[14] = -ht;
#pragma unroll
      for (int c = 0; c < 4; ++c)
        if (c == vx) oh[c] = kPenalty;
#pragma unroll
      for (int c = 0; c < 8; ++c)
        if (c == vy) oh[4 + c] = kPenalty;
#pragma unroll
      for (int q = 0; q < 8; ++q) w[16 + q] = pack2<BF16>(oh[2 * q], oh[2 * q + 1]);
#pragma unroll
      for (int j = 0; j < 6; ++j)
        *reinterpret_cast<uint4 *>(sbase + kOffA + j * kAKg + m * 16) =
            make_uint4(w[4 * j], w[4 * j + 1], w[4 * j + 2], w[4 * j + 3]);
      ptx::fence_proxy_async_smem();
      ptx::mbar_arrive(bar.a_ready);
    };
    float *row = reinterpret_cast<float *>(sbase + kOffStash) + m * kStashStride;
    volatile int *redo_flag = abort_flag + 1;
    const int n_tiles = tiles_of(p);
    if ((int)blockIdx.x < n_tiles) build_a(tile_at(p, blockIdx.x), in);
    for (int i = blockIdx.x; i < n_tiles && !stop; i += gridDim.x, ++k) {
      const int t = tile_at(p, i);
      const int ty = t % p.tiles_y, r = t / p.tiles_y;
      const int tx = r % p.tiles_x, tz = r / p.tiles_x;
      const int gz = lo + tz * kTZ + vz, gx = lo + tx * kTX + vx, gy = lo + ty * kTY + vy;
      const bool valid = gz < p.nz - lo && gx < p.nx - lo && gy < p.ny - lo;
      const long long vox = (long long)gz * nxy + (long long)gx * p.ny + gy;
      // the selection's start: the 16th best found so far must beat it
      const float start = (p.warm && valid) ? kWarmMargin * p.s16[vox] : kFloorScore;
      float tv[kTop];
#pragma unroll
      for (int j = 0; j < kTop; ++j) tv[j] = start;
      for (int c = 0; c < kChunks; ++c, ++u) {
        const uint32_t b = u & 1;
        const bool ok = ptx::mbar_wait_bounded(bar.tfull + 8 * b, (u >> 1) & 1, kTimeoutNs);
        if (!__all_sync(0xffffffffu, ok && !*abort_flag)) {
          if (lane == 0) {
            *abort_flag = 1;
            atomicExch(p.err, 4);
          }
          stop = true;
          break;
        }
        fence_after_sync();
        int pz, half;
        chunk_of(c, pz, half);
        const int dz = pz - 5 - vz;  // this warp's voxels share z: the plane is in their window
        if (dz >= -5 && dz <= 5) {   // iff |dz| <= 5 (warp-uniform)
#pragma unroll 1
          for (int grp = 0; grp < 4; ++grp) {
            float v[32];
            tmem_ld32(my_tmem + b * 128 + grp * 32, v);
            const float thr = tv[kTop - 1];
            if (__any_sync(0xffffffffu, max32(v) > thr)) {
              // each lane walks its own columns above its 16th best (parked in shared memory,
              // so that the lanes need not agree on a column): the warp loops as often as its
              // busiest lane has candidates, not once per column any lane wants
              uint32_t msk = 0;
#pragma unroll
              for (int q = 0; q < 32; ++q) {
                msk |= (v[q] > thr ? 1u : 0u) << q;
                row[q] = v[q];
              }
              while (__any_sync(0xffffffffu, msk != 0u)) {
                if (msk) {
                  const int q = __ffs(msk) - 1;
                  msk &= msk - 1;
                  const float val = row[q];
                  if (val > tv[kTop - 1]) {
                    const int n = grp * 32 + q;
                    const int px = half * kHalfX + n / kPY, py = n % kPY;
                    insert_key(tv, pack_key(val, ((dz + 5) * 11 + (px - vx)) * 11 + (py - vy)));
                  }
                }
              }
            }
          }
        }
        fence_before_sync();
        ptx::mbar_arrive(bar.tempty + 8 * b);
      }
      if (stop) break;
      // the MMAs of this tile are complete (its last accumulator was read): the next tile's
      // voxel operand may replace this one while this tile is rescored
      float nin[27];
      const int inext = i + gridDim.x;
      if (inext < n_tiles) build_a(tile_at(p, inext), nin);
      // a voxel whose start held back part of its 16 sends the tile to the exact redo launch
      const bool short_list = p.warm && valid && !(tv[kTop - 1] > start);
      if (short_list) *redo_flag = 1;
      named_barrier_epilogue();
      const bool redo = *redo_flag != 0;
      // exact FP32 rescoring of the survivors from the FP32 region
      if (!ptx::mbar_wait_bounded(bar.reg_full, k & 1, kTimeoutNs)) {
        *abort_flag = 1;
        atomicExch(p.err, 4);
        break;
      }
      float P = 0.f, W = 0.f;
      if (!redo) {
#pragma unroll
        for (int j = 0; j < kTop; ++j) {  // unrolled: the top-16 must stay in registers
          const int o = __float_as_int(tv[j]) & 0x7FF;
          // an entry never replaced (only inputs whose 16-bit scores leave (-1e9, 1e9) can
          // leave one) holds no offset
          if (!(tv[j] > kFloorScore) || o > 1330) continue;
          const int dzz = o / 121 - 5, dx = (o / 11) % 11 - 5, dy = o % 11 - 5;
          // position (vz + dz, vx + dx, vy + dy) + 5 in box coordinates; the region starts at -6
          const int rz = vz + dzz + 5, rx = vx + dx + 5, ry = vy + dy + 5;
          float ssd = 0.f;
#pragma unroll
          for (int q = 0; q < 27; ++q) {
            const float d =
                in[q] - region[((rz + q / 9) * kRX + (rx + (q / 3) % 3)) * kRY + ry + q % 3];
            ssd = fmaf(d, d, ssd);
          }
          if (valid) {
            const float w = ptx::ex2_approx(ssd * p.neg_k);
            P = fmaf(w, __ldg(L + ((long long)(gz + dzz) * p.nx + gx + dx) * p.apitch + gy + dy),
                     P);
            W += w;
            if (p.dbg_top) p.dbg_top[vox * kTop + j] = (int16_t)o;
          }
        }
      }
      ptx::mbar_arrive(bar.reg_empty);
      if (redo) {
        if (m == 0) p.redo_list[atomicAdd(p.redo_count, 1)] = t;
      } else if (valid) {
        p.pacc[vox] += P;
        p.wacc[vox] += W;
        // the lowest 16th best so far: the next atlas starts below it
        const float s16v = __int_as_float(__float_as_int(tv[kTop - 1]) & ~0x7FF);
        p.s16[vox] = (p.warm || p.list) ? fminf(p.s16[vox], s16v) : s16v;
      }
      named_barrier_epilogue();  // every lane has read the flag: it may be cleared
      if (m == 0) *redo_flag = 0;
#pragma unroll
      for (int q = 0; q < 27; ++q) in[q] = nin[q];
    }
  }
  fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    fence_after_sync();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTmemCols)
                 : "memory");
  }
}

// ------------------------------------------------------------------ host side

// [4 K groups][nz][nx][ny] x 16 B, addressed in 8-byte elements (2 per position); one box = one
// chunk: 18 y x 7 x-rows x 1 plane x 4 K groups (8,064 bytes).
cudaError_t make_feature_map(CUtensorMap *map, const void *feat, const Geometry &g) {
  auto fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(tensor_map_encoder());
  if (!fn) return cudaErrorNotSupported;
  const cuuint64_t dims[4] = {2 * (cuuint64_t)g.ny, (cuuint64_t)g.nx, (cuuint64_t)g.nz, 4};
  const cuuint64_t strides[3] = {16 * (cuuint64_t)g.ny, 16 * (cuuint64_t)g.ny * g.nx,
                                 16 * (cuuint64_t)g.nvox()};
  const cuuint32_t box[4] = {2 * kPY, (cuuint32_t)kHalfX, 1, 4};
  const cuuint32_t estr[4] = {1u, 1u, 1u, 1u};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, const_cast<void *>(feat), dims, strides,
                  box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

// The pitched FP32 atlas MRI stack [num][nz][nx][pitch]; one box = a tile's region 20 y x 16 x x
// 16 z of one atlas, out-of-volume elements zero.
cudaError_t make_region_map(CUtensorMap *map, const float *atlas, const Geometry &g, int pitch) {
  auto fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(tensor_map_encoder());
  if (!fn) return cudaErrorNotSupported;
  const cuuint64_t dims[4] = {(cuuint64_t)g.ny, (cuuint64_t)g.nx, (cuuint64_t)g.nz,
                              (cuuint64_t)g.num};
  const cuuint64_t strides[3] = {(cuuint64_t)pitch * 4, (cuuint64_t)pitch * 4 * g.nx,
                                 (cuuint64_t)pitch * 4 * g.nx * g.nz};
  const cuuint32_t box[4] = {kRY, kRX, kRZ, 1};
  const cuuint32_t estr[4] = {1u, 1u, 1u, 1u};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<float *>(atlas), dims, strides,
                  box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

int sm_count() {
  int dev = 0, n = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  return n;
}

struct Scratch {
  uint4 *feat;
  float *pacc, *wacc, *mu, *s16;
  int *redo_count, *redo_list;
};

Scratch carve(void *scratch, const Geometry &g) {
  const long long nvox = g.nvox();
  unsigned char *sc = static_cast<unsigned char *>(scratch);
  Scratch r;
  r.feat = reinterpret_cast<uint4 *>(sc);
  r.pacc = reinterpret_cast<float *>(sc + 64 * (size_t)nvox);
  r.wacc = r.pacc + nvox;
  r.s16 = r.wacc + nvox;
  r.mu = r.s16 + nvox;                                   // 16 bytes
  r.redo_count = reinterpret_cast<int *>(r.mu + 4);      // 16 bytes
  r.redo_list = r.redo_count + 4;
  return r;
}

int num_tiles(const Geometry &g) {
  if (g.ix <= 0 || g.iy <= 0 || g.iz <= 0) return 0;
  return ((g.iz + kTZ - 1) / kTZ) * ((g.ix + kTX - 1) / kTX) * ((g.iy + kTY - 1) / kTY);
}

template <bool BF16>
cudaError_t launch_all(const Geometry &g, const SlabInputs &in, float *out, double div, int *err,
                       int16_t *dbg_top, void *scratch, cudaStream_t s) {
  const long long nvox = g.nvox();
  const Scratch sc = carve(scratch, g);
  cudaError_t e;
  if ((e = cudaMemsetAsync(sc.pacc, 0, 8 * (size_t)nvox, s)) != cudaSuccess) return e;
  mean_kernel<<<1, 1024, 0, s>>>(in.img, nvox, sc.mu);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  CUtensorMap tm_feat, tm_atlas;
  if ((e = make_feature_map(&tm_feat, sc.feat, g)) != cudaSuccess) return e;
  if ((e = make_region_map(&tm_atlas, in.atlas, g, in.pitch)) != cudaSuccess) return e;
  auto kern = tc_fuse_kernel<BF16>;
  if ((e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes)) !=
      cudaSuccess)
    return e;
  Params p{};
  p.img = in.img;
  p.label = in.label;
  p.pacc = sc.pacc;
  p.wacc = sc.wacc;
  p.nx = g.nx;
  p.ny = g.ny;
  p.nz = g.nz;
  p.apitch = in.pitch;
  p.tiles_z = (g.iz + kTZ - 1) / kTZ;
  p.tiles_x = (g.ix + kTX - 1) / kTX;
  p.tiles_y = (g.iy + kTY - 1) / kTY;
  p.ntiles = p.tiles_z * p.tiles_x * p.tiles_y;
  p.neg_k = (float)(-1.4426950408889634 / div);
  p.mu = sc.mu;
  p.err = err;
  p.s16 = sc.s16;
  p.redo_list = sc.redo_list;
  p.redo_count = sc.redo_count;
  const int blocks = std::min(p.ntiles, 2 * sm_count());
  const long long astride = (long long)g.nz * g.nx * in.pitch;
  for (int a = 0; a < g.num; ++a) {
    features_kernel<BF16><<<sm_count() * 8, 256, 0, s>>>(in.atlas + a * astride, g.nx, g.ny, g.nz,
                                                         in.pitch, sc.mu, sc.feat);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(sc.redo_count, 0, sizeof(int), s)) != cudaSuccess) return e;
    p.atlas = a;
    p.dbg_top = a == 0 ? dbg_top : nullptr;
    // atlas 0 selects from scratch; later atlases start from their voxels' 16th best so far
    p.warm = a > 0;
    p.list = p.list_count = nullptr;
    kern<<<blocks, kThreads, kSmemBytes, s>>>(tm_feat, tm_atlas, p);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (a > 0) {  // the tiles whose start was too high, exactly (count read on the device)
      Params q = p;
      q.warm = 0;
      q.list = sc.redo_list;
      q.list_count = sc.redo_count;
      kern<<<blocks, kThreads, kSmemBytes, s>>>(tm_feat, tm_atlas, q);
      if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
  }
  finalize_kernel<<<sm_count() * 8, 256, 0, s>>>(sc.pacc, sc.wacc, out, g.nx, g.ny, g.nz);
  return cudaGetLastError();
}

}  // namespace

size_t scratch_bytes(const Geometry &g) {
  return 76 * (size_t)g.nvox() + 32 + 4 * (size_t)num_tiles(g) + 256;
}

cudaError_t launch_tc(const Geometry &g, const SlabInputs &in, float *out, double div, bool bf16,
                      int *err, int16_t *dbg_top, void *scratch, cudaStream_t s) {
  if (g.ix <= 0 || g.iy <= 0 || g.iz <= 0) return cudaSuccess;
  if (g.hw != 5 || in.pitch % 4 != 0 || reinterpret_cast<uintptr_t>(in.atlas) % 16 != 0)
    return cudaErrorInvalidValue;
  return bf16 ? launch_all<true>(g, in, out, div, err, dbg_top, scratch, s)
              : launch_all<false>(g, in, out, div, err, dbg_top, scratch, s);
}

}  // namespace tc
}  // namespace pct
