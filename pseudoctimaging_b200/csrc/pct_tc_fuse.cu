// Tensor-core form (EXEC_CHOICE 5 = FP16, 6 = BF16): the SSD's cross term as a dense correlation
// on tcgen05, top-16 selection per (voxel, atlas), exact FP32 rescoring of the survivors.
//
// A CTA owns a tile of 4 (z) x 4 (x) x 8 (y) = 128 interior voxels (one tcgen05 row each; warp w
// holds the voxels of tile plane z = w, which is also its TMEM lane quarter) and loops over the
// atlases. The positions any of its voxels can be compared with form a 14 x 14 x 18 box; the
// correlation runs in 28 chunks of one z plane x 7 x-rows x 18 y (126 positions, N = 128):
//
//   A [128 voxels][32]   : the voxel's 27 input taps (v - mu) * s, then 1, 1 (, 1), then zeros
//   B [128 positions][32]: the position's 27 atlas taps (v - mu) * s, then -h, -l (, -t), zeros
//   D = A B^T (FP32, TMEM) = a.b - |b|^2/2   with |b|^2/2 = h + l (+ t) split over 16-bit parts
//
// mu is the tile's mean input intensity (the SSD does not change when both patches move by the
// same amount, and removing it keeps the 16-bit values small) and s = 1/64. |b|^2 is the FP32
// sum of squares of the already rounded taps, so D ranks the positions exactly by the SSD of the
// rounded patches, |a|^2 + |b|^2 - 2 a.b = |a - b|^2, up to FP32 accumulation; the cancellation
// the expanded form is known for stays out of the FP32 result. The 16 positions of largest D in
// each voxel's 11^3 window are kept, their SSD is recomputed from the FP32 volumes, and only they
// are weighted: out = sum w L / sum w over atlases, w = exp(-SSD/div), NaN rule as the plain path.
//
// Both operands are K-major without swizzling: core matrices of 8 rows x 16 bytes; row r's
// 16-byte group j sits at j * 2048 + r * 16 (leading-dimension offset 2048 between the two
// groups of one MMA's K = 16, stride-dimension offset 128 between 8-row groups).
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "pct_internal.h"
#include "pct_ptx.cuh"

namespace pct {
namespace tc {
namespace {

constexpr int kTZ = 4, kTX = 4, kTY = 8;       // voxel tile
constexpr int kPZ = 14, kPY = 18;              // position box (14 x 14 x 18)
constexpr int kRZ = 16, kRX = 16, kRY = 20;    // atlas region (positions + patch halo)
constexpr int kIZ = 6, kIX = 6, kIY = 10;      // input region (voxels + patch halo)
constexpr int kHalfX = 7;                      // x-rows per chunk
constexpr int kChunkPos = kHalfX * kPY;        // 126 positions per chunk
constexpr int kN = 128, kM = 128, kK = 32;
constexpr int kChunks = kPZ * 2;
constexpr int kTop = 16;
constexpr int kThreads = 128;
constexpr float kScale = 1.0f / 64.0f;
constexpr float kDblEpsilonF = 2.220446049250313080847e-16f;
constexpr unsigned long long kTimeoutNs = 2000000000ULL;

// shared memory map (bytes)
constexpr int kOffA = 0;                                   // 8 KB
constexpr int kOffB = kOffA + kM * kK * 2;                 // 8 KB
constexpr int kOffAtlas = kOffB + kN * kK * 2;             // 20 KB
constexpr int kOffInput = kOffAtlas + kRZ * kRX * kRY * 4;
constexpr int kStashStride = 33;                           // floats per lane row (no bank conflicts)
constexpr int kOffStash = kOffInput + kIZ * kIX * kIY * 4;
constexpr int kOffMisc = kOffStash + kThreads * kStashStride * 4;  // barrier, TMEM slot, flags
constexpr int kSmemUsed = kOffMisc + 256;
// at least 48 KB per CTA, so that at most 4 CTAs (4 x 128 TMEM columns) share an SM
constexpr int kSmemBytes = kSmemUsed > 49152 ? kSmemUsed : 49152;

struct Params {
  const float *img, *atlas, *label;
  float *out;
  int nx, ny, nz, num;
  int apitch;  // row pitch (floats) of the atlas MRI and CT stacks, >= ny
  int tiles_z, tiles_x, tiles_y;
  float neg_k;  // -log2(e) / div
  int *err;
  int16_t *dbg_top;  // optional: atlas 0's survivors per voxel [nvox][16], best first
};

// ------------------------------------------------------------------ tcgen05 wrappers

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
  // start >> 4 | LBO 2048 >> 4 | SBO 128 >> 4 | version 1 | no swizzle
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)(2048 >> 4) << 16) |
         ((uint64_t)(128 >> 4) << 32) | (1ull << 46);
}

template <bool BF16>
__device__ __forceinline__ uint32_t instr_desc() {
  const uint32_t fmt = BF16 ? 1u : 0u;
  return (1u << 4) | (fmt << 7) | (fmt << 10) | ((uint32_t)(kN >> 3) << 17) |
         ((uint32_t)(kM >> 4) << 24);
}

__device__ __forceinline__ void tmem_alloc(uint32_t slot_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot_smem),
               "r"(ncols)
               : "memory");
}

__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}

__device__ __forceinline__ void mma_f16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                        uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
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

// Writes one 32-element K-major row (27 taps + the extra columns) at row r of an operand.
__device__ __forceinline__ void store_row(unsigned char *op, int r, const uint32_t (&w)[16]) {
#pragma unroll
  for (int j = 0; j < 4; ++j)
    *reinterpret_cast<uint4 *>(op + j * 2048 + r * 16) =
        make_uint4(w[4 * j], w[4 * j + 1], w[4 * j + 2], w[4 * j + 3]);
}

// Inserts (val, id) into a descending top-16 held in registers (val beats the 16th).
__device__ __forceinline__ void insert_top(float (&tv)[kTop], int (&ti)[kTop], float val, int id) {
  float cur = val;
  int cid = id;
#pragma unroll
  for (int j = 0; j < kTop; ++j) {
    const bool sw = cur > tv[j];
    const float tvj = tv[j];
    const int tij = ti[j];
    tv[j] = sw ? cur : tvj;
    ti[j] = sw ? cid : tij;
    cur = sw ? tvj : cur;
    cid = sw ? tij : cid;
  }
}

// ------------------------------------------------------------------ the kernel

template <bool BF16>
__global__ void __launch_bounds__(kThreads, 4) tc_fuse_kernel(Params p) {
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char *opA = smem + kOffA;
  unsigned char *opB = smem + kOffB;
  float *areg = reinterpret_cast<float *>(smem + kOffAtlas);
  float *ireg = reinterpret_cast<float *>(smem + kOffInput);
  float *stash = reinterpret_cast<float *>(smem + kOffStash);
  unsigned char *misc = smem + kOffMisc;
  const uint32_t bar = ptx::smem_u32(misc);              // mbarrier (8 B)
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(misc + 8);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(misc + 12);
  float *red = reinterpret_cast<float *>(misc + 16);     // 4 floats: per-warp partial sums
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

  // tile
  int t = blockIdx.x;
  const int ty = t % p.tiles_y;
  t /= p.tiles_y;
  const int tx = t % p.tiles_x, tz = t / p.tiles_x;
  const int lo = 6;
  const int oz = lo + tz * kTZ, ox = lo + tx * kTX, oy = lo + ty * kTY;  // tile origin
  const int nxy = p.nx * p.ny;

  // this thread's voxel (row m = tid)
  const int vz = tid >> 5, vx = (tid >> 3) & 3, vy = tid & 7;
  const int gz = oz + vz, gx = ox + vx, gy = oy + vy;
  const bool valid = gz < p.nz - lo && gx < p.nx - lo && gy < p.ny - lo;

  if (warp == 0) {
    tmem_alloc(ptx::smem_u32(tmem_slot), kN);
    tmem_relinquish();
  }
  if (tid == 0) {
    ptx::mbar_init(bar, 1);
    *abort_flag = 0;
    ptx::fence_mbarrier_init();
  }
  // input region, zero outside the volume
  for (int i = tid; i < kIZ * kIX * kIY; i += kThreads) {
    const int z = oz - 1 + i / (kIX * kIY), x = ox - 1 + (i / kIY) % kIX, y = oy - 1 + i % kIY;
    ireg[i] = (z < p.nz && x < p.nx && y < p.ny) ? __ldg(p.img + (long long)z * nxy + (long long)x * p.ny + y) : 0.f;
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = *tmem_slot;

  // tile mean of the input region
  {
    float s = 0.f;
    for (int i = tid; i < kIZ * kIX * kIY; i += kThreads) s += ireg[i];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if (lane == 0) red[warp] = s;
  }
  __syncthreads();
  const float mu = (red[0] + red[1] + red[2] + red[3]) * (1.0f / (kIZ * kIX * kIY));

  // A row: the voxel's taps, then ones for the bias columns
  float in[27];
  {
    uint32_t w[16];
#pragma unroll
    for (int k = 0; k < 27; ++k) {
      in[k] = ireg[((vz + k / 9) * kIX + (vx + (k / 3) % 3)) * kIY + vy + k % 3];
    }
#pragma unroll
    for (int k = 0; k < 13; ++k)
      w[k] = pack2<BF16>((in[2 * k] - mu) * kScale, (in[2 * k + 1] - mu) * kScale);
    w[13] = pack2<BF16>((in[26] - mu) * kScale, 1.f);  // column 27: 1
    w[14] = pack2<BF16>(1.f, BF16 ? 1.f : 0.f);         // columns 28, 29
    w[15] = 0u;
    store_row(opA, tid, w);
  }

  // window masks: bit i of wmask[h][g] = column 32g + i of a chunk of half h lies in this
  // voxel's x/y window (the z test is per chunk)
  uint32_t wmask[2][4];
#pragma unroll
  for (int h = 0; h < 2; ++h)
#pragma unroll
    for (int g = 0; g < 4; ++g) {
      uint32_t m = 0;
#pragma unroll
      for (int i = 0; i < 32; ++i) {
        const int n = g * 32 + i;
        if (n >= kChunkPos) continue;
        const int px = h * kHalfX + n / kPY, py = n % kPY;
        if ((unsigned)(px - vx) <= 10u && (unsigned)(py - vy) <= 10u) m |= 1u << i;
      }
      wmask[h][g] = m;
    }

  float P = 0.f, W = 0.f;
  const uint32_t idesc = instr_desc<BF16>();
  const uint64_t a0 = smem_desc(ptx::smem_u32(opA)), a1 = smem_desc(ptx::smem_u32(opA) + 4096);
  const uint64_t b0 = smem_desc(ptx::smem_u32(opB)), b1 = smem_desc(ptx::smem_u32(opB) + 4096);
  const uint32_t my_tmem = tmem + ((uint32_t)(warp * 32) << 16);
  uint32_t phase = 0;
  bool aborted = false;

  for (int a = 0; a < p.num && !aborted; ++a) {
    const long long astride = (long long)p.nz * p.nx * p.apitch;
    const float *A = p.atlas + (long long)a * astride;
    // atlas region (positions and their patch halo), zero outside the volume
    __syncthreads();  // the previous atlas' rescoring is done with the region
    for (int i = tid; i < kRZ * kRX * kRY; i += kThreads) {
      const int z = oz - 6 + i / (kRX * kRY), x = ox - 6 + (i / kRY) % kRX, y = oy - 6 + i % kRY;
      areg[i] = (z >= 0 && z < p.nz && x >= 0 && x < p.nx && y >= 0 && y < p.ny)
                    ? __ldg(A + ((long long)z * p.nx + x) * p.apitch + y)
                    : 0.f;
    }
    float tv[kTop];
    int ti[kTop];
#pragma unroll
    for (int j = 0; j < kTop; ++j) {
      tv[j] = -INFINITY;
      ti[j] = 0;
    }
    for (int c = 0; c < kChunks; ++c) {
      // chunks from the box's centre plane outwards, so good candidates arrive early
      const int dzc = (c >> 1), pz = (dzc & 1) ? 7 - (dzc + 1) / 2 : 7 + dzc / 2;
      const int half = c & 1;
      __syncthreads();  // the region is loaded / the previous chunk's B and TMEM are consumed
      // B row: thread n builds position n of the chunk
      {
        uint32_t w[16];
        const int n = tid;
        if (n < kChunkPos) {
          const int px = half * kHalfX + n / kPY, py = n % kPY;
          float b[27];
          float s2 = 0.f;
#pragma unroll
          for (int k = 0; k < 27; ++k) {
            const float v = areg[((pz + k / 9) * kRX + (px + (k / 3) % 3)) * kRY + py + k % 3];
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
          w[14] = pack2<BF16>(-hl, BF16 ? -ht : 0.f);
          w[15] = 0u;
        } else {
#pragma unroll
          for (int k = 0; k < 16; ++k) w[k] = 0u;
        }
        store_row(opB, n, w);
      }
      ptx::fence_proxy_async_smem();
      fence_before_sync();
      __syncthreads();
      if (tid == 0) {
        fence_after_sync();
        mma_f16(tmem, a0, b0, idesc, 0u);
        mma_f16(tmem, a1, b1, idesc, 1u);
        mma_commit(bar);
      }
      if (!ptx::mbar_wait_bounded(bar, phase, kTimeoutNs)) *abort_flag = 1;
      phase ^= 1u;
      fence_after_sync();
      // this warp's voxels share z = warp; the chunk's plane is in their window iff
      // pz - 5 - warp in [-5, 5]
      const int dz = pz - 5 - vz;
      if (dz >= -5 && dz <= 5) {
#pragma unroll
        for (int g = 0; g < 4; ++g) {
          float v[32];
          tmem_ld32(my_tmem + g * 32, v);
          // columns of this group that are in the voxel's window and beat its 16th best
          const float thr = tv[kTop - 1];
          uint32_t m = 0;
#pragma unroll
          for (int i = 0; i < 32; ++i) m |= (v[i] > thr) ? (1u << i) : 0u;
          m &= half ? wmask[1][g] : wmask[0][g];
          if (__any_sync(0xffffffffu, m != 0u)) {
            // rare: park the group in shared memory and insert its candidates one by one
            float *row = stash + (warp * 32 + lane) * kStashStride;
#pragma unroll
            for (int i = 0; i < 32; ++i) row[i] = v[i];
            while (m) {
              const int i = __ffs(m) - 1;
              m &= m - 1;
              const float val = row[i];
              if (!(val > tv[kTop - 1])) continue;
              const int n = g * 32 + i;
              const int px = half * kHalfX + n / kPY, py = n % kPY;
              insert_top(tv, ti, val, ((dz + 5) * 11 + (px - vx)) * 11 + (py - vy));
            }
          }
        }
      }
      fence_before_sync();
      __syncthreads();
      if (*abort_flag) {
        aborted = true;
        break;
      }
    }
    if (aborted) break;
    // exact FP32 rescoring of the survivors from the FP32 region
    const float *L = p.label + (long long)a * astride;
#pragma unroll
    for (int j = 0; j < kTop; ++j) {
      const int o = ti[j];
      const int dz = o / 121 - 5, dx = (o / 11) % 11 - 5, dy = o % 11 - 5;
      // position (vz+dz, vx+dx, vy+dy) in box coordinates is +5 on each axis; region +6
      const int rz = vz + dz + 5, rx = vx + dx + 5, ry = vy + dy + 5;
      float ssd = 0.f;
#pragma unroll
      for (int k = 0; k < 27; ++k) {
        const float d = in[k] - areg[((rz + k / 9) * kRX + (rx + (k / 3) % 3)) * kRY + ry + k % 3];
        ssd = fmaf(d, d, ssd);
      }
      if (valid && tv[j] > -INFINITY) {
        const float w = ptx::ex2_approx(ssd * p.neg_k);
        P = fmaf(w, __ldg(L + ((long long)(gz + dz) * p.nx + gx + dx) * p.apitch + gy + dy), P);
        W += w;
      }
      if (a == 0 && p.dbg_top && valid)
        p.dbg_top[((long long)gz * nxy + (long long)gx * p.ny + gy) * kTop + j] = (int16_t)o;
    }
  }
  if (aborted) {
    if (tid == 0) {
      atomicExch(p.err, 4);
      ptx::mbar_wait_bounded(bar, phase ^ 1u, kTimeoutNs);  // the MMA in flight, if any
    }
  } else if (valid) {
    p.out[(long long)gz * nxy + (long long)gx * p.ny + gy] =
        (fabsf(P) > kDblEpsilonF && fabsf(W) > kDblEpsilonF) ? __fdiv_rn(P, W)
                                                            : __int_as_float(0x7fc00000);
  }
  fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    fence_after_sync();
    tmem_dealloc(tmem, kN);
  }
}

}  // namespace

cudaError_t launch_tc(const Geometry &g, const SlabInputs &in, float *out, double div, bool bf16,
                      int *err, int16_t *dbg_top, cudaStream_t s) {
  Params p;
  p.img = in.img;
  p.atlas = in.atlas;
  p.label = in.label;
  p.apitch = in.pitch;
  p.out = out;
  p.nx = g.nx;
  p.ny = g.ny;
  p.nz = g.nz;
  p.num = g.num;
  const int lo = 6;
  const int iz = g.nz - 2 * lo, ix = g.nx - 2 * lo, iy = g.ny - 2 * lo;
  if (iz <= 0 || ix <= 0 || iy <= 0) return cudaSuccess;
  p.tiles_z = (iz + kTZ - 1) / kTZ;
  p.tiles_x = (ix + kTX - 1) / kTX;
  p.tiles_y = (iy + kTY - 1) / kTY;
  p.neg_k = (float)(-1.4426950408889634 / div);
  p.err = err;
  p.dbg_top = dbg_top;
  const int blocks = p.tiles_z * p.tiles_x * p.tiles_y;
  cudaError_t e;
  if (bf16) {
    if ((e = cudaFuncSetAttribute(tc_fuse_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  kSmemBytes)) != cudaSuccess)
      return e;
    tc_fuse_kernel<true><<<blocks, kThreads, kSmemBytes, s>>>(p);
  } else {
    if ((e = cudaFuncSetAttribute(tc_fuse_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  kSmemBytes)) != cudaSuccess)
      return e;
    tc_fuse_kernel<false><<<blocks, kThreads, kSmemBytes, s>>>(p);
  }
  return cudaGetLastError();
}

}  // namespace tc
}  // namespace pct
