// Plain FP32 patch-based multi-atlas fusion for sm_100a.
//
// Computes, for every interior voxel x of the input MRI I and every candidate offset d in the
// NH^3 window of every atlas a (reference: MultiAtlasPatchBasedSegmentationOpenMP and
// PatchSimilarity, NewPatchedBrainPureC.cpp:1184-1212,1350-1449):
//     SSD(x,d) = sum_{p in 3x3x3} (I(x+p) - A_a(x+d+p))^2
//     w        = exp(-SSD/div)
//     out(x)   = sum w*L_a(x+d) / sum w     (NaN unless both sums exceed DBL_EPSILON)
//
// Design (one warp = one tile of 30 (y) x RX (x) x 2*TZ (z) output voxels):
//  * Lanes run along the contiguous y axis; lanes 1..30 own outputs, lanes 0 and 31 carry the
//    y-halo. For a fixed offset d, SSD is a 3x3x3 box sum of D_d(u) = (I(u)-A(u+d))^2. Each lane
//    box-sums along x and z in registers (its RX+2 rows x TZ+2 planes) and the y-box is two warp
//    shuffles of the finished x/z sums, so every D element is computed once per lane.
//  * The two z-halves of a thread (planes z0..z0+TZ-1 and z0+TZ..z0+2TZ-1) are packed into
//    float2 and processed with sm_100's paired FP32 instructions (add/mul/fma .f32x2), halving
//    the instruction count of the D, box and accumulate steps.
//  * Offsets are walked with dw (z) innermost. Stepping dw by one shifts the atlas planes the
//    tile needs by one, so the atlas window (TZ+2 planes x RX+2 rows) and the CT window (TZ x RX)
//    live in registers as ring buffers and each dw step loads only one new plane.
//  * exp(-SSD/div) = 2^(SSD * -log2(e)/div) on the MUFU ex2 unit; the weight sum and the
//    weighted CT sum stay in FP32 registers across all atlases and offsets.
#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

#include "pct_internal.h"

namespace pct {
namespace {

constexpr int kOutY = 30;                     // outputs per warp along y
constexpr float kDblEpsilonF = 2.220446049250313080847e-16f;  // DBL_EPSILON, exact in float

__device__ __forceinline__ float ex2_approx(float x) {
  float r;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

// Output rule of NewPatchedBrainPureC.cpp:1325-1331 in FP32: product/sum_weight when both
// exceed DBL_EPSILON in magnitude, else NaN (the C NAN bit pattern).
__device__ __forceinline__ float fuse_result(float product, float sum_weight) {
  return (fabsf(product) > kDblEpsilonF && fabsf(sum_weight) > kDblEpsilonF)
             ? __fdiv_rn(product, sum_weight)
             : __int_as_float(0x7fc00000);
}

struct FuseParams {
  const float *img;
  const float *atlas;
  const float *label;
  float *out;
  int nx, ny, nz, num;
  int nxy;
  long long nvox;
  float neg_k;  // -log2(e) / div
  int tiles_y, tiles_x, tiles_z;
};

template <int HW, int RX, int TZ>
__global__ void __launch_bounds__(128) fuse_plain_kernel(const FuseParams p) {
  constexpr int NQ = TZ + 2;  // D planes per half
  constexpr int NR = RX + 2;  // D rows
  constexpr int NS = 2 * HW + 1;
  const int lane = threadIdx.x & 31;
  int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (t >= p.tiles_y * p.tiles_x * p.tiles_z) return;  // warp-uniform
  const int ty = t % p.tiles_y;
  t /= p.tiles_y;
  const int tx = t % p.tiles_x;
  const int tz = t / p.tiles_x;

  const int lo = HW + 1;
  const int y0 = lo + ty * kOutY, x0 = lo + tx * RX;
  const int y = y0 - 1 + lane;
  // y and x are never slid across offsets, so lanes and rows past the interior are simply
  // clamped to [HW, n-1-HW] (keeping +-HW inside the volume); they only feed outputs that are
  // never stored. z IS slid (dw ring buffer), which needs consecutive planes: a half that would
  // run past the interior is shifted back inside it instead, and then stores only the planes it
  // owns (those at or after its unshifted start), so every voxel is written exactly once.
  // The launcher guarantees at least TZ interior planes, so a shifted half starts at >= lo.
  const int yc = min(y, p.ny - 1 - HW);
  int rowoff[NR];
#pragma unroll
  for (int r = 0; r < NR; ++r) rowoff[r] = min(x0 - 1 + r, p.nx - 1 - HW) * p.ny + yc;
  int zs[2], zown[2];
  int planeoff[2][NQ];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    zown[h] = lo + tz * (2 * TZ) + h * TZ;
    zs[h] = min(zown[h], p.nz - lo - TZ);
#pragma unroll
    for (int q = 0; q < NQ; ++q) planeoff[h][q] = (zs[h] - 1 + q) * p.nxy;
  }

  // Input patch values, negated so that D = (A + In)^2, paired over the two z-halves.
  float2 In[NQ][NR];
#pragma unroll
  for (int q = 0; q < NQ; ++q)
#pragma unroll
    for (int r = 0; r < NR; ++r)
      In[q][r] = make_float2(-__ldg(p.img + planeoff[0][q] + rowoff[r]),
                             -__ldg(p.img + planeoff[1][q] + rowoff[r]));

  float2 P[TZ][RX], W[TZ][RX];
#pragma unroll
  for (int q = 0; q < TZ; ++q)
#pragma unroll
    for (int r = 0; r < RX; ++r) {
      P[q][r] = make_float2(0.f, 0.f);
      W[q][r] = make_float2(0.f, 0.f);
    }
  const float2 negk2 = make_float2(p.neg_k, p.neg_k);

#pragma unroll 1
  for (int a = 0; a < p.num; ++a) {
    const float *A = p.atlas + (long long)a * p.nvox;
    const float *L = p.label + (long long)a * p.nvox;
#pragma unroll 1
    for (int du = -HW; du <= HW; ++du) {
#pragma unroll 1
      for (int dv = -HW; dv <= HW; ++dv) {
        // Pointers at offset (dw=-HW, du, dv); step s adds s planes.
        const float *Ab = A + (du * p.ny + dv - HW * p.nxy);
        const float *Lb = L + (du * p.ny + dv - HW * p.nxy);
        float2 Aw[NQ][NR];  // logical plane q at step s lives in slot (q+s)%NQ
        float2 Lw[TZ][RX];  // logical output plane q at step s lives in slot (q+s)%TZ
#pragma unroll
        for (int q = 0; q < NQ - 1; ++q)
#pragma unroll
          for (int r = 0; r < NR; ++r)
            Aw[q][r] = make_float2(__ldg(Ab + planeoff[0][q] + rowoff[r]),
                                   __ldg(Ab + planeoff[1][q] + rowoff[r]));
#pragma unroll
        for (int q = 0; q < TZ - 1; ++q)
#pragma unroll
          for (int r = 0; r < RX; ++r)
            Lw[q][r] = make_float2(__ldg(Lb + planeoff[0][q + 1] + rowoff[r + 1]),
                                   __ldg(Lb + planeoff[1][q + 1] + rowoff[r + 1]));
#pragma unroll
        for (int s = 0; s < NS; ++s) {
          const int soff = s * p.nxy;
          // New atlas plane (logical NQ-1) and new CT plane (logical TZ-1) for this dw.
          {
            constexpr int qa = NQ - 1;
            const int sa = (qa + s) % NQ;
#pragma unroll
            for (int r = 0; r < NR; ++r)
              Aw[sa][r] = make_float2(__ldg(Ab + soff + planeoff[0][qa] + rowoff[r]),
                                      __ldg(Ab + soff + planeoff[1][qa] + rowoff[r]));
            constexpr int ql = TZ - 1;
            const int sl = (ql + s) % TZ;
#pragma unroll
            for (int r = 0; r < RX; ++r)
              Lw[sl][r] = make_float2(__ldg(Lb + soff + planeoff[0][ql + 1] + rowoff[r + 1]),
                                      __ldg(Lb + soff + planeoff[1][ql + 1] + rowoff[r + 1]));
          }
          // x-box of D per plane.
          float2 g[NQ][RX];
#pragma unroll
          for (int q = 0; q < NQ; ++q) {
            const int sq = (q + s) % NQ;
            float2 D[NR];
#pragma unroll
            for (int r = 0; r < NR; ++r) {
              const float2 d = add2(Aw[sq][r], In[q][r]);
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
          // z-box, y-box (shuffles), weight, accumulate.
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
                const float2 c = S[k];
                const float2 lft = make_float2(__shfl_up_sync(0xffffffffu, c.x, 1),
                                               __shfl_up_sync(0xffffffffu, c.y, 1));
                const float2 rgt = make_float2(__shfl_down_sync(0xffffffffu, c.x, 1),
                                               __shfl_down_sync(0xffffffffu, c.y, 1));
                const float2 ssd = add2(add2(c, lft), rgt);
                const float2 e = mul2(ssd, negk2);
                const float2 w = make_float2(ex2_approx(e.x), ex2_approx(e.y));
                const int sl = (q + k + s) % TZ;
                P[q + k][x] = fma2(w, Lw[sl][x], P[q + k][x]);
                W[q + k][x] = add2(W[q + k][x], w);
              }
            }
          }
        }
      }
    }
  }

  // NaN rule of NewPatchedBrainPureC.cpp:1325-1331, in FP32.
  if (lane >= 1 && lane <= kOutY && y < p.ny - lo) {
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
      for (int q = 0; q < TZ; ++q) {
        const int z = zs[h] + q;
        if (z < zown[h] || z >= p.nz - lo) continue;
#pragma unroll
        for (int r = 0; r < RX; ++r) {
          const int x = x0 + r;
          if (x >= p.nx - lo) continue;
          const float pr = h ? P[q][r].y : P[q][r].x;
          const float sw = h ? W[q][r].y : W[q][r].x;
          p.out[(long long)z * p.nxy + (long long)x * p.ny + y] = fuse_result(pr, sw);
        }
      }
  }
}

// Direct form for volumes with fewer interior z-planes than one tile half: one thread per
// interior voxel, every candidate's 27-tap SSD summed directly in FP32. Same arithmetic
// contract as the tiled kernel, no sliding windows, no tile constraints.
template <int HW>
__global__ void __launch_bounds__(128) fuse_direct_kernel(const FuseParams p) {
  const int lo = HW + 1;
  const int ix = p.nx - 2 * lo, iy = p.ny - 2 * lo, iz = p.nz - 2 * lo;
  const long long total = (long long)ix * iy * iz;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int y = (int)(i % iy) + lo;
    const long long rest = i / iy;
    const int x = (int)(rest % ix) + lo;
    const int z = (int)(rest / ix) + lo;
    const int c = z * p.nxy + x * p.ny + y;
    float in[27];
    int k = 0;
    for (int a = -1; a <= 1; ++a)
      for (int b = -1; b <= 1; ++b)
        for (int e = -1; e <= 1; ++e) in[k++] = __ldg(p.img + c + a * p.nxy + b * p.ny + e);
    float pr = 0.f, sw = 0.f;
    for (int at = 0; at < p.num; ++at) {
      const float *A = p.atlas + (long long)at * p.nvox;
      const float *L = p.label + (long long)at * p.nvox;
      for (int dw = -HW; dw <= HW; ++dw)
        for (int du = -HW; du <= HW; ++du)
          for (int dv = -HW; dv <= HW; ++dv) {
            const int cc = c + dw * p.nxy + du * p.ny + dv;
            float ssd = 0.f;
            k = 0;
            for (int a = -1; a <= 1; ++a)
              for (int b = -1; b <= 1; ++b)
                for (int e = -1; e <= 1; ++e) {
                  const float d = in[k++] - __ldg(A + cc + a * p.nxy + b * p.ny + e);
                  ssd = fmaf(d, d, ssd);
                }
            const float w = ex2_approx(ssd * p.neg_k);
            pr = fmaf(w, __ldg(L + cc), pr);
            sw += w;
          }
    }
    p.out[c] = fuse_result(pr, sw);
  }
}

constexpr int kThreads = 128;

// Per-window tile shape (x rows RX, z planes per half TZ), chosen so the register-resident
// windows fit in 255 registers without spilling.
template <int HW> struct TileShape { static constexpr int RX = 4, TZ = 2; };
template <> struct TileShape<5> { static constexpr int RX = 3, TZ = 3; };

template <int HW>
cudaError_t launch_hw(const Geometry &g, const FuseParams &base, cudaStream_t stream) {
  constexpr int RX = TileShape<HW>::RX, TZ = TileShape<HW>::TZ;
  FuseParams p = base;
  if (g.iz < TZ) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long long total = (long long)g.ix * g.iy * g.iz;
    const long long want = (total + kThreads - 1) / kThreads;
    const unsigned blocks = (unsigned)(want < (long long)sms * 16 ? want : (long long)sms * 16);
    fuse_direct_kernel<HW><<<blocks, kThreads, 0, stream>>>(p);
    return cudaGetLastError();
  }
  p.tiles_y = (g.iy + kOutY - 1) / kOutY;
  p.tiles_x = (g.ix + RX - 1) / RX;
  p.tiles_z = (g.iz + 2 * TZ - 1) / (2 * TZ);
  const long long warps = (long long)p.tiles_y * p.tiles_x * p.tiles_z;
  const long long blocks = (warps * 32 + kThreads - 1) / kThreads;
  fuse_plain_kernel<HW, RX, TZ><<<(unsigned)blocks, kThreads, 0, stream>>>(p);
  return cudaGetLastError();
}

}  // namespace

int fuse_plain_launches(const Geometry &g) { return (g.ix > 0 && g.iy > 0 && g.iz > 0) ? 1 : 0; }

cudaError_t launch_fuse_plain(const Geometry &g, const float *img, const float *atlas,
                              const float *label, float *out, double div, cudaStream_t stream) {
  if (g.ix <= 0 || g.iy <= 0 || g.iz <= 0) return cudaSuccess;  // no interior voxel
  FuseParams p{};
  p.img = img;
  p.atlas = atlas;
  p.label = label;
  p.out = out;
  p.nx = g.nx;
  p.ny = g.ny;
  p.nz = g.nz;
  p.num = g.num;
  p.nxy = g.nx * g.ny;
  p.nvox = g.nvox();
  p.neg_k = (float)(-1.4426950408889634 / div);
  switch (g.hw) {
    case 1: return launch_hw<1>(g, p, stream);
    case 2: return launch_hw<2>(g, p, stream);
    case 3: return launch_hw<3>(g, p, stream);
    case 4: return launch_hw<4>(g, p, stream);
    case 5: return launch_hw<5>(g, p, stream);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace pct
