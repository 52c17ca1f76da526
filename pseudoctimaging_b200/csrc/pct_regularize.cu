// NaN median fill after the path (RegularizationStep + Median,
// NewPatchedBrainPureC.cpp:1024-1047,1059-1106; PatchBasedPseudoCT.cu:1501-1595).
//
// The reference sweeps the interior in z, x, y order and replaces each NaN, in place, by the
// median of the non-NaN values of its 3x3x3 neighbourhood, so a voxel sees the fills of voxels
// before it in the sweep and the NaNs of voxels after it. That order is reproduced exactly,
// in parallel, by rounds: a NaN voxel is filled in the first round in which none of its NaN
// neighbours that come EARLIER in the sweep is still NaN. Its earlier neighbours then hold
// their final fills and its later NaN neighbours are still NaN (each of them waits for it), so
// the median sees exactly what the sequential sweep would. Two voxels filled in the same round
// are never neighbours, so a round has no read/write conflicts that change a result.
//
// With a non-NaN border every NaN has a non-NaN earlier neighbour by the time it is ready, so
// one sweep's worth of rounds fills everything; the number of rounds is the longest chain of
// NaN voxels that follow each other in sweep order. Rounds are bounded by the number of NaN
// voxels; a batch of rounds that fills nothing stops the loop (only possible with NaN in the
// border).
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "pct_internal.h"

namespace pct {
namespace {

__global__ void collect_nan_kernel(const float *__restrict__ vol, int nx, int ny, int nz, int lo,
                                   int *__restrict__ list, int *__restrict__ count) {
  const int ix = nx - 2 * lo, iy = ny - 2 * lo, iz = nz - 2 * lo;
  const long long total = (long long)ix * iy * iz;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int y = (int)(i % iy) + lo;
    const long long r = i / iy;
    const int x = (int)(r % ix) + lo;
    const int z = (int)(r / ix) + lo;
    const int k = z * nx * ny + x * ny + y;
    if (isnan(vol[k])) list[atomicAdd(count, 1)] = k;
  }
}

// Median of the non-NaN values among the 27 neighbours in (z, x, y) order, as Median() does:
// stable sort, middle element, or the double average of the two middle ones.
__device__ float median27(const float *v, int *cnt_out) {
  float buf[27];
  int cnt = 0;
#pragma unroll
  for (int j = 0; j < 27; ++j)
    if (!isnan(v[j])) buf[cnt++] = v[j];
  for (int i = 1; i < cnt; ++i) {  // stable insertion sort (strict >)
    const float key = buf[i];
    int j = i - 1;
    while (j >= 0 && buf[j] > key) {
      buf[j + 1] = buf[j];
      --j;
    }
    buf[j + 1] = key;
  }
  *cnt_out = cnt;
  if (cnt <= 0) return __int_as_float(0x7fc00000);
  if ((cnt & 1) == 0) return (float)(((double)buf[cnt / 2 - 1] + (double)buf[cnt / 2]) / 2.0);
  return buf[cnt / 2];
}

__global__ void fill_round_kernel(float *vol, int nx, int ny, int nz, int lo,
                                  const int *__restrict__ list,
                                  const int *__restrict__ count_in, int *__restrict__ next,
                                  int *__restrict__ count_next, unsigned long long *fills) {
  const int n = *count_in;
  const int nxy = nx * ny;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int k = list[i];
    const int z = k / nxy, x = (k % nxy) / ny, y = k % ny;
    float v[27];
    bool ready = true;
    int j = 0;
    for (int dz = -1; dz <= 1; ++dz)
      for (int dx = -1; dx <= 1; ++dx)
        for (int dy = -1; dy <= 1; ++dy, ++j) {
          const int kk = k + dz * nxy + dx * ny + dy;
          const float val = *((volatile const float *)vol + kk);
          v[j] = val;
          // An earlier interior NaN neighbour is still pending. (NaNs outside the interior are
          // never filled by the reference; they only drop out of the median.)
          const bool interior = z + dz >= lo && z + dz < nz - lo && x + dx >= lo &&
                                x + dx < nx - lo && y + dy >= lo && y + dy < ny - lo;
          if (kk < k && interior && isnan(val)) ready = false;
        }
    if (!ready) {
      next[atomicAdd(count_next, 1)] = k;
      continue;
    }
    int cnt;
    const float m = median27(v, &cnt);
    if (cnt > 0) {
      vol[k] = m;
      atomicAdd(fills, 1ULL);
    } else {
      next[atomicAdd(count_next, 1)] = k;
    }
  }
}

}  // namespace

size_t regularize_scratch_bytes(long long nvox) {
  // Two index lists of at most nvox entries, two counters and a fill counter.
  return (size_t)nvox * 2 * sizeof(int) + 64;
}

cudaError_t launch_regularize(float *vol, int nx, int ny, int nz, int nh, void *scratch,
                              cudaStream_t stream, long long *fills_out, int *rounds_out) {
  const int lo = (nh - 1) / 2 + 1;
  if (fills_out) *fills_out = 0;
  if (rounds_out) *rounds_out = 0;
  if (nx <= 2 * lo || ny <= 2 * lo || nz <= 2 * lo) return cudaSuccess;
  const long long nvox = (long long)nx * ny * nz;
  char *base = static_cast<char *>(scratch);
  int *counters = reinterpret_cast<int *>(base);  // [0], [1]: list sizes
  unsigned long long *fills = reinterpret_cast<unsigned long long *>(base + 16);
  int *list[2] = {reinterpret_cast<int *>(base + 64),
                  reinterpret_cast<int *>(base + 64) + nvox};
  cudaError_t e = cudaMemsetAsync(base, 0, 64, stream);
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  collect_nan_kernel<<<sms * 4, 256, 0, stream>>>(vol, nx, ny, nz, lo, list[0], &counters[0]);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  int pending = 0;
  if ((e = cudaMemcpyAsync(&pending, &counters[0], sizeof(int), cudaMemcpyDeviceToHost, stream)) !=
      cudaSuccess)
    return e;
  if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) return e;
  // Rounds are enqueued in batches (4, 8, ... 64) between host reads: a round reads its list's
  // length on the device, so rounds after the last NaN cost only an empty launch, and the host
  // waits once per batch instead of once per round.
  const int max_rounds = pending + 1;
  int cur = 0, rounds = 0, batch = 4;
  while (pending > 0) {
    if (rounds >= max_rounds) return cudaErrorUnknown;
    const int blocks = (int)((pending + 255) / 256 < sms * 8 ? (pending + 255) / 256 : sms * 8);
    for (int r = 0; r < batch; ++r) {
      const int nxt = cur ^ 1;
      if ((e = cudaMemsetAsync(&counters[nxt], 0, sizeof(int), stream)) != cudaSuccess) return e;
      fill_round_kernel<<<blocks, 256, 0, stream>>>(vol, nx, ny, nz, lo, list[cur], &counters[cur],
                                                    list[nxt], &counters[nxt], fills);
      if ((e = cudaGetLastError()) != cudaSuccess) return e;
      cur = nxt;
    }
    int left = 0;
    if ((e = cudaMemcpyAsync(&left, &counters[cur], sizeof(int), cudaMemcpyDeviceToHost,
                             stream)) != cudaSuccess)
      return e;
    if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) return e;
    rounds += batch;
    // a batch that filled nothing means only voxels with no non-NaN neighbour remain (possible
    // only with NaN in the border), and no later round could fill them either
    if (left == pending) break;
    pending = left;
    if (batch < 64) batch *= 2;
  }
  unsigned long long f = 0;
  if ((e = cudaMemcpyAsync(&f, fills, sizeof(f), cudaMemcpyDeviceToHost, stream)) != cudaSuccess)
    return e;
  if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) return e;
  if (fills_out) *fills_out = (long long)f;
  if (rounds_out) *rounds_out = rounds;
  return cudaSuccess;
}

}  // namespace pct
