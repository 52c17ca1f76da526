// Allocation-free variant of the NaN median fill (pct_regularize_device_noalloc).
//
// Who needs it: callers that are not allowed to allocate GPU memory once they are running —
// for example applications that hand all device memory to their own pool allocator up front and
// forbid other libraries from calling cudaMalloc (to avoid fragmentation and surprise
// out-of-memory failures), or latency-critical pipelines that must not allocate after start-up.
// The regular entry point takes its scratch (two index lists over the volume) from a handle,
// which allocates on first use; this one uses a fixed array that lives in the library instead.
//
// The array below is allocated when the CUDA runtime loads this library's device code on a GPU,
// and every GPU that loads it keeps it until the process exits. CUDA loads modules lazily by
// default, so on each device that happens at the first call of this entry point (or of any
// other kernel of the library): make that first call at start-up, before the caller's own pool
// takes the device memory and before any stream capture (or set CUDA_MODULE_LOADING=EAGER, which
// loads the array with the library). Host code cannot use the array's name as a device address,
// so every call looks the address up with cudaGetSymbolAddress on the current device; after the
// first call on a device that lookup allocates nothing, and it stays correct if the caller resets
// the device. All calls share the array and it keeps the last call's contents; the counters that
// must start at zero are cleared by every call. Calls whose work overlaps on the GPU race on the
// array: issue them one after another.
#include <cuda_runtime.h>
#include <stdint.h>

#include "pct_b200.h"
#include "pct_internal.h"

namespace {

// Largest volume this entry point accepts, and the scratch it needs: a 64-byte header of
// counters plus two index lists of kMaxVoxels ints each (64 MiB in total).
constexpr long long kMaxVoxels = 1LL << 23;
constexpr size_t kScratchBytes = 64 + 2 * (size_t)kMaxVoxels * sizeof(int);

static __device__ __align__(256) unsigned char g_fill_scratch[kScratchBytes];

// Device address of g_fill_scratch on the current device. Looked up on every call (it is cheap),
// so that a cudaDeviceReset between calls cannot leave a stale address behind.
cudaError_t scratch_address(void **out) {
  void *p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_fill_scratch);
  if (e != cudaSuccess) return e;
  *out = p;
  return cudaSuccess;
}

}  // namespace

extern "C" int pct_regularize_device_noalloc(float *d_vol, int nx, int ny, int nz, int nh,
                                             int64_t *fills, void *stream) {
  if (!d_vol || nx <= 0 || ny <= 0 || nz <= 0 || nh < 1 || (nh % 2) == 0)
    return PCT_ERR_INVALID_ARG;
  // Compared factor by factor, so no product can overflow before the check.
  if (nx > kMaxVoxels || ny > kMaxVoxels / nx || nz > kMaxVoxels / ((long long)nx * ny))
    return PCT_ERR_TOO_LARGE;
  static_assert(kScratchBytes >= 64 + 2 * (size_t)kMaxVoxels * sizeof(int), "scratch too small");
  void *scratch = nullptr;
  if (scratch_address(&scratch) != cudaSuccess) {
    cudaGetLastError();
    return PCT_ERR_CUDA;
  }
  long long f = 0;
  int rounds = 0;
  // launch_regularize zeroes the counter header itself before using the lists.
  const cudaError_t e = pct::launch_regularize(d_vol, nx, ny, nz, nh, scratch,
                                               static_cast<cudaStream_t>(stream), &f, &rounds);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return PCT_ERR_CUDA;
  }
  if (fills) *fills = f;
  return PCT_OK;
}
