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
// and every GPU that loads it keeps it until the process exits. Host code cannot use the
// array's name as a device address, so the first call on each device (with that device
// current) looks the address up with cudaGetSymbolAddress; make that first call before any
// stream capture. All calls share the array and it keeps the last call's contents; the counters
// that must start at zero are cleared by every call. Calls whose work overlaps on the GPU race on
// the array: issue them one after another.
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "pct_b200.h"
#include "pct_internal.h"

namespace {

// Largest volume this entry point accepts, and the scratch it needs: a 64-byte header of
// counters plus two index lists of kMaxVoxels ints each (64 MiB in total).
constexpr long long kMaxVoxels = 1LL << 23;
constexpr size_t kScratchBytes = 64 + 2 * (size_t)kMaxVoxels * sizeof(int);

static __device__ __align__(256) unsigned char g_fill_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void *g_addr[kMaxDevices] = {};

// Device address of g_fill_scratch for the current device, looked up once per device.
cudaError_t scratch_address(void **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_addr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_fill_scratch);
    if (e != cudaSuccess) return e;
    g_addr[dev] = p;
  }
  *out = g_addr[dev];
  return cudaSuccess;
}

}  // namespace

extern "C" int pct_regularize_device_noalloc(float *d_vol, int nx, int ny, int nz, int nh,
                                             int64_t *fills, void *stream) {
  if (!d_vol || nx <= 0 || ny <= 0 || nz <= 0 || nh < 1 || (nh % 2) == 0)
    return PCT_ERR_INVALID_ARG;
  if ((long long)nx * ny * nz > kMaxVoxels) return PCT_ERR_TOO_LARGE;
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
