// Element-wise pre/post steps of the path: label normalisation before it and the map back to
// HU after it. Both are HBM-bound streams: float4 grid-stride loops sized to the SM count.
#include <cuda_runtime.h>
#include <stdint.h>

#include "pct_internal.h"

namespace pct {
namespace {

// L' = 255*((L+1024)/4095) in float, same operation order as NewPatchedBrainPureC.cpp:1588-1589.
__device__ __forceinline__ float normalize_one(float l) {
  return __fmul_rn(255.0f, __fdiv_rn(__fadd_rn(l, 1024.0f), 4095.0f));
}

// RoundMatrix then round(4095*(v/255)) - 1024 (NewPatchedBrainPureC.cpp:1221-1227,1732-1738).
__device__ __forceinline__ float finalize_one(float v) {
  const float r = roundf(v);
  return __fsub_rn(roundf(__fmul_rn(4095.0f, __fdiv_rn(r, 255.0f))), 1024.0f);
}

template <int OP>
__global__ void pointwise_kernel(float *__restrict__ v, size_t n, bool vec4) {
  // vec4: v is 16-byte aligned, so the body can move float4s; the tail goes element-wise.
  const size_t n4 = vec4 ? n / 4 : 0;
  float4 *v4 = reinterpret_cast<float4 *>(v);
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += stride) {
    float4 x = v4[i];
    if (OP == 0) {
      x.x = normalize_one(x.x); x.y = normalize_one(x.y);
      x.z = normalize_one(x.z); x.w = normalize_one(x.w);
    } else {
      x.x = finalize_one(x.x); x.y = finalize_one(x.y);
      x.z = finalize_one(x.z); x.w = finalize_one(x.w);
    }
    v4[i] = x;
  }
  for (size_t i = n4 * 4 + (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    v[i] = OP == 0 ? normalize_one(v[i]) : finalize_one(v[i]);
}

template <int OP>
cudaError_t launch(float *v, size_t n, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const size_t want = (n / 4 + 255) / 256;
  const size_t cap = (size_t)sms * 8;
  const unsigned blocks = (unsigned)(want < 1 ? 1 : (want > cap ? cap : want));
  const bool vec4 = reinterpret_cast<uintptr_t>(v) % 16 == 0;
  pointwise_kernel<OP><<<blocks, 256, 0, stream>>>(v, n, vec4);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_normalize_labels(float *label, size_t n, cudaStream_t stream) {
  return launch<0>(label, n, stream);
}

cudaError_t launch_finalize_hu(float *vol, size_t n, cudaStream_t stream) {
  return launch<1>(vol, n, stream);
}

}  // namespace pct
