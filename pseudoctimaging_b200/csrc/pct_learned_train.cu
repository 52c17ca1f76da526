// Training side of the learned proposal: exact targets, forward/backward, Adam.
//
// Targets: for a sampled (subject, atlas, voxel) the plain method's SSD of every one of the 11^3
// offsets is computed directly in FP32 (the same 27-tap arithmetic as the path), the 32 smallest
// are kept (ties broken by offset order) and turned into one distribution per axis: the share of
// the 32 that has each dw, du and dv.
//
// Training: one CTA per sample at a time. The sample's two 9^3 patches (scaled input MRI and
// atlas MRI) are staged in shared memory and the whole network runs there: forward through the
// four valid 3x3x3 convolutions and the three heads, softmax cross-entropy per axis against the
// targets, and backward. Weights are read as BF16 (the inference precision); the math and the
// gradients are FP32. Each CTA sums its samples' gradients in shared memory and adds them to the
// global FP32 gradient once. Adam then updates FP32 master weights and re-rounds the BF16 copy.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "pct_internal.h"
#include "pct_learned.h"

namespace pct {
namespace learned {
namespace {

constexpr int kTrainThreads = 256;
constexpr int kN1 = 7 * 7 * 7, kN2 = 5 * 5 * 5, kN3 = 3 * 3 * 3, kNX = 9 * 9 * 9;

struct SubjectRef {
  const float *img;
  const float *atlas;
  int nx, ny, nz, num;
};

__device__ __forceinline__ int cube(int z, int x, int y, int s) { return (z * s + x) * s + y; }

// ---------------------------------------------------------------- targets

__global__ void targets_kernel(const SubjectRef *__restrict__ subs, const int *__restrict__ samples,
                               int n, float *__restrict__ targets, short *__restrict__ top_out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int s = samples[3 * i], a = samples[3 * i + 1], vox = samples[3 * i + 2];
  const SubjectRef sr = subs[s];
  const int nxy = sr.nx * sr.ny;
  const long long nvox = (long long)nxy * sr.nz;
  const float *img = sr.img;
  const float *A = sr.atlas + (long long)a * nvox;
  float in[27];
  {
    int k = 0;
    for (int dz = -1; dz <= 1; ++dz)
      for (int dx = -1; dx <= 1; ++dx)
        for (int dy = -1; dy <= 1; ++dy) in[k++] = __ldg(img + vox + dz * nxy + dx * sr.ny + dy);
  }
  float best[kTopK];
  short idx[kTopK];
  int cnt = 0;
  for (int o = 0; o < kAxis * kAxis * kAxis; ++o) {
    const int dw = o / (kAxis * kAxis) - 5, du = (o / kAxis) % kAxis - 5, dv = o % kAxis - 5;
    const int c = vox + dw * nxy + du * sr.ny + dv;
    float ssd = 0.f;
    int k = 0;
    for (int pz = -1; pz <= 1; ++pz)
      for (int px = -1; px <= 1; ++px)
        for (int py = -1; py <= 1; ++py) {
          const float d = in[k++] - __ldg(A + c + pz * nxy + px * sr.ny + py);
          ssd = fmaf(d, d, ssd);
        }
    if (cnt < kTopK || ssd < best[cnt - 1]) {  // insertion into the sorted top-32
      int j = cnt < kTopK ? cnt++ : kTopK - 1;
      while (j > 0 && best[j - 1] > ssd) {
        best[j] = best[j - 1];
        idx[j] = idx[j - 1];
        --j;
      }
      best[j] = ssd;
      idx[j] = (short)o;
    }
  }
  float *t = targets + (long long)i * kHeads;
  for (int j = 0; j < kHeads; ++j) t[j] = 0.f;
  for (int j = 0; j < kTopK; ++j) {
    const int o = idx[j];
    t[o / (kAxis * kAxis)] += 1.0f / kTopK;
    t[kAxis + (o / kAxis) % kAxis] += 1.0f / kTopK;
    t[2 * kAxis + o % kAxis] += 1.0f / kTopK;
    if (top_out) top_out[(long long)i * kTopK + j] = idx[j];
  }
}

// ---------------------------------------------------------------- forward / backward

struct TrainSmem {
  __nv_bfloat16 w[kParams];  // weights at inference precision
  float g[kParams];          // this CTA's gradient sum
  float x0[kCin * kNX];      // scaled input patches
  float a1[kC * kN1], a2[kC * kN2], a3[kC * kN3], a4[kC];
  float d1[kC * kN1], d2[kC * kN2], d3[kC * kN3], d4[kC];
  float logits[kHeads], dlog[kHeads];
  float loss;
};

__device__ __forceinline__ float wv(const TrainSmem &S, int i) { return __bfloat162float(S.w[i]); }

// out[co][p] = relu(b[co] + sum_ci,k W[co][ci][k] in[ci][p+k]) on an `so`-cube from an `si`-cube
__device__ void conv_fwd(const TrainSmem &S, int woff, int boff, int cin, const float *in, int si,
                         float *out, int so) {
  const int nout = kC * so * so * so;
  for (int o = threadIdx.x; o < nout; o += blockDim.x) {
    const int co = o / (so * so * so), p = o % (so * so * so);
    const int z = p / (so * so), x = (p / so) % so, y = p % so;
    float acc = wv(S, boff + co);
    for (int ci = 0; ci < cin; ++ci) {
      const float *src = in + ci * si * si * si;
      const int wb = woff + (co * cin + ci) * 27;
#pragma unroll
      for (int k = 0; k < 27; ++k) {
        const int kz = k / 9, kx = (k / 3) % 3, ky = k % 3;
        acc = fmaf(wv(S, wb + k), src[cube(z + kz, x + kx, y + ky, si)], acc);
      }
    }
    out[o] = fmaxf(acc, 0.f);
  }
}

// Given dZ (gradient at the pre-activation of a conv layer, already masked by its ReLU):
// accumulate dW, db, and (if din) the gradient w.r.t. the layer's input cube.
__device__ void conv_bwd(TrainSmem &S, int woff, int boff, int cin, const float *in, int si,
                         const float *dz, int so, float *din) {
  const int sosq = so * so * so;
  // weight and bias gradients
  for (int e = threadIdx.x; e < kC * cin * 27; e += blockDim.x) {
    const int co = e / (cin * 27), ci = (e / 27) % cin, k = e % 27;
    const int kz = k / 9, kx = (k / 3) % 3, ky = k % 3;
    const float *src = in + ci * si * si * si;
    const float *g = dz + co * sosq;
    float acc = 0.f;
    for (int p = 0; p < sosq; ++p) {
      const int z = p / (so * so), x = (p / so) % so, y = p % so;
      acc = fmaf(g[p], src[cube(z + kz, x + kx, y + ky, si)], acc);
    }
    S.g[woff + e] += acc;
  }
  for (int co = threadIdx.x; co < kC; co += blockDim.x) {
    float acc = 0.f;
    for (int p = 0; p < sosq; ++p) acc += dz[co * sosq + p];
    S.g[boff + co] += acc;
  }
  if (!din) return;
  // input gradient: din[ci][q] = sum_co,k W[co][ci][k] dz[co][q-k]
  const int sisq = si * si * si;
  for (int e = threadIdx.x; e < cin * sisq; e += blockDim.x) {
    const int ci = e / sisq, q = e % sisq;
    const int qz = q / (si * si), qx = (q / si) % si, qy = q % si;
    float acc = 0.f;
    for (int k = 0; k < 27; ++k) {
      const int z = qz - k / 9, x = qx - (k / 3) % 3, y = qy - k % 3;
      if (z < 0 || x < 0 || y < 0 || z >= so || x >= so || y >= so) continue;
      const int p = cube(z, x, y, so);
      for (int co = 0; co < kC; ++co)
        acc = fmaf(wv(S, woff + (co * cin + ci) * 27 + k), dz[co * sosq + p], acc);
    }
    din[e] = acc;
  }
}

__global__ void __launch_bounds__(kTrainThreads, 1)
    train_kernel(const SubjectRef *__restrict__ subs, const int *__restrict__ samples,
                 const float *__restrict__ targets, int begin, int count,
                 const __nv_bfloat16 *__restrict__ wbf, float *__restrict__ grad,
                 float *__restrict__ loss_sum) {
  extern __shared__ unsigned char smem_raw[];
  TrainSmem &S = *reinterpret_cast<TrainSmem *>(smem_raw);
  for (int i = threadIdx.x; i < kParams; i += blockDim.x) {
    S.w[i] = wbf[i];
    S.g[i] = 0.f;
  }
  if (threadIdx.x == 0) S.loss = 0.f;
  __syncthreads();
  for (int si = blockIdx.x; si < count; si += gridDim.x) {
    const int smp = begin + si;
    const int s = samples[3 * smp], a = samples[3 * smp + 1], vox = samples[3 * smp + 2];
    const SubjectRef sr = subs[s];
    const int nxy = sr.nx * sr.ny;
    const long long nvox = (long long)nxy * sr.nz;
    for (int e = threadIdx.x; e < kCin * kNX; e += blockDim.x) {
      const int c = e / kNX, p = e % kNX;
      const int z = p / 81 - 4, x = (p / 9) % 9 - 4, y = p % 9 - 4;
      const float *src = c == 0 ? sr.img : sr.atlas + (long long)a * nvox;
      S.x0[e] = __ldg(src + vox + z * nxy + x * sr.ny + y) * kInScale;
    }
    __syncthreads();
    conv_fwd(S, kW1, kB1, kCin, S.x0, 9, S.a1, 7);
    __syncthreads();
    conv_fwd(S, kW2, kB2, kC, S.a1, 7, S.a2, 5);
    __syncthreads();
    conv_fwd(S, kW3, kB3, kC, S.a2, 5, S.a3, 3);
    __syncthreads();
    conv_fwd(S, kW4, kB4, kC, S.a3, 3, S.a4, 1);
    __syncthreads();
    for (int o = threadIdx.x; o < kHeads; o += blockDim.x) {
      float acc = wv(S, kHB + o);
      for (int c = 0; c < kC; ++c) acc = fmaf(wv(S, kH + o * kC + c), S.a4[c], acc);
      S.logits[o] = acc;
    }
    __syncthreads();
    // softmax cross-entropy per axis: dlogits = softmax - target
    if (threadIdx.x < 3) {
      const int h = threadIdx.x;
      const float *t = targets + (long long)smp * kHeads + h * kAxis;
      float m = -1e30f;
      for (int j = 0; j < kAxis; ++j) m = fmaxf(m, S.logits[h * kAxis + j]);
      float z = 0.f;
      for (int j = 0; j < kAxis; ++j) z += __expf(S.logits[h * kAxis + j] - m);
      const float lz = __logf(z) + m;
      float l = 0.f;
      for (int j = 0; j < kAxis; ++j) {
        const float lp = S.logits[h * kAxis + j] - lz;
        l -= t[j] * lp;
        S.dlog[h * kAxis + j] = __expf(lp) - t[j];
      }
      atomicAdd(&S.loss, l);
    }
    __syncthreads();
    // heads: dH, dhb, d4
    for (int e = threadIdx.x; e < kHeads * kC; e += blockDim.x)
      S.g[kH + e] += S.dlog[e / kC] * S.a4[e % kC];
    for (int o = threadIdx.x; o < kHeads; o += blockDim.x) S.g[kHB + o] += S.dlog[o];
    for (int c = threadIdx.x; c < kC; c += blockDim.x) {
      float acc = 0.f;
      for (int o = 0; o < kHeads; ++o) acc = fmaf(wv(S, kH + o * kC + c), S.dlog[o], acc);
      S.d4[c] = S.a4[c] > 0.f ? acc : 0.f;
    }
    __syncthreads();
    conv_bwd(S, kW4, kB4, kC, S.a3, 3, S.d4, 1, S.d3);
    __syncthreads();
    for (int e = threadIdx.x; e < kC * kN3; e += blockDim.x)
      if (!(S.a3[e] > 0.f)) S.d3[e] = 0.f;
    __syncthreads();
    conv_bwd(S, kW3, kB3, kC, S.a2, 5, S.d3, 3, S.d2);
    __syncthreads();
    for (int e = threadIdx.x; e < kC * kN2; e += blockDim.x)
      if (!(S.a2[e] > 0.f)) S.d2[e] = 0.f;
    __syncthreads();
    conv_bwd(S, kW2, kB2, kC, S.a1, 7, S.d2, 5, S.d1);
    __syncthreads();
    for (int e = threadIdx.x; e < kC * kN1; e += blockDim.x)
      if (!(S.a1[e] > 0.f)) S.d1[e] = 0.f;
    __syncthreads();
    conv_bwd(S, kW1, kB1, kCin, S.x0, 9, S.d1, 7, nullptr);
    __syncthreads();
  }
  for (int i = threadIdx.x; i < kParams; i += blockDim.x)
    if (S.g[i] != 0.f) atomicAdd(grad + i, S.g[i]);
  if (threadIdx.x == 0) atomicAdd(loss_sum, S.loss);
}

__global__ void adam_kernel(float *__restrict__ master, __nv_bfloat16 *__restrict__ wbf,
                            float *__restrict__ m, float *__restrict__ v,
                            float *__restrict__ grad, float scale, float lr, float b1, float b2,
                            float eps, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kParams) return;
  const float g = grad[i] * scale;
  const float mi = b1 * m[i] + (1.f - b1) * g;
  const float vi = b2 * v[i] + (1.f - b2) * g * g;
  m[i] = mi;
  v[i] = vi;
  const float w = master[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  master[i] = w;
  wbf[i] = __float2bfloat16_rn(w);
  grad[i] = 0.f;
}

__global__ void round_weights_kernel(const float *__restrict__ master,
                                     __nv_bfloat16 *__restrict__ wbf) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < kParams) wbf[i] = __float2bfloat16_rn(master[i]);
}

}  // namespace

size_t train_smem_bytes() { return sizeof(TrainSmem); }

cudaError_t launch_targets(const void *subject_refs, const int *samples, int n, float *targets,
                           short *top, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  targets_kernel<<<(n + 127) / 128, 128, 0, s>>>(static_cast<const SubjectRef *>(subject_refs),
                                                 samples, n, targets, top);
  return cudaGetLastError();
}

cudaError_t launch_train_grads(const void *subject_refs, const int *samples, const float *targets,
                               int begin, int count, const __nv_bfloat16 *wbf, float *grad,
                               float *loss_sum, cudaStream_t s) {
  if (count <= 0) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)sizeof(TrainSmem));
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int blocks = count < sms ? count : sms;
  train_kernel<<<blocks, kTrainThreads, sizeof(TrainSmem), s>>>(
      static_cast<const SubjectRef *>(subject_refs), samples, targets, begin, count, wbf, grad,
      loss_sum);
  return cudaGetLastError();
}

cudaError_t launch_adam(float *master, __nv_bfloat16 *wbf, float *m, float *v, float *grad,
                        float grad_scale, float lr, int step, cudaStream_t s) {
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
  adam_kernel<<<(kParams + 255) / 256, 256, 0, s>>>(master, wbf, m, v, grad, grad_scale, lr, b1, b2,
                                                    eps, c1, c2);
  return cudaGetLastError();
}

cudaError_t launch_round_weights(const float *master, __nv_bfloat16 *wbf, cudaStream_t s) {
  round_weights_kernel<<<(kParams + 255) / 256, 256, 0, s>>>(master, wbf);
  return cudaGetLastError();
}

size_t subject_ref_bytes() { return sizeof(SubjectRef); }

}  // namespace learned
}  // namespace pct
