// C ABI of the learned-proposal form: model lifecycle, training set, training, checkpoints.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <new>
#include <string>
#include <vector>

#include "pct_b200.h"
#include "pct_internal.h"
#include "pct_learned.h"

namespace pct {
namespace learned {
size_t train_smem_bytes();
size_t subject_ref_bytes();
cudaError_t launch_targets(const void *subject_refs, const int *samples, int n, float *targets,
                           short *top, cudaStream_t s);
cudaError_t launch_train_grads(const void *subject_refs, const int *samples, const float *targets,
                               int begin, int count, const __nv_bfloat16 *wbf, float *grad,
                               float *loss_sum, cudaStream_t s);
cudaError_t launch_adam(float *master, __nv_bfloat16 *wbf, float *m, float *v, float *grad,
                        float grad_scale, float lr, int step, cudaStream_t s);
cudaError_t launch_round_weights(const float *master, __nv_bfloat16 *wbf, cudaStream_t s);
}  // namespace learned
}  // namespace pct

using namespace pct::learned;

struct pct_model {
  int device = 0;
  cudaStream_t stream = nullptr;
  float *master = nullptr, *m = nullptr, *v = nullptr, *grad = nullptr, *loss = nullptr;
  __nv_bfloat16 *wbf = nullptr;
  int step = 0;
  std::string last_error;
};

struct pct_train_set {
  int device = 0;
  int n = 0;
  void *subjects = nullptr;  // device SubjectRef table
  int *samples = nullptr;    // device [n][3]
  float *targets = nullptr;  // device [n][33]
  short *top = nullptr;      // device [n][32]
  int pos = 0;               // next sample of the current epoch
};

const void *pct::learned::model_weights(const pct_model *m) { return m->wbf; }
int pct::learned::model_device(const pct_model *m) { return m->device; }

namespace {

uint64_t mix64(uint64_t z) {
  z += 0x9e3779b97f4a7c15ULL;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

double normal(uint64_t seed, uint64_t i) {
  const double u1 = ((mix64(seed ^ (2 * i)) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
  const double u2 = ((mix64(seed ^ (2 * i + 1)) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
  return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

// He-normal convolution weights, small heads, zero biases; deterministic in `seed`.
std::vector<float> init_params(uint64_t seed) {
  std::vector<float> p(kParams, 0.f);
  auto fill = [&](int off, int count, double sd) {
    for (int i = 0; i < count; ++i) p[off + i] = (float)(sd * normal(seed, (uint64_t)off + i));
  };
  fill(kW1, kC * kCin * 27, sqrt(2.0 / (kCin * 27)));
  fill(kW2, kC * kC * 27, sqrt(2.0 / (kC * 27)));
  fill(kW3, kC * kC * 27, sqrt(2.0 / (kC * 27)));
  fill(kW4, kC * kC * 27, sqrt(2.0 / (kC * 27)));
  fill(kH, kHeads * kC, 0.1 * sqrt(1.0 / kC));
  return p;
}

int model_fail(pct_model *m, int st, const std::string &msg) {
  if (m) m->last_error = msg;
  return st;
}

#define MCUDA(m, call)                                                                        \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess) return model_fail(m, PCT_ERR_CUDA, std::string(#call) + ": " +       \
                                                                  cudaGetErrorString(e_));    \
  } while (0)

}  // namespace

extern "C" {

int pct_model_num_params(void) { return kParams; }

int pct_model_create(int device, uint64_t seed, pct_model **out) {
  if (!out) return PCT_ERR_INVALID_ARG;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
    cudaGetLastError();
    return PCT_ERR_NO_DEVICE;
  }
  pct_model *m = new (std::nothrow) pct_model();
  if (!m) return PCT_ERR_OUT_OF_MEMORY;
  m->device = device;
  auto bail = [&](int st) {
    pct_model_destroy(m);
    return st;
  };
  if (cudaSetDevice(device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess)
    return bail(PCT_ERR_CUDA);
  const size_t fb = kParams * sizeof(float);
  if (cudaMalloc(&m->master, fb) != cudaSuccess || cudaMalloc(&m->m, fb) != cudaSuccess ||
      cudaMalloc(&m->v, fb) != cudaSuccess || cudaMalloc(&m->grad, fb) != cudaSuccess ||
      cudaMalloc(&m->loss, sizeof(float)) != cudaSuccess ||
      cudaMalloc(&m->wbf, kParams * sizeof(__nv_bfloat16)) != cudaSuccess) {
    cudaGetLastError();
    return bail(PCT_ERR_OUT_OF_MEMORY);
  }
  const std::vector<float> p = init_params(seed);
  const int st = pct_model_set_params(m, p.data());
  if (st) return bail(st);
  *out = m;
  return PCT_OK;
}

int pct_model_destroy(pct_model *m) {
  if (!m) return PCT_ERR_INVALID_ARG;
  cudaSetDevice(m->device);
  if (m->stream) cudaStreamSynchronize(m->stream);
  for (void *p : {(void *)m->master, (void *)m->m, (void *)m->v, (void *)m->grad, (void *)m->loss,
                  (void *)m->wbf})
    if (p) cudaFree(p);
  if (m->stream) cudaStreamDestroy(m->stream);
  delete m;
  return PCT_OK;
}

const char *pct_model_last_error(const pct_model *m) { return m ? m->last_error.c_str() : ""; }

int pct_model_set_params(pct_model *m, const float *params) {
  if (!m || !params) return PCT_ERR_INVALID_ARG;
  MCUDA(m, cudaSetDevice(m->device));
  const size_t fb = kParams * sizeof(float);
  MCUDA(m, cudaMemcpyAsync(m->master, params, fb, cudaMemcpyHostToDevice, m->stream));
  MCUDA(m, cudaMemsetAsync(m->m, 0, fb, m->stream));
  MCUDA(m, cudaMemsetAsync(m->v, 0, fb, m->stream));
  MCUDA(m, cudaMemsetAsync(m->grad, 0, fb, m->stream));
  MCUDA(m, launch_round_weights(m->master, m->wbf, m->stream));
  MCUDA(m, cudaStreamSynchronize(m->stream));
  m->step = 0;
  return PCT_OK;
}

int pct_model_get_params(pct_model *m, float *params, int inference_precision) {
  if (!m || !params) return PCT_ERR_INVALID_ARG;
  MCUDA(m, cudaSetDevice(m->device));
  if (inference_precision) {
    std::vector<__nv_bfloat16> b(kParams);
    MCUDA(m, cudaMemcpyAsync(b.data(), m->wbf, kParams * sizeof(__nv_bfloat16),
                             cudaMemcpyDeviceToHost, m->stream));
    MCUDA(m, cudaStreamSynchronize(m->stream));
    for (int i = 0; i < kParams; ++i) params[i] = __bfloat162float(b[i]);
    return PCT_OK;
  }
  MCUDA(m, cudaMemcpyAsync(params, m->master, kParams * sizeof(float), cudaMemcpyDeviceToHost,
                           m->stream));
  MCUDA(m, cudaStreamSynchronize(m->stream));
  return PCT_OK;
}

int pct_model_load_file(pct_model *m, const char *path) {
  if (!m || !path) return PCT_ERR_INVALID_ARG;
  FILE *f = fopen(path, "rb");
  if (!f) return model_fail(m, PCT_ERR_INVALID_ARG, std::string("cannot open ") + path);
  unsigned char hdr[16];
  std::vector<float> p(kParams);
  const bool ok = fread(hdr, 1, 16, f) == 16 && memcmp(hdr, "PCTLRN01", 8) == 0 &&
                  (uint32_t)(hdr[8] | hdr[9] << 8 | hdr[10] << 16 | (uint32_t)hdr[11] << 24) ==
                      (uint32_t)kParams &&
                  fread(p.data(), sizeof(float), kParams, f) == (size_t)kParams &&
                  fgetc(f) == EOF;
  fclose(f);
  if (!ok)
    return model_fail(m, PCT_ERR_INVALID_ARG,
                      std::string(path) + ": not a checkpoint of " + std::to_string(kParams) +
                          " parameters");
  return pct_model_set_params(m, p.data());
}

int pct_model_save_file(pct_model *m, const char *path) {
  if (!m || !path) return PCT_ERR_INVALID_ARG;
  std::vector<float> p(kParams);
  int st = pct_model_get_params(m, p.data(), 0);
  if (st) return st;
  FILE *f = fopen(path, "wb");
  if (!f) return model_fail(m, PCT_ERR_INVALID_ARG, std::string("cannot create ") + path);
  unsigned char hdr[16] = {'P', 'C', 'T', 'L', 'R', 'N', '0', '1', 0, 0, 0, 0, 0, 0, 0, 0};
  const uint32_t n = (uint32_t)kParams;
  for (int i = 0; i < 4; ++i) hdr[8 + i] = (unsigned char)(n >> (8 * i));
  const bool ok = fwrite(hdr, 1, 16, f) == 16 &&
                  fwrite(p.data(), sizeof(float), kParams, f) == (size_t)kParams;
  if (fclose(f) != 0 || !ok) return model_fail(m, PCT_ERR_INTERNAL, std::string("cannot write ") + path);
  return PCT_OK;
}

int pct_train_set_create(int device, const pct_train_subject *subjects, int nsub,
                         const int *samples, int n, pct_train_set **out) {
  if (!subjects || nsub <= 0 || !samples || n <= 0 || !out) return PCT_ERR_INVALID_ARG;
  *out = nullptr;
  // Every sample must be an NH=11 interior voxel: the 11^3 window and its 3^3 patches (and the
  // 9^3 network patch) stay inside the volume.
  for (int i = 0; i < n; ++i) {
    const int s = samples[3 * i], a = samples[3 * i + 1], vox = samples[3 * i + 2];
    if (s < 0 || s >= nsub || a < 0 || a >= subjects[s].num_atlas) return PCT_ERR_INVALID_ARG;
    const pct_train_subject &t = subjects[s];
    const int nxy = t.nx * t.ny;
    if (vox < 0 || (long long)vox >= (long long)nxy * t.nz) return PCT_ERR_INVALID_ARG;
    const int z = vox / nxy, x = (vox % nxy) / t.ny, y = vox % t.ny;
    if (z < 6 || x < 6 || y < 6 || z >= t.nz - 6 || x >= t.nx - 6 || y >= t.ny - 6)
      return PCT_ERR_INVALID_ARG;
  }
  if (cudaSetDevice(device) != cudaSuccess) return PCT_ERR_NO_DEVICE;
  pct_train_set *ts = new (std::nothrow) pct_train_set();
  if (!ts) return PCT_ERR_OUT_OF_MEMORY;
  ts->device = device;
  ts->n = n;
  auto bail = [&](int st) {
    pct_train_set_destroy(ts);
    return st;
  };
  // Host copy of the subject table in the kernel's layout (pointer, pointer, 4 ints).
  struct Ref {
    const float *img;
    const float *atlas;
    int nx, ny, nz, num;
  };
  static_assert(sizeof(Ref) == 32, "subject table layout");
  if (subject_ref_bytes() != sizeof(Ref)) return bail(PCT_ERR_INTERNAL);
  std::vector<Ref> refs(nsub);
  for (int i = 0; i < nsub; ++i)
    refs[i] = Ref{subjects[i].img, subjects[i].atlas, subjects[i].nx, subjects[i].ny, subjects[i].nz,
                  subjects[i].num_atlas};
  if (cudaMalloc(&ts->subjects, nsub * sizeof(Ref)) != cudaSuccess ||
      cudaMalloc(&ts->samples, (size_t)n * 3 * sizeof(int)) != cudaSuccess ||
      cudaMalloc(&ts->targets, (size_t)n * kHeads * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&ts->top, (size_t)n * kTopK * sizeof(short)) != cudaSuccess) {
    cudaGetLastError();
    return bail(PCT_ERR_OUT_OF_MEMORY);
  }
  if (cudaMemcpy(ts->subjects, refs.data(), nsub * sizeof(Ref), cudaMemcpyHostToDevice) ||
      cudaMemcpy(ts->samples, samples, (size_t)n * 3 * sizeof(int), cudaMemcpyHostToDevice) ||
      launch_targets(ts->subjects, ts->samples, n, ts->targets, ts->top, 0) ||
      cudaDeviceSynchronize()) {
    cudaGetLastError();
    return bail(PCT_ERR_CUDA);
  }
  *out = ts;
  return PCT_OK;
}

int pct_train_set_targets(pct_train_set *ts, float *targets, int16_t *top) {
  if (!ts) return PCT_ERR_INVALID_ARG;
  if (cudaSetDevice(ts->device) != cudaSuccess) return PCT_ERR_CUDA;
  if (targets && cudaMemcpy(targets, ts->targets, (size_t)ts->n * kHeads * sizeof(float),
                            cudaMemcpyDeviceToHost) != cudaSuccess)
    return PCT_ERR_CUDA;
  if (top && cudaMemcpy(top, ts->top, (size_t)ts->n * kTopK * sizeof(short),
                        cudaMemcpyDeviceToHost) != cudaSuccess)
    return PCT_ERR_CUDA;
  return PCT_OK;
}

int pct_train_set_destroy(pct_train_set *ts) {
  if (!ts) return PCT_ERR_INVALID_ARG;
  cudaSetDevice(ts->device);
  for (void *p : {ts->subjects, (void *)ts->samples, (void *)ts->targets, (void *)ts->top})
    if (p) cudaFree(p);
  delete ts;
  return PCT_OK;
}

int pct_model_gradients(pct_model *m, pct_train_set *ts, int begin, int count, float *grad,
                        float *loss) {
  if (!m || !ts || begin < 0 || count <= 0 || begin + count > ts->n) return PCT_ERR_INVALID_ARG;
  MCUDA(m, cudaSetDevice(m->device));
  MCUDA(m, cudaMemsetAsync(m->grad, 0, kParams * sizeof(float), m->stream));
  MCUDA(m, cudaMemsetAsync(m->loss, 0, sizeof(float), m->stream));
  MCUDA(m, launch_train_grads(ts->subjects, ts->samples, ts->targets, begin, count, m->wbf, m->grad,
                              m->loss, m->stream));
  std::vector<float> g(kParams);
  float l = 0.f;
  MCUDA(m, cudaMemcpyAsync(g.data(), m->grad, kParams * sizeof(float), cudaMemcpyDeviceToHost,
                           m->stream));
  MCUDA(m, cudaMemcpyAsync(&l, m->loss, sizeof(float), cudaMemcpyDeviceToHost, m->stream));
  MCUDA(m, cudaMemsetAsync(m->grad, 0, kParams * sizeof(float), m->stream));
  MCUDA(m, cudaStreamSynchronize(m->stream));
  // Mean over the batch, as the training step uses.
  if (grad)
    for (int i = 0; i < kParams; ++i) grad[i] = g[i] / count;
  if (loss) *loss = l / count;
  return PCT_OK;
}

int pct_model_train(pct_model *m, pct_train_set *ts, int batch, int steps, float lr,
                    float *mean_loss) {
  if (!m || !ts || batch <= 0 || steps <= 0 || !(lr > 0)) return PCT_ERR_INVALID_ARG;
  MCUDA(m, cudaSetDevice(m->device));
  MCUDA(m, cudaMemsetAsync(m->loss, 0, sizeof(float), m->stream));
  long long seen = 0;
  int pos = ts->pos;
  for (int k = 0; k < steps; ++k) {
    const int count = batch < ts->n - pos ? batch : ts->n - pos;
    MCUDA(m, launch_train_grads(ts->subjects, ts->samples, ts->targets, pos, count, m->wbf,
                                m->grad, m->loss, m->stream));
    MCUDA(m, launch_adam(m->master, m->wbf, m->m, m->v, m->grad, 1.0f / count, lr, ++m->step,
                         m->stream));
    seen += count;
    pos += count;
    if (pos >= ts->n) pos = 0;  // next epoch over the (pre-shuffled) samples
  }
  ts->pos = pos;
  float l = 0.f;
  MCUDA(m, cudaMemcpyAsync(&l, m->loss, sizeof(float), cudaMemcpyDeviceToHost, m->stream));
  MCUDA(m, cudaStreamSynchronize(m->stream));
  if (mean_loss) *mean_loss = (float)(l / (double)seen);
  return PCT_OK;
}

int pct_model_probe(pct_model *m, const float *d_img, const float *d_atlas, int nx, int ny, int nz,
                    const int64_t *voxels, int n, float *features, int8_t *top, float *conf) {
  if (!m || !d_img || !d_atlas || !voxels || n <= 0) return PCT_ERR_INVALID_ARG;
  pct::Geometry g;
  if (nx <= 0 || ny <= 0 || nz <= 0 || !pct::make_geometry(nx, ny, nz, 1, 11, &g))
    return PCT_ERR_INVALID_ARG;
  if ((long long)n * 24 + 16 > g.nvox() * 8) return PCT_ERR_INVALID_ARG;
  for (int i = 0; i < n; ++i)
    if (voxels[i] < 0 || voxels[i] >= g.nvox()) return PCT_ERR_INVALID_ARG;
  MCUDA(m, cudaSetDevice(m->device));
  void *scratch = nullptr;
  if (cudaMalloc(&scratch, infer_scratch_bytes(g)) != cudaSuccess) {
    cudaGetLastError();
    return model_fail(m, PCT_ERR_OUT_OF_MEMORY, "feature scratch");
  }
  const cudaError_t e = learned_probe(g, m->wbf, d_img, d_atlas, scratch, voxels, n, features,
                                      reinterpret_cast<signed char *>(top), conf, m->stream);
  cudaFree(scratch);
  if (e != cudaSuccess) return model_fail(m, PCT_ERR_CUDA, cudaGetErrorString(e));
  return PCT_OK;
}

}  // extern "C"
