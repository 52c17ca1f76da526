// C ABI of libpct_b200.so (declared in include/pct_b200.h).
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <new>
#include <string>
#include <vector>

#include "pct_b200.h"
#include "pct_internal.h"

namespace {

struct DevBuf {
  void *ptr = nullptr;
  size_t bytes = 0;
};

}  // namespace

struct pct_handle {
  int device = 0;
  cudaStream_t stream = nullptr;       // the handle's own stream
  cudaStream_t user_stream = nullptr;  // set by pct_set_stream for host-pointer calls
  size_t mem_limit = 0;  // 0 = unlimited
  size_t allocated = 0;
  DevBuf img, atlas, label, out, scratch;
  DevBuf err;      // device status word written by kernels with bounded waits
  DevBuf partial;  // per-atlas-group partial sums of the fusion kernel
  DevBuf stage;    // contiguous host->device staging before the pitched repack
  unsigned long long wait_test_ns = 0;  // one-shot testing hook, see pct_test_wait_timeout
  int tile_set = 0;                     // register-tile set (pct_autotune / pct_set_tile_set)
  DevBuf batch_stage, batch_meta;       // pct_synthesize_batch: pitched stacks, subject table
  pct_model *model = nullptr;           // learned form (EXEC_CHOICE 7), see pct_attach_model
  float learned_conf = 0.f;             // its full-search fallback threshold
  int learned_block = 4;                // rows per proposal block along z and x
  bool learned_every_voxel = false;     // convolutions over the whole volume (diagnostic)
  int learned_level = 4;                // kept rank triples i + j + k <= level (32 offsets)
  int learned_prior_k = 0;              // > 0: EXEC_CHOICE 7 runs the no-network centre prior
  DevBuf learned;                       // its feature volumes and sums
  DevBuf tcbuf;                         // tensor-core form: 16-bit patch rows, sums, offset
  long long learned_nvox = 0;           // volume size of the last learned run (0: none yet)
  pct::learned::LearnedStreams learned_streams{};  // convolutions beside the rescoring
  cudaEvent_t learned_done = nullptr;   // recorded after the last learned run's kernels
  cudaStream_t copy_stream = nullptr;     // uploads of the pipelined host path
  cudaStream_t compute_stream = nullptr;  // its second compute stream
  cudaStream_t output_stream = nullptr;   // its combine and download by plane ranges
  std::vector<cudaEvent_t> pipe_ev;       // its fork, one per uploaded part, two joins
  bool time_kernels = false;              // pct_set_kernel_timing
  std::vector<cudaEvent_t> kt_ev;         // start / stop pairs around timed fusion launches
  size_t kt_used = 0;                     // pairs recorded since the last pct_kernel_time
  std::string last_error;
};

namespace {

int fail(pct_handle *h, int status, const std::string &msg) {
  if (h) h->last_error = msg;
  return status;
}

int cuda_fail(pct_handle *h, cudaError_t e, const char *what) {
  std::string m = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
  if (e == cudaErrorMemoryAllocation) return fail(h, PCT_ERR_OUT_OF_MEMORY, m);
  return fail(h, PCT_ERR_CUDA, m);
}

#define PCT_CUDA(h, call)                                    \
  do {                                                       \
    cudaError_t pct_e_ = (call);                             \
    if (pct_e_ != cudaSuccess) return cuda_fail(h, pct_e_, #call); \
  } while (0)

// Grow-only device buffer owned by the handle, subject to the handle's memory cap.
int ensure(pct_handle *h, DevBuf &b, size_t bytes) {
  if (b.bytes >= bytes) return PCT_OK;
  const size_t others = h->allocated - b.bytes;
  if (h->mem_limit && others + bytes > h->mem_limit)
    return fail(h, PCT_ERR_OUT_OF_MEMORY,
                "allocation of " + std::to_string(bytes) + " bytes exceeds the handle's memory limit");
  if (b.ptr) {
    cudaFree(b.ptr);
    h->allocated -= b.bytes;
    b.ptr = nullptr;
    b.bytes = 0;
  }
  void *p = nullptr;
  cudaError_t e = cudaMalloc(&p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return cuda_fail(h, e, "cudaMalloc");
  }
  b.ptr = p;
  b.bytes = bytes;
  h->allocated += bytes;
  return PCT_OK;
}

int check_choice(pct_handle *h, int exec_choice) {
  switch (exec_choice) {
    case PCT_EXEC_GM:
    case PCT_EXEC_GM2:
    case PCT_EXEC_SM:
    case PCT_EXEC_B200_FP32:
      return PCT_OK;
    case PCT_EXEC_BATCHED:
      return fail(h, PCT_ERR_UNSUPPORTED,
                  "exec_choice 8 (batched) runs through pct_synthesize_batch / pct_batch_create");
    case PCT_EXEC_LEARNED:
      if (h && (h->model || h->learned_prior_k > 0)) return PCT_OK;
      return fail(h, PCT_ERR_UNSUPPORTED,
                  "exec_choice 7 (learned proposal) needs a model attached with pct_attach_model "
                  "(or the centre prior, pct_set_learned_prior)");
    case PCT_EXEC_TC_FP16:
    case PCT_EXEC_TC_BF16:
      return PCT_OK;
    default:
      return fail(h, PCT_ERR_INVALID_ARG, "unknown exec_choice " + std::to_string(exec_choice));
  }
}

int check_shape(pct_handle *h, int nx, int ny, int nz, int num, int nh, double div,
                pct::Geometry *g) {
  if (nx <= 0 || ny <= 0 || nz <= 0 || num <= 0)
    return fail(h, PCT_ERR_INVALID_ARG, "volume sizes and atlas count must be positive");
  if (nh < 3 || (nh % 2) == 0)
    return fail(h, PCT_ERR_INVALID_ARG, "NH must be odd and >= 3, got " + std::to_string(nh));
  if (nh > 11)
    return fail(h, PCT_ERR_UNSUPPORTED, "NH > 11 is not compiled in (NH in 3..11)");
  const long long nvox = (long long)nx * ny * nz;
  if (nvox >= (1LL << 31))
    return fail(h, PCT_ERR_INVALID_ARG, "volume has 2^31 or more voxels");
  if (!(div > 0.0) || !isfinite(div))
    return fail(h, PCT_ERR_INVALID_ARG, "div must be positive and finite");
  if (!pct::make_geometry(nx, ny, nz, num, nh, g))
    return fail(h, PCT_ERR_INVALID_ARG, "bad geometry");
  return PCT_OK;
}

int select_device(pct_handle *h) {
  PCT_CUDA(h, cudaSetDevice(h->device));
  return PCT_OK;
}

constexpr size_t kMaxTimedLaunches = 4096;  // pct_set_kernel_timing: pairs kept between reads

// Zeroes the device status word and enqueues the TMA-staged fusion kernel.
int launch_fusion(pct_handle *h, const pct::Geometry &g, const pct::SlabInputs &in, float *d_out,
                  double div, cudaStream_t s) {
  int st = ensure(h, h->err, 16);
  if (st) return st;
  int *err = static_cast<int *>(h->err.ptr);
  const size_t pbytes = pct::fuse_tma_partial_bytes(g, h->tile_set);
  if (pbytes && (st = ensure(h, h->partial, pbytes))) return st;
  PCT_CUDA(h, cudaMemsetAsync(err, 0, sizeof(int), s));
  pct::LaunchHooks wt{h->wait_test_ns, nullptr, nullptr};
  h->wait_test_ns = 0;
  // (an empty interior launches nothing, so it records no pair)
  if (h->time_kernels && h->kt_used < kMaxTimedLaunches && g.ix > 0 && g.iy > 0 && g.iz > 0) {
    while (h->kt_ev.size() < 2 * (h->kt_used + 1)) {
      cudaEvent_t e = nullptr;
      PCT_CUDA(h, cudaEventCreate(&e));
      h->kt_ev.push_back(e);
    }
    wt.start = h->kt_ev[2 * h->kt_used];
    wt.stop = h->kt_ev[2 * h->kt_used + 1];
  }
  PCT_CUDA(h, pct::launch_fuse_tma(g, in, d_out, div, static_cast<float *>(h->partial.ptr), err, wt,
                                   h->tile_set, s));
  if (wt.stop) ++h->kt_used;  // a pair is read only once the launch between its events was enqueued
  return PCT_OK;
}

// Marks the end of a learned run on `s`, so that pct_learned_stats can read its counters later
// without touching the caller's stream (which may be gone by then).
int learned_ran(pct_handle *h, const pct::Geometry &g, cudaStream_t s) {
  if (!h->learned_done)
    PCT_CUDA(h, cudaEventCreateWithFlags(&h->learned_done, cudaEventDisableTiming));
  PCT_CUDA(h, cudaEventRecord(h->learned_done, s));
  h->learned_nvox = g.nvox();
  return PCT_OK;
}

// The learned form: conv features, proposal and exact rescoring over all atlases (NH = 11).
int launch_learned_path(pct_handle *h, const pct::Geometry &g, const pct::SlabInputs &in,
                        float *d_out, double div, cudaStream_t s) {
  // The network scores the 11 offsets of each axis; smaller windows keep the offsets inside them
  // (NH 7 and 9). Below 7 the interior would start fewer than 4 voxels from a face, inside the
  // reach of the network's four 3x3x3 layers.
  if (g.nh != 7 && g.nh != 9 && g.nh != 11)
    return fail(h, PCT_ERR_UNSUPPORTED,
                "exec_choice 7 (learned proposal) runs NH = 7, 9 or 11, got NH = " +
                    std::to_string(g.nh));
  if (h->learned_prior_k > 0) {
    const int window = g.nh * g.nh * g.nh;
    if (h->learned_prior_k > window)
      return fail(h, PCT_ERR_INVALID_ARG,
                  "the centre prior's k = " + std::to_string(h->learned_prior_k) +
                      " exceeds the NH^3 = " + std::to_string(window) + " window");
    if (g.ix < 4)
      return fail(h, PCT_ERR_UNSUPPORTED, "the centre prior needs at least 4 interior x-rows");
    int st = ensure(h, h->learned, pct::learned::infer_scratch_bytes(g));
    if (st) return st;
    PCT_CUDA(h, pct::learned::launch_prior(g, in, d_out, div, h->learned_prior_k, h->learned.ptr, s));
    return learned_ran(h, g, s);
  }
  if (pct::learned::model_device(h->model) != h->device)
    return fail(h, PCT_ERR_INVALID_ARG, "the attached model lives on another device");
  int st = ensure(h, h->learned, pct::learned::infer_scratch_bytes(g));
  if (st || (st = ensure(h, h->err, 16))) return st;
  int *err = static_cast<int *>(h->err.ptr);
  pct::learned::LearnedStreams &ls = h->learned_streams;
  if (!ls.aux) {
    // the convolution stream gets the higher priority, so that its CTAs take the SMs the
    // rescoring's CTAs free
    int least = 0, greatest = 0;
    PCT_CUDA(h, cudaDeviceGetStreamPriorityRange(&least, &greatest));
    PCT_CUDA(h, cudaStreamCreateWithPriority(&ls.aux, cudaStreamNonBlocking, greatest));
  }
  for (cudaEvent_t &e : ls.ev)
    if (!e) PCT_CUDA(h, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  // the confidence fallback's full search writes per-pair partial sums (NH = 11 tiles only)
  float *fb_partial = nullptr;
  if (h->learned_conf > 0.f && g.nh == 11) {
    if ((st = ensure(h, h->partial, pct::learned::fallback_partial_bytes(g)))) return st;
    fb_partial = static_cast<float *>(h->partial.ptr);
  }
  PCT_CUDA(h, cudaMemsetAsync(err, 0, sizeof(int), s));
  PCT_CUDA(h, pct::learned::launch_learned(g, pct::learned::model_weights(h->model), in, d_out, div,
                                           h->learned_conf, h->learned_block, h->learned_level,
                                           h->learned_every_voxel, h->learned.ptr, fb_partial, err,
                                           &ls, s));
  return learned_ran(h, g, s);
}

// The tensor-core form (NH = 11). Its TMA loads need 16-byte row strides: unaligned stacks are
// repacked into the handle's pitched buffers first.
int launch_tc_path(pct_handle *h, const pct::Geometry &g, const pct::SlabInputs &in, float *d_out,
                   double div, bool bf16, int16_t *dbg_top, cudaStream_t s) {
  if (g.nh != 11)
    return fail(h, PCT_ERR_UNSUPPORTED,
                "exec_choice 5/6 (tensor-core form) is built for NH = 11 only, got NH = " +
                    std::to_string(g.nh));
  int st = ensure(h, h->err, 16);
  if (st || (st = ensure(h, h->tcbuf, pct::tc::scratch_bytes(g)))) return st;
  pct::SlabInputs tin = in;
  const bool aligned = (in.pitch % 4 == 0) && (reinterpret_cast<uintptr_t>(in.atlas) % 16 == 0) &&
                       (reinterpret_cast<uintptr_t>(in.label) % 16 == 0);
  if (!aligned) {
    const int pitch = pct::slab_pitch(g.ny);
    const long long rows = (long long)g.num * g.nz * g.nx;
    const size_t bytes = (size_t)rows * pitch * sizeof(float);
    if ((st = ensure(h, h->atlas, bytes)) || (st = ensure(h, h->label, bytes))) return st;
    // copies read rows `in.pitch` floats apart
    PCT_CUDA(h, cudaMemcpy2DAsync(h->atlas.ptr, pitch * sizeof(float), in.atlas,
                                  in.pitch * sizeof(float), g.ny * sizeof(float), rows,
                                  cudaMemcpyDeviceToDevice, s));
    PCT_CUDA(h, cudaMemcpy2DAsync(h->label.ptr, pitch * sizeof(float), in.label,
                                  in.pitch * sizeof(float), g.ny * sizeof(float), rows,
                                  cudaMemcpyDeviceToDevice, s));
    tin = pct::SlabInputs{in.img, static_cast<const float *>(h->atlas.ptr),
                          static_cast<const float *>(h->label.ptr), pitch};
  }
  int *err = static_cast<int *>(h->err.ptr);
  PCT_CUDA(h, cudaMemsetAsync(err, 0, sizeof(int), s));
  PCT_CUDA(h, pct::tc::launch_tc(g, tin, d_out, div, bf16, err, dbg_top, h->tcbuf.ptr, s));
  return PCT_OK;
}

// Whether a choice runs the TMA-staged plain kernel (which needs 16-byte row strides).
bool uses_tma_rows(int exec_choice) { return exec_choice <= PCT_EXEC_B200_FP32; }

// The learned form with a confidence threshold sends low-confidence tiles to the plain kernel,
// whose TMA maps need the same 16-byte row strides.
bool needs_tma_rows(const pct_handle *h, int exec_choice) {
  return uses_tma_rows(exec_choice) ||
         (exec_choice == PCT_EXEC_LEARNED && h->learned_prior_k == 0 && h->learned_conf > 0.f);
}

int launch_path(pct_handle *h, const pct::Geometry &g, const pct::SlabInputs &in, float *d_out,
                double div, int exec_choice, cudaStream_t s) {
  if (exec_choice == PCT_EXEC_LEARNED) return launch_learned_path(h, g, in, d_out, div, s);
  if (exec_choice == PCT_EXEC_TC_FP16 || exec_choice == PCT_EXEC_TC_BF16)
    return launch_tc_path(h, g, in, d_out, div, exec_choice == PCT_EXEC_TC_BF16, nullptr, s);
  return launch_fusion(h, g, in, d_out, div, s);
}

// Reads (and clears) the device status word after `s` has drained.
int read_device_status(pct_handle *h, cudaStream_t s) {
  if (!h->err.ptr) return PCT_OK;
  int v = 0;
  PCT_CUDA(h, cudaMemcpyAsync(&v, h->err.ptr, sizeof(int), cudaMemcpyDeviceToHost, s));
  PCT_CUDA(h, cudaStreamSynchronize(s));
  if (v != 0) {
    PCT_CUDA(h, cudaMemsetAsync(h->err.ptr, 0, sizeof(int), s));
    PCT_CUDA(h, cudaStreamSynchronize(s));
    return fail(h, PCT_ERR_TIMEOUT, "a bounded device-side wait gave up (code " + std::to_string(v) + ")");
  }
  return PCT_OK;
}

// Copies host atlas volumes [num*nz*nx][ny] into a pitched device stack for TMA: one
// contiguous host->device copy (full PCIe/C2C rate) into a staging buffer, then an on-device
// repack. When ny is already a multiple of 4 the copy lands in place.
int stage_pitched_h2d(pct_handle *h, DevBuf &buf, const float *src, const pct::Geometry &g,
                      cudaStream_t s) {
  const int pitch = pct::slab_pitch(g.ny);
  const size_t rows = (size_t)g.num * g.nz * g.nx;
  int st = ensure(h, buf, rows * pitch * sizeof(float));
  if (st) return st;
  const size_t bytes = rows * g.ny * sizeof(float);
  if (pitch == g.ny) {
    PCT_CUDA(h, cudaMemcpyAsync(buf.ptr, src, bytes, cudaMemcpyHostToDevice, s));
    return PCT_OK;
  }
  if ((st = ensure(h, h->stage, bytes))) return st;
  PCT_CUDA(h, cudaMemcpyAsync(h->stage.ptr, src, bytes, cudaMemcpyHostToDevice, s));
  PCT_CUDA(h, pct::launch_pitch_copy(static_cast<const float *>(h->stage.ptr),
                                     static_cast<float *>(buf.ptr), (long long)rows, g.ny, pitch, s));
  return PCT_OK;
}

// Uploads planes [z0, z1) of atlases [a0, a1) of a host stack into the pitched device stack
// `buf`; `stage` (the same [num][nz][nx][ny] shape as the host stack) holds the contiguous copy
// before the repack when the pitch differs from ny. Whole atlases are one run of rows, a plane
// range one run per atlas.
int stage_pitched_slice(pct_handle *h, DevBuf &buf, float *stage_base, const float *src,
                        const pct::Geometry &g, int a0, int a1, int z0, int z1, bool normalize,
                        cudaStream_t s) {
  const int pitch = pct::slab_pitch(g.ny);
  const bool whole = z0 == 0 && z1 == g.nz;
  for (int a = a0; a < (whole ? a0 + 1 : a1); ++a) {
    const size_t rows = whole ? (size_t)(a1 - a0) * g.nz * g.nx : (size_t)(z1 - z0) * g.nx;
    const size_t first_row = ((size_t)a * g.nz + z0) * g.nx;
    float *dst = static_cast<float *>(buf.ptr) + first_row * pitch;
    const float *from = src + first_row * g.ny;
    const size_t bytes = rows * g.ny * sizeof(float);
    if (pitch == g.ny) {
      PCT_CUDA(h, cudaMemcpyAsync(dst, from, bytes, cudaMemcpyHostToDevice, s));
    } else {
      float *stage = stage_base + first_row * g.ny;
      PCT_CUDA(h, cudaMemcpyAsync(stage, from, bytes, cudaMemcpyHostToDevice, s));
      PCT_CUDA(h, pct::launch_pitch_copy(stage, dst, (long long)rows, g.ny, pitch, s));
    }
    if (normalize) PCT_CUDA(h, pct::launch_normalize_labels(dst, rows * pitch, s));
  }
  return PCT_OK;
}

// The host-pointer path with uploads overlapped with the fusion. The handle's copy stream
// uploads (and repacks) the subject in parts, each part's work items starting as soon as it has
// landed: the input MRI and the first atlas group in up to three plane ranges (the first holds
// the planes read by just enough z-tiles to give every CTA of the grid an item, the second as
// many z-tiles again, the third the rest), then one part per further group. The launches
// alternate between `s` and the handle's second compute stream, so that the last round of one
// launch overlaps the first round of the next. With `host_out`, the last group runs in up to
// three z-tile ranges as well (the last two as small as the first group's first), and the
// handle's output stream combines and downloads each range's planes once its items and every
// earlier launch are done, so that only the last range's combine and download follow the
// fusion; without it, the group sums are combined into d_out on `s` at the end. Every stream
// joins `s` before the call returns. Used when the plan has two or more atlas groups; returns
// PCT_ERR_UNSUPPORTED (nothing enqueued) otherwise. `normalize` applies the label normalisation
// to the CT stack on the device (the pipeline entry point). The items and the combine's group
// order are those of the one-launch path, so the result is the same bit for bit.
int fuse_pipelined(pct_handle *h, const pct::Geometry &g, const float *img, const float *atlas,
                   const float *atlas_ct, float *d_out, double div, bool normalize,
                   float *host_out, cudaStream_t s) {
  pct::FusePlanInfo pl;
  PCT_CUDA(h, pct::fuse_tma_plan(g, h->tile_set, &pl));
  if (pl.groups < 2 || h->wait_test_ns) return PCT_ERR_UNSUPPORTED;
  const int pitch = pct::slab_pitch(g.ny);
  const size_t rows = (size_t)g.num * g.nz * g.nx;
  int st;
  if ((st = ensure(h, h->atlas, rows * pitch * sizeof(float))) ||
      (st = ensure(h, h->label, rows * pitch * sizeof(float))) ||
      (st = ensure(h, h->partial, pl.partial_bytes)) || (st = ensure(h, h->err, 16)))
    return st;
  if (pitch != g.ny && ensure(h, h->stage, 2 * rows * g.ny * sizeof(float))) {
    h->last_error.clear();  // over the handle's memory cap: the one-upload path needs half
    return PCT_ERR_UNSUPPORTED;
  }
  struct Part {
    bool with_img;
    int a0, a1, z0, z1;  // upload atlases [a0, a1), planes [z0, z1) (none when z0 == z1)
    int i0, i1;          // work items that may run once it has landed
    int o0, o1;          // output planes to combine and download after it (none when o0 == o1)
  };
  std::vector<Part> parts;
  const int per = g.num / pl.groups;
  // z-tile tz holds the output planes [lo + 2 tz TZ, lo + 2 tz TZ + 2 TZ)
  auto out_plane = [&](int tz) { return tz >= pl.tiles_z ? g.nz : g.lo + 2 * pl.tz * tz; };
  const int first = std::min(pl.tiles_z, (pl.ctas + pl.tiles_xy - 1) / pl.tiles_xy);
  {
    // z-tile ends of the first group's leading parts; part k reads planes [0, planes_read(end))
    const int ends[2] = {first, std::min(pl.tiles_z, 2 * first)};
    int z0 = 0, t0 = 0;
    for (const int e : ends) {
      if (e <= t0 || e >= pl.tiles_z) continue;
      const int z1 = pct::fuse_tma_planes_read(g, pl, e);
      if (z1 >= g.nz) continue;
      parts.push_back(Part{true, 0, per, z0, z1, t0 * pl.tiles_xy, e * pl.tiles_xy, 0, 0});
      z0 = z1;
      t0 = e;
    }
    parts.push_back(Part{true, 0, per, z0, g.nz, t0 * pl.tiles_xy, pl.tiles, 0, 0});
    for (int grp = 1; grp < pl.groups - 1; ++grp)
      parts.push_back(Part{false, grp * per, (grp + 1) * per, 0, g.nz, grp * pl.tiles,
                           (grp + 1) * pl.tiles, 0, 0});
    const int last = pl.groups - 1;
    const int base = last * pl.tiles;
    if (!host_out) {
      parts.push_back(Part{false, last * per, g.num, 0, g.nz, base, base + pl.tiles, 0, 0});
    } else {
      // the last group uploads whole; its items run in z-tile ranges ending with two of `first`
      // z-tiles, each range's planes combined and downloaded after it
      const int starts[3] = {0, std::max(0, pl.tiles_z - 2 * first),
                             std::max(0, pl.tiles_z - first)};
      bool uploaded = false;
      for (int k = 0; k < 3; ++k) {
        const int t0 = starts[k], t1 = k < 2 ? starts[k + 1] : pl.tiles_z;
        if (t1 <= t0) continue;
        parts.push_back(Part{false, last * per, g.num, 0, uploaded ? 0 : g.nz,
                             base + t0 * pl.tiles_xy, base + t1 * pl.tiles_xy,
                             t0 == 0 ? 0 : out_plane(t0), out_plane(t1)});
        uploaded = true;
      }
    }
  }
  if (!h->copy_stream)
    PCT_CUDA(h, cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking));
  if (!h->compute_stream)
    PCT_CUDA(h, cudaStreamCreateWithFlags(&h->compute_stream, cudaStreamNonBlocking));
  if (host_out && !h->output_stream)
    PCT_CUDA(h, cudaStreamCreateWithFlags(&h->output_stream, cudaStreamNonBlocking));
  // events: the fork, per part its upload and its launch's completion, three joins
  const size_t nev = 1 + 2 * parts.size() + 3;
  while (h->pipe_ev.size() < nev) {
    cudaEvent_t e = nullptr;
    PCT_CUDA(h, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    h->pipe_ev.push_back(e);
  }
  const cudaStream_t cs = h->copy_stream, os = host_out ? h->output_stream : nullptr;
  const cudaStream_t lanes[2] = {s, h->compute_stream};
  int *err = static_cast<int *>(h->err.ptr);
  PCT_CUDA(h, cudaMemsetAsync(err, 0, sizeof(int), s));
  // fork: the copy stream and the other streams follow the work already on s (the output's
  // memset among it)
  PCT_CUDA(h, cudaEventRecord(h->pipe_ev[0], s));
  PCT_CUDA(h, cudaStreamWaitEvent(cs, h->pipe_ev[0], 0));
  PCT_CUDA(h, cudaStreamWaitEvent(lanes[1], h->pipe_ev[0], 0));
  if (os) PCT_CUDA(h, cudaStreamWaitEvent(os, h->pipe_ev[0], 0));
  const size_t plane = (size_t)g.nx * g.ny;
  float *stage_mri = static_cast<float *>(h->stage.ptr);
  float *stage_ct = stage_mri ? stage_mri + rows * g.ny : nullptr;
  const pct::SlabInputs in{static_cast<const float *>(h->img.ptr),
                           static_cast<const float *>(h->atlas.ptr),
                           static_cast<const float *>(h->label.ptr), pitch};
  float *partial = static_cast<float *>(h->partial.ptr);
  // (config 1 end to end: 34.0 ms with the first group uploaded whole and the group launches on
  // one stream, 29.99 ms with the parts on two streams and the download after the fusion;
  // pitched 2-D host copies of the 888-byte rows instead of the repack kernel made the uploads
  // several times slower: 82.9 ms)
  auto landed = [&](size_t k) { return h->pipe_ev[1 + 2 * k]; };
  auto done = [&](size_t k) { return h->pipe_ev[2 + 2 * k]; };
  size_t last_upload = 0;
  auto run_part = [&](size_t k) -> int {
    const Part &p = parts[k];
    if (p.z1 > p.z0) {
      if (p.with_img)
        PCT_CUDA(h, cudaMemcpyAsync(static_cast<float *>(h->img.ptr) + p.z0 * plane,
                                    img + p.z0 * plane,
                                    (size_t)(p.z1 - p.z0) * plane * sizeof(float),
                                    cudaMemcpyHostToDevice, cs));
      int r = stage_pitched_slice(h, h->atlas, stage_mri, atlas, g, p.a0, p.a1, p.z0, p.z1, false,
                                  cs);
      if (!r)
        r = stage_pitched_slice(h, h->label, stage_ct, atlas_ct, g, p.a0, p.a1, p.z0, p.z1,
                                normalize, cs);
      if (r) return r;
      PCT_CUDA(h, cudaEventRecord(landed(k), cs));
      last_upload = k;
    }
    const cudaStream_t ls = lanes[k & 1];
    PCT_CUDA(h, cudaStreamWaitEvent(ls, landed(last_upload), 0));
    PCT_CUDA(h, pct::launch_fuse_tma_items(g, in, div, partial, err, h->tile_set, p.i0, p.i1, ls));
    PCT_CUDA(h, cudaEventRecord(done(k), ls));
    return PCT_OK;
  };
  // A range's planes are complete once its launch and the other stream's launch before it are
  // (each stream runs its launches in order). Every launch is enqueued before the first download:
  // a download into pageable memory returns only when it has run.
  auto run_output = [&](size_t k) -> int {
    const Part &p = parts[k];
    PCT_CUDA(h, cudaStreamWaitEvent(os, done(k), 0));
    PCT_CUDA(h, cudaStreamWaitEvent(os, done(k - 1), 0));
    PCT_CUDA(h, pct::launch_fuse_tma_combine(g, partial, h->tile_set, d_out, p.o0, p.o1, os));
    PCT_CUDA(h, cudaMemcpyAsync(host_out + p.o0 * plane, d_out + p.o0 * plane,
                                (size_t)(p.o1 - p.o0) * plane * sizeof(float),
                                cudaMemcpyDeviceToHost, os));
    return PCT_OK;
  };
  st = PCT_OK;
  for (size_t k = 0; k < parts.size() && !st; ++k) st = run_part(k);
  for (size_t k = 1; k < parts.size() && !st; ++k)
    if (parts[k].o1 > parts[k].o0) st = run_output(k);
  // join (on failure too, so that nothing of this call is still running on the other streams
  // when the caller's next call reuses the buffers)
  const cudaStream_t others[3] = {lanes[1], cs, os};
  for (int k = 0; k < 3; ++k) {
    if (!others[k]) continue;
    const cudaEvent_t joined = h->pipe_ev[1 + 2 * parts.size() + k];
    if (st) {  // best effort: the call already failed
      if (cudaEventRecord(joined, others[k]) == cudaSuccess) cudaStreamWaitEvent(s, joined, 0);
      continue;
    }
    PCT_CUDA(h, cudaEventRecord(joined, others[k]));
    PCT_CUDA(h, cudaStreamWaitEvent(s, joined, 0));
  }
  if (st) return st;
  if (!host_out)
    PCT_CUDA(h, pct::launch_fuse_tma_combine(g, partial, h->tile_set, d_out, 0, g.nz, s));
  return PCT_OK;
}

// ---- FP64 error reduction -------------------------------------------------------------------

struct ErrAccum {
  double sum_abs;
  unsigned long long max_abs_bits;  // non-negative doubles order like their bit patterns
  unsigned long long max_rel_bits;
  unsigned long long compared, nan_mismatch, nan_both;
};

__global__ void error_stats_kernel(const float *__restrict__ a, const float *__restrict__ b, int nx,
                                   int ny, int nz, int lo, ErrAccum *acc) {
  const int ix = nx - 2 * lo, iy = ny - 2 * lo, iz = nz - 2 * lo;
  const long long total = (long long)ix * iy * iz;
  double s = 0.0, mabs = 0.0, mrel = 0.0;
  unsigned long long cmp = 0, mis = 0, both = 0;
  const double to_hu = 4095.0 / 255.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int y = (int)(i % iy) + lo;
    const long long r = i / iy;
    const int x = (int)(r % ix) + lo;
    const int z = (int)(r / ix) + lo;
    const long long k = (long long)z * nx * ny + (long long)x * ny + y;
    const float va = a[k], vb = b[k];
    const bool na = isnan(va), nb = isnan(vb);
    if (na && nb) { ++both; continue; }
    if (na || nb) { ++mis; continue; }
    const double d = fabs((double)va - (double)vb);
    s += d * to_hu;
    mabs = fmax(mabs, d * to_hu);
    mrel = fmax(mrel, d / fmax(fabs((double)vb), 1e-30));
    ++cmp;
  }
  // Warp then block reduction, one atomic set per block.
  for (int o = 16; o > 0; o >>= 1) {
    s += __shfl_down_sync(0xffffffffu, s, o);
    mabs = fmax(mabs, __shfl_down_sync(0xffffffffu, mabs, o));
    mrel = fmax(mrel, __shfl_down_sync(0xffffffffu, mrel, o));
    cmp += __shfl_down_sync(0xffffffffu, cmp, o);
    mis += __shfl_down_sync(0xffffffffu, mis, o);
    both += __shfl_down_sync(0xffffffffu, both, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&acc->sum_abs, s);
    atomicMax(&acc->max_abs_bits, (unsigned long long)__double_as_longlong(mabs));
    atomicMax(&acc->max_rel_bits, (unsigned long long)__double_as_longlong(mrel));
    atomicAdd(&acc->compared, cmp);
    atomicAdd(&acc->nan_mismatch, mis);
    atomicAdd(&acc->nan_both, both);
  }
}

// Normalised cross-correlation of two volumes over the interior voxels finite in both, from FP64
// sums (n, sum a, sum b, sum a^2, sum b^2, sum ab).
struct NccAccum {
  double s[5];
  unsigned long long n;
};

__global__ void ncc_kernel(const float *__restrict__ a, const float *__restrict__ b, int nx, int ny,
                           int nz, int lo, NccAccum *acc) {
  const int ix = nx - 2 * lo, iy = ny - 2 * lo, iz = nz - 2 * lo;
  const long long total = (long long)ix * iy * iz;
  double s[5] = {0, 0, 0, 0, 0};
  unsigned long long n = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int y = (int)(i % iy) + lo;
    const long long r = i / iy;
    const int x = (int)(r % ix) + lo;
    const int z = (int)(r / ix) + lo;
    const long long k = (long long)z * nx * ny + (long long)x * ny + y;
    const double va = a[k], vb = b[k];
    if (isnan(va) || isnan(vb)) continue;
    s[0] += va;
    s[1] += vb;
    s[2] += va * va;
    s[3] += vb * vb;
    s[4] += va * vb;
    ++n;
  }
  for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
    for (int j = 0; j < 5; ++j) s[j] += __shfl_down_sync(0xffffffffu, s[j], o);
    n += __shfl_down_sync(0xffffffffu, n, o);
  }
  if ((threadIdx.x & 31) == 0) {
#pragma unroll
    for (int j = 0; j < 5; ++j) atomicAdd(&acc->s[j], s[j]);
    atomicAdd(&acc->n, n);
  }
}

}  // namespace

namespace pct {

bool make_geometry(int nx, int ny, int nz, int num, int nh, Geometry *g) {
  if (!g || nh < 1 || (nh % 2) == 0) return false;
  g->nx = nx;
  g->ny = ny;
  g->nz = nz;
  g->num = num;
  g->nh = nh;
  g->hw = (nh - 1) / 2;
  g->lo = g->hw + 1;
  g->ix = nx - 2 * g->lo;
  g->iy = ny - 2 * g->lo;
  g->iz = nz - 2 * g->lo;
  return true;
}

}  // namespace pct

extern "C" {

int pct_abi_version(void) { return PCT_ABI_VERSION; }

const char *pct_strerror(int status) {
  switch (status) {
    case PCT_OK: return "ok";
    case PCT_ERR_INVALID_ARG: return "invalid argument";
    case PCT_ERR_CUDA: return "CUDA runtime error";
    case PCT_ERR_OUT_OF_MEMORY: return "out of device memory";
    case PCT_ERR_UNSUPPORTED: return "unsupported configuration";
    case PCT_ERR_NO_DEVICE: return "no usable sm_100 device";
    case PCT_ERR_TIMEOUT: return "device-side wait timed out";
    case PCT_ERR_INTERNAL: return "internal error";
    case PCT_ERR_TOO_LARGE: return "input larger than this entry point's fixed scratch accepts";
    default: return "unknown status";
  }
}

const char *pct_last_error_message(const pct_handle *h) { return h ? h->last_error.c_str() : ""; }

int pct_create(int device, pct_handle **out) {
  if (!out) return PCT_ERR_INVALID_ARG;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count <= 0) {
    cudaGetLastError();
    return PCT_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= count) return PCT_ERR_NO_DEVICE;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return PCT_ERR_NO_DEVICE;
  if (prop.major != 10) return PCT_ERR_NO_DEVICE;  // kernels are built for sm_100a only
  pct_handle *h = new (std::nothrow) pct_handle();
  if (!h) return PCT_ERR_OUT_OF_MEMORY;
  h->device = device;
  if (cudaSetDevice(device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    delete h;
    return PCT_ERR_CUDA;
  }
  *out = h;
  return PCT_OK;
}

int pct_destroy(pct_handle *h) {
  if (!h) return PCT_ERR_INVALID_ARG;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  for (DevBuf *b : {&h->img, &h->atlas, &h->label, &h->out, &h->scratch, &h->err, &h->partial,
                    &h->stage, &h->batch_stage, &h->batch_meta, &h->learned, &h->tcbuf})
    if (b->ptr) cudaFree(b->ptr);
  if (h->copy_stream) cudaStreamDestroy(h->copy_stream);
  if (h->compute_stream) cudaStreamDestroy(h->compute_stream);
  if (h->output_stream) cudaStreamDestroy(h->output_stream);
  if (h->learned_done) cudaEventDestroy(h->learned_done);
  if (h->learned_streams.aux) cudaStreamDestroy(h->learned_streams.aux);
  for (cudaEvent_t e : h->learned_streams.ev)
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : h->pipe_ev)
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : h->kt_ev)
    if (e) cudaEventDestroy(e);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return PCT_OK;
}

int pct_set_stream(pct_handle *h, void *stream) {
  if (!h) return PCT_ERR_INVALID_ARG;
  h->user_stream = static_cast<cudaStream_t>(stream);
  return PCT_OK;
}

int pct_set_memory_limit(pct_handle *h, size_t bytes) {
  if (!h) return PCT_ERR_INVALID_ARG;
  h->mem_limit = bytes;
  return PCT_OK;
}

int pct_tc_survivors(pct_handle *h, int exec_choice, const float *d_img, const float *d_atlas,
                     const float *d_label, float *d_out, int nx, int ny, int nz, double div,
                     int16_t *d_top, void *stream) {
  if (!h) return PCT_ERR_INVALID_ARG;
  h->last_error.clear();
  if (exec_choice != PCT_EXEC_TC_FP16 && exec_choice != PCT_EXEC_TC_BF16)
    return fail(h, PCT_ERR_INVALID_ARG, "pct_tc_survivors takes exec_choice 5 or 6");
  if (!d_img || !d_atlas || !d_label || !d_out || !d_top)
    return fail(h, PCT_ERR_INVALID_ARG, "null device pointer");
  pct::Geometry g;
  int st = check_shape(h, nx, ny, nz, 1, 11, div, &g);
  if (st || (st = select_device(h))) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const pct::SlabInputs in{d_img, d_atlas, d_label, ny};
  if ((st = launch_tc_path(h, g, in, d_out, div, exec_choice == PCT_EXEC_TC_BF16, d_top, s)))
    return st;
  return read_device_status(h, s);
}

int pct_attach_model(pct_handle *h, pct_model *m, float conf_threshold) {
  if (!h) return PCT_ERR_INVALID_ARG;
  h->last_error.clear();
  if (!(conf_threshold >= 0.f) || !isfinite(conf_threshold))
    return fail(h, PCT_ERR_INVALID_ARG, "conf_threshold must be finite and >= 0");
  if (m && pct::learned::model_device(m) != h->device)
    return fail(h, PCT_ERR_INVALID_ARG, "the model lives on another device than the handle");
  h->model = m;
  h->learned_conf = conf_threshold;
  return PCT_OK;
}

int pct_set_learned_block(pct_handle *h, int block) {
  if (!h) return PCT_ERR_INVALID_ARG;
  if (block < 1 || block > 16)
    return fail(h, PCT_ERR_INVALID_ARG, "learned proposal block must be 1..16 rows");
  h->learned_block = block;
  return PCT_OK;
}

int pct_set_learned_k(pct_handle *h, int k) {
  if (!h) return PCT_ERR_INVALID_ARG;
  if (k != 10 && k != 20 && k != 32)
    return fail(h, PCT_ERR_INVALID_ARG, "learned proposal k must be 10, 20 or 32");
  h->learned_level = k == 10 ? 2 : k == 20 ? 3 : 4;
  return PCT_OK;
}

int pct_set_learned_prior(pct_handle *h, int k) {
  if (!h) return PCT_ERR_INVALID_ARG;
  if (k < 0 || k > 125)
    return fail(h, PCT_ERR_INVALID_ARG, "centre prior k must be 0 (use the network) .. 125");
  h->learned_prior_k = k;
  return PCT_OK;
}

int pct_set_learned_convs(pct_handle *h, int every_voxel) {
  if (!h) return PCT_ERR_INVALID_ARG;
  if (every_voxel != 0 && every_voxel != 1)
    return fail(h, PCT_ERR_INVALID_ARG, "every_voxel must be 0 or 1");
  h->learned_every_voxel = every_voxel == 1;
  return PCT_OK;
}

int pct_set_kernel_timing(pct_handle *h, int on) {
  if (!h) return PCT_ERR_INVALID_ARG;
  h->time_kernels = on != 0;
  return PCT_OK;
}

int pct_kernel_time(pct_handle *h, double *ms_total, int *launches) {
  if (!h || !ms_total || !launches) return PCT_ERR_INVALID_ARG;
  h->last_error.clear();
  *ms_total = 0.0;
  *launches = 0;
  const size_t n = h->kt_used;
  h->kt_used = 0;
  if (n == 0) return PCT_OK;
  int st = select_device(h);
  if (st) return st;
  PCT_CUDA(h, cudaEventSynchronize(h->kt_ev[2 * n - 1]));
  double total = 0.0;
  for (size_t i = 0; i < n; ++i) {
    float ms = 0.f;
    PCT_CUDA(h, cudaEventElapsedTime(&ms, h->kt_ev[2 * i], h->kt_ev[2 * i + 1]));
    total += ms;
  }
  *ms_total = total;
  *launches = (int)n;
  return PCT_OK;
}

int pct_learned_stats(pct_handle *h, uint64_t *fallback_pairs, uint64_t *row_offsets) {
  if (!h) return PCT_ERR_INVALID_ARG;
  if (fallback_pairs) *fallback_pairs = 0;
  if (row_offsets) *row_offsets = 0;
  if (!h->learned_nvox) return PCT_OK;
  int st = select_device(h);
  if (st) return st;
  unsigned long long v[2] = {0, 0};
  if (h->learned_done) PCT_CUDA(h, cudaEventSynchronize(h->learned_done));
  PCT_CUDA(h, cudaMemcpyAsync(v, pct::learned::infer_counters(h->learned.ptr, h->learned_nvox),
                              sizeof(v), cudaMemcpyDeviceToHost, h->stream));
  PCT_CUDA(h, cudaStreamSynchronize(h->stream));
  if (fallback_pairs) *fallback_pairs = v[0];
  if (row_offsets) *row_offsets = v[1];
  return PCT_OK;
}

int pct_synthesize_device(pct_handle *h, const float *d_img, const float *d_atlas,
                          const float *d_atlas_label, float *d_out, int nx, int ny, int nz,
                          int num_atlas, int nh, double div, int exec_choice, void *stream) {
  if (!h) return PCT_ERR_INVALID_ARG;
  h->last_error.clear();
  if (!d_img || !d_atlas || !d_atlas_label || !d_out)
    return fail(h, PCT_ERR_INVALID_ARG, "null device pointer");
  int st = check_choice(h, exec_choice);
  if (st) return st;
  pct::Geometry g;
  st = check_shape(h, nx, ny, nz, num_atlas, nh, div, &g);
  if (st) return st;
  st = select_device(h);
  if (st) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  pct::SlabInputs in{d_img, d_atlas, d_atlas_label, g.ny};
  const bool aligned = (g.ny % 4 == 0) && (reinterpret_cast<uintptr_t>(d_atlas) % 16 == 0) &&
                       (reinterpret_cast<uintptr_t>(d_atlas_label) % 16 == 0);
  if (!aligned && needs_tma_rows(h, exec_choice)) {  // TMA needs 16-byte row strides: stage a pitched copy on the handle
    const int pitch = pct::slab_pitch(g.ny);
    const long long rows = (long long)g.num * g.nz * g.nx;
    const size_t bytes = (size_t)rows * pitch * sizeof(float);
    if ((st = ensure(h, h->atlas, bytes)) || (st = ensure(h, h->label, bytes))) return st;
    PCT_CUDA(h, pct::launch_pitch_copy(d_atlas, static_cast<float *>(h->atlas.ptr), rows, g.ny,
                                       pitch, s));
    PCT_CUDA(h, pct::launch_pitch_copy(d_atlas_label, static_cast<float *>(h->label.ptr), rows,
                                       g.ny, pitch, s));
    in = pct::SlabInputs{d_img, static_cast<const float *>(h->atlas.ptr),
                         static_cast<const float *>(h->label.ptr), pitch};
  }
  return launch_path(h, g, in, d_out, div, exec_choice, s);
}

int pct_synthesize(pct_handle *h, const float *img, const float *atlas, const float *atlas_label,
                   float *label_segmentation, int nx, int ny, int nz, int num_atlas, int nh,
                   double div, int exec_choice) {
  if (!h) return PCT_ERR_INVALID_ARG;
  h->last_error.clear();
  if (!img || !atlas || !atlas_label || !label_segmentation)
    return fail(h, PCT_ERR_INVALID_ARG, "null host pointer");
  int st = check_choice(h, exec_choice);
  if (st) return st;
  pct::Geometry g;
  st = check_shape(h, nx, ny, nz, num_atlas, nh, div, &g);
  if (st) return st;
  st = select_device(h);
  if (st) return st;
  const size_t vol = (size_t)g.nvox() * sizeof(float);
  if ((st = ensure(h, h->img, vol)) || (st = ensure(h, h->out, vol))) return st;
  cudaStream_t s = h->user_stream ? h->user_stream : h->stream;
  PCT_CUDA(h, cudaMemsetAsync(h->out.ptr, 0, vol, s));
  if (uses_tma_rows(exec_choice)) {
    // uploads overlapped with the fusion when the plan has two or more atlas groups
    st = fuse_pipelined(h, g, img, atlas, atlas_label, static_cast<float *>(h->out.ptr), div,
                        false, label_segmentation, s);
    if (st == PCT_OK) {  // the download ran by plane ranges inside, joined into s
      PCT_CUDA(h, cudaStreamSynchronize(s));
      return read_device_status(h, s);
    }
    if (st != PCT_ERR_UNSUPPORTED) return st;
    h->last_error.clear();
  }
  PCT_CUDA(h, cudaMemcpyAsync(h->img.ptr, img, vol, cudaMemcpyHostToDevice, s));
  if ((st = stage_pitched_h2d(h, h->atlas, atlas, g, s)) ||
      (st = stage_pitched_h2d(h, h->label, atlas_label, g, s)))
    return st;
  pct::SlabInputs in{static_cast<const float *>(h->img.ptr), static_cast<const float *>(h->atlas.ptr),
                     static_cast<const float *>(h->label.ptr), pct::slab_pitch(g.ny)};
  if ((st = launch_path(h, g, in, static_cast<float *>(h->out.ptr), div, exec_choice, s)))
    return st;
  PCT_CUDA(h, cudaMemcpyAsync(label_segmentation, h->out.ptr, vol, cudaMemcpyDeviceToHost, s));
  PCT_CUDA(h, cudaStreamSynchronize(s));
  return read_device_status(h, s);
}

int pct_slab_plan(int nz, int nh, int parts, int part, int *z_begin, int *z_end, int *src_begin,
                  int *src_end) {
  if (nz <= 0 || nh < 3 || (nh % 2) == 0 || parts <= 0 || part < 0 || part >= parts || !z_begin ||
      !z_end || !src_begin || !src_end)
    return PCT_ERR_INVALID_ARG;
  const int lo = (nh - 1) / 2 + 1;  // first interior plane, hw + 1
  const int planes = nz - 2 * lo > 0 ? nz - 2 * lo : 0;
  // part p gets planes [lo + floor(p*planes/parts), lo + floor((p+1)*planes/parts))
  const int b = lo + (int)((long long)part * planes / parts);
  const int e = lo + (int)((long long)(part + 1) * planes / parts);
  *z_begin = b;
  *z_end = e;
  if (b == e) {
    *src_begin = *src_end = b;
  } else {
    *src_begin = b - lo;  // the patch and search window reach lo planes past the slab
    *src_end = e + lo;
  }
  return PCT_OK;
}

int pct_query_plan(int device, int nx, int ny, int nz, int num_atlas, int nh, pct_plan *plan) {
  if (!plan) return PCT_ERR_INVALID_ARG;
  memset(plan, 0, sizeof(*plan));
  pct::Geometry g;
  int st = check_shape(nullptr, nx, ny, nz, num_atlas, nh, 1.0, &g);
  if (st) return st;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
    cudaGetLastError();
    return PCT_ERR_NO_DEVICE;
  }
  int prev = 0;
  cudaGetDevice(&prev);
  if (cudaSetDevice(device) != cudaSuccess) return PCT_ERR_NO_DEVICE;
  pct::FusePlanInfo info;
  const cudaError_t e = pct::fuse_tma_plan(g, 0, &info);
  cudaSetDevice(prev);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return PCT_ERR_CUDA;
  }
  const bool work = g.ix > 0 && g.iy > 0 && g.iz > 0;
  plan->groups = info.groups;
  plan->tiles = info.tiles;
  plan->ctas = info.ctas;
  plan->tile_rows = info.rx;
  plan->tile_planes = info.tz;
  plan->scratch_bytes = info.partial_bytes;
  plan->launches = work ? 1 + (ny % 4 != 0 ? 2 : 0) + (info.groups > 1 ? 1 : 0) : 0;
  return PCT_OK;
}

int pct_device_status(pct_handle *h, void *stream) {
  if (!h) return PCT_ERR_INVALID_ARG;
  h->last_error.clear();
  int st = select_device(h);
  if (st) return st;
  return read_device_status(h, static_cast<cudaStream_t>(stream));
}

int pct_normalize_labels_device(pct_handle *h, float *d_label, size_t n, void *stream) {
  if (!h) return PCT_ERR_INVALID_ARG;
  h->last_error.clear();
  if (!d_label && n) return fail(h, PCT_ERR_INVALID_ARG, "null device pointer");
  int st = select_device(h);
  if (st) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  PCT_CUDA(h, pct::launch_normalize_labels(d_label, n, s));
  return PCT_OK;
}

int pct_finalize_hu_device(pct_handle *h, float *d_vol, size_t n, void *stream) {
  if (!h) return PCT_ERR_INVALID_ARG;
  h->last_error.clear();
  if (!d_vol && n) return fail(h, PCT_ERR_INVALID_ARG, "null device pointer");
  int st = select_device(h);
  if (st) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  PCT_CUDA(h, pct::launch_finalize_hu(d_vol, n, s));
  return PCT_OK;
}

int pct_regularize_device(pct_handle *h, float *d_vol, int nx, int ny, int nz, int nh,
                          int64_t *fills, void *stream) {
  if (!h) return PCT_ERR_INVALID_ARG;
  h->last_error.clear();
  if (!d_vol) return fail(h, PCT_ERR_INVALID_ARG, "null device pointer");
  if (nx <= 0 || ny <= 0 || nz <= 0 || nh < 1 || (nh % 2) == 0)
    return fail(h, PCT_ERR_INVALID_ARG, "bad volume shape or NH");
  if ((long long)nx * ny * nz >= (1LL << 31))
    return fail(h, PCT_ERR_INVALID_ARG, "volume has 2^31 or more voxels");
  int st = select_device(h);
  if (st) return st;
  if ((st = ensure(h, h->scratch, pct::regularize_scratch_bytes((long long)nx * ny * nz)))) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  long long f = 0;
  int rounds = 0;
  PCT_CUDA(h, pct::launch_regularize(d_vol, nx, ny, nz, nh, h->scratch.ptr, s, &f, &rounds));
  if (fills) *fills = f;
  return PCT_OK;
}

int pct_run_pipeline(pct_handle *h, const float *img, const float *atlas_mri,
                     const float *atlas_ct_hu, float *out, int nx, int ny, int nz, int num_atlas,
                     int nh, double sigma, double beta, int exec_choice, int regularize) {
  if (!h) return PCT_ERR_INVALID_ARG;
  h->last_error.clear();
  if (!img || !atlas_mri || !atlas_ct_hu || !out)
    return fail(h, PCT_ERR_INVALID_ARG, "null host pointer");
  // div = 2*27*beta*sigma^2 (PatchBasedPseudoCT.cu:2154).
  const double div = 2.0 * 27.0 * beta * (sigma * sigma);
  int st = check_choice(h, exec_choice);
  if (st) return st;
  pct::Geometry g;
  st = check_shape(h, nx, ny, nz, num_atlas, nh, div, &g);
  if (st) return st;
  st = select_device(h);
  if (st) return st;
  const size_t vol = (size_t)g.nvox() * sizeof(float);
  if ((st = ensure(h, h->img, vol)) || (st = ensure(h, h->out, vol))) return st;
  if (regularize && (st = ensure(h, h->scratch, pct::regularize_scratch_bytes(g.nvox())))) return st;
  cudaStream_t s = h->user_stream ? h->user_stream : h->stream;
  float *d_img = static_cast<float *>(h->img.ptr), *d_out = static_cast<float *>(h->out.ptr);
  PCT_CUDA(h, cudaMemsetAsync(d_out, 0, vol, s));
  st = uses_tma_rows(exec_choice)
           ? fuse_pipelined(h, g, img, atlas_mri, atlas_ct_hu, d_out, div, true, nullptr, s)
           : PCT_ERR_UNSUPPORTED;
  if (st == PCT_ERR_UNSUPPORTED) {  // one upload, then the path
    h->last_error.clear();
    PCT_CUDA(h, cudaMemcpyAsync(d_img, img, vol, cudaMemcpyHostToDevice, s));
    if ((st = stage_pitched_h2d(h, h->atlas, atlas_mri, g, s)) ||
        (st = stage_pitched_h2d(h, h->label, atlas_ct_hu, g, s)))
      return st;
    const int pitch = pct::slab_pitch(g.ny);
    // Label normalisation over the whole pitched stack (padding columns are never read).
    PCT_CUDA(h, pct::launch_normalize_labels(static_cast<float *>(h->label.ptr),
                                             (size_t)g.num * g.nz * g.nx * pitch, s));
    pct::SlabInputs in{d_img, static_cast<const float *>(h->atlas.ptr),
                       static_cast<const float *>(h->label.ptr), pitch};
    if ((st = launch_path(h, g, in, d_out, div, exec_choice, s))) return st;
  } else if (st) {
    return st;
  }
  if ((st = read_device_status(h, s))) return st;
  if (regularize) {
    long long f = 0;
    int rounds = 0;
    PCT_CUDA(h, pct::launch_regularize(d_out, nx, ny, nz, nh, h->scratch.ptr, s, &f, &rounds));
    PCT_CUDA(h, pct::launch_finalize_hu(d_out, (size_t)g.nvox(), s));
  }
  PCT_CUDA(h, cudaMemcpyAsync(out, d_out, vol, cudaMemcpyDeviceToHost, s));
  PCT_CUDA(h, cudaStreamSynchronize(s));
  return PCT_OK;
}

int pct_ncc_device(pct_handle *h, const float *d_a, const float *d_b, int nx, int ny, int nz,
                   int nh, double *ncc, int64_t *count, void *stream) {
  if (!h) return PCT_ERR_INVALID_ARG;
  h->last_error.clear();
  if (!d_a || !d_b || !ncc) return fail(h, PCT_ERR_INVALID_ARG, "null pointer");
  if (nx <= 0 || ny <= 0 || nz <= 0 || nh < 1 || (nh % 2) == 0)
    return fail(h, PCT_ERR_INVALID_ARG, "bad volume shape or NH");
  int st = select_device(h);
  if (st) return st;
  if ((st = ensure(h, h->scratch, sizeof(NccAccum)))) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  NccAccum *acc = static_cast<NccAccum *>(h->scratch.ptr);
  PCT_CUDA(h, cudaMemsetAsync(acc, 0, sizeof(NccAccum), s));
  const int lo = (nh - 1) / 2 + 1;
  if (nx > 2 * lo && ny > 2 * lo && nz > 2 * lo) {
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device);
    ncc_kernel<<<sms * 4, 256, 0, s>>>(d_a, d_b, nx, ny, nz, lo, acc);
    PCT_CUDA(h, cudaGetLastError());
  }
  NccAccum host;
  PCT_CUDA(h, cudaMemcpyAsync(&host, acc, sizeof(host), cudaMemcpyDeviceToHost, s));
  PCT_CUDA(h, cudaStreamSynchronize(s));
  if (count) *count = (int64_t)host.n;
  const double n = (double)host.n;
  const double cov = host.s[4] - host.s[0] * host.s[1] / (n > 0 ? n : 1);
  const double va = host.s[2] - host.s[0] * host.s[0] / (n > 0 ? n : 1);
  const double vb = host.s[3] - host.s[1] * host.s[1] / (n > 0 ? n : 1);
  *ncc = (host.n > 1 && va > 0 && vb > 0) ? cov / sqrt(va * vb) : NAN;
  return PCT_OK;
}

int pct_test_wait_timeout(pct_handle *h, double timeout_ms) {
  if (!h || !(timeout_ms > 0) || timeout_ms > 60000) return PCT_ERR_INVALID_ARG;
  h->wait_test_ns = (unsigned long long)(timeout_ms * 1e6);
  return PCT_OK;
}

int pct_error_stats_device(pct_handle *h, const float *d_a, const float *d_b, int nx, int ny,
                           int nz, int nh, pct_error_stats *stats, void *stream) {
  if (!h) return PCT_ERR_INVALID_ARG;
  h->last_error.clear();
  if (!d_a || !d_b || !stats) return fail(h, PCT_ERR_INVALID_ARG, "null pointer");
  if (nx <= 0 || ny <= 0 || nz <= 0 || nh < 1 || (nh % 2) == 0)
    return fail(h, PCT_ERR_INVALID_ARG, "bad volume shape or NH");
  int st = select_device(h);
  if (st) return st;
  if ((st = ensure(h, h->scratch, sizeof(ErrAccum)))) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  ErrAccum *acc = static_cast<ErrAccum *>(h->scratch.ptr);
  PCT_CUDA(h, cudaMemsetAsync(acc, 0, sizeof(ErrAccum), s));
  const int lo = (nh - 1) / 2 + 1;
  memset(stats, 0, sizeof(*stats));
  if (nx > 2 * lo && ny > 2 * lo && nz > 2 * lo) {
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device);
    error_stats_kernel<<<sms * 4, 256, 0, s>>>(d_a, d_b, nx, ny, nz, lo, acc);
    PCT_CUDA(h, cudaGetLastError());
  }
  ErrAccum host;
  PCT_CUDA(h, cudaMemcpyAsync(&host, acc, sizeof(host), cudaMemcpyDeviceToHost, s));
  PCT_CUDA(h, cudaStreamSynchronize(s));
  double mabs, mrel;
  memcpy(&mabs, &host.max_abs_bits, sizeof(double));
  memcpy(&mrel, &host.max_rel_bits, sizeof(double));
  stats->compared = (int64_t)host.compared;
  stats->nan_mismatch = (int64_t)host.nan_mismatch;
  stats->nan_both = (int64_t)host.nan_both;
  stats->mae_hu = host.compared ? host.sum_abs / (double)host.compared : 0.0;
  stats->max_abs_hu = mabs;
  stats->max_rel = mrel;
  return PCT_OK;
}

}  // extern "C"

// ---- batched form, CUDA graph, autotuner ----------------------------------------------------

struct pct_batch {
  pct_handle *h = nullptr;
  DevBuf stage, meta, err;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  size_t bytes = 0;
};

namespace {

int check_subjects(pct_handle *h, const pct_subject *subs, int n, std::vector<pct::Geometry> &geo) {
  if (!subs || n <= 0) return fail(h, PCT_ERR_INVALID_ARG, "no subjects");
  geo.resize(n);
  for (int i = 0; i < n; ++i) {
    const pct_subject &s = subs[i];
    if (!s.img || !s.atlas || !s.atlas_label || !s.out)
      return fail(h, PCT_ERR_INVALID_ARG, "subject " + std::to_string(i) + ": null device pointer");
    int st = check_shape(h, s.nx, s.ny, s.nz, s.num_atlas, s.nh, s.div, &geo[i]);
    if (st) return st;
    if (s.nh != 7 && s.nh != 9 && s.nh != 11)
      return fail(h, PCT_ERR_UNSUPPORTED, "batched form: NH must be 7, 9 or 11");
  }
  return PCT_OK;
}

// Bytes of pitched staging the batch needs (subjects whose stacks are not TMA-ready).
size_t batch_stage_bytes(const pct_subject *subs, int n) {
  size_t total = 0;
  for (int i = 0; i < n; ++i) {
    const pct_subject &s = subs[i];
    const bool ready = (s.ny % 4 == 0) && (reinterpret_cast<uintptr_t>(s.atlas) % 16 == 0) &&
                       (reinterpret_cast<uintptr_t>(s.atlas_label) % 16 == 0);
    if (!ready)
      total += 2 * (size_t)s.num_atlas * s.nz * s.nx * pct::slab_pitch(s.ny) * sizeof(float) + 256;
  }
  return total;
}

// Enqueues the repacks of the subjects that need them into `stage` and fills `in`.
int stage_batch(pct_handle *h, const pct_subject *subs, int n, const std::vector<pct::Geometry> &geo,
                void *stage, std::vector<pct::BatchSubjectIn> &in, cudaStream_t s) {
  in.resize(n);
  unsigned char *p = static_cast<unsigned char *>(stage);
  for (int i = 0; i < n; ++i) {
    const pct_subject &sb = subs[i];
    const bool ready = (sb.ny % 4 == 0) && (reinterpret_cast<uintptr_t>(sb.atlas) % 16 == 0) &&
                       (reinterpret_cast<uintptr_t>(sb.atlas_label) % 16 == 0);
    pct::SlabInputs si{sb.img, sb.atlas, sb.atlas_label, sb.ny};
    if (!ready) {
      const int pitch = pct::slab_pitch(sb.ny);
      const long long rows = (long long)sb.num_atlas * sb.nz * sb.nx;
      const size_t bytes = (size_t)rows * pitch * sizeof(float);
      float *a = reinterpret_cast<float *>(p);
      float *l = reinterpret_cast<float *>(p + bytes);
      p += 2 * bytes + 256 - (2 * bytes) % 256;
      PCT_CUDA(h, pct::launch_pitch_copy(sb.atlas, a, rows, sb.ny, pitch, s));
      PCT_CUDA(h, pct::launch_pitch_copy(sb.atlas_label, l, rows, sb.ny, pitch, s));
      si = pct::SlabInputs{sb.img, a, l, pitch};
    }
    in[i] = pct::BatchSubjectIn{geo[i], si, sb.out, sb.div};
  }
  return PCT_OK;
}

int run_batch_once(pct_handle *h, const pct_subject *subs, int n, int set, cudaStream_t s) {
  std::vector<pct::Geometry> geo;
  int st = check_subjects(h, subs, n, geo);
  if (st) return st;
  st = select_device(h);
  if (st) return st;
  if ((st = ensure(h, h->batch_stage, batch_stage_bytes(subs, n) + 256)) ||
      (st = ensure(h, h->batch_meta, pct::batch_scratch_bytes(n))) || (st = ensure(h, h->err, 16)))
    return st;
  std::vector<pct::BatchSubjectIn> in;
  if ((st = stage_batch(h, subs, n, geo, h->batch_stage.ptr, in, s))) return st;
  int *err = static_cast<int *>(h->err.ptr);
  PCT_CUDA(h, cudaMemsetAsync(err, 0, sizeof(int), s));
  pct::BatchSetup setup;
  PCT_CUDA(h, pct::prepare_batch(in.data(), n, set, h->batch_meta.ptr, err, s, &setup));
  PCT_CUDA(h, pct::launch_prepared_batch(setup, s));
  return PCT_OK;
}

std::string batch_signature(const pct_subject *subs, int n) {
  std::vector<std::string> parts;
  for (int i = 0; i < n; ++i)
    parts.push_back(std::to_string(subs[i].nx) + "x" + std::to_string(subs[i].ny) + "x" +
                    std::to_string(subs[i].nz) + "a" + std::to_string(subs[i].num_atlas) + "n" +
                    std::to_string(subs[i].nh));
  std::sort(parts.begin(), parts.end());
  std::string sig;
  for (auto &p : parts) sig += (sig.empty() ? "" : ",") + p;
  return sig;
}

// Tuning cache: one JSON object per line {"device": ..., "signature": ..., "set": k, "ms": [...]}.
bool cache_lookup(const char *path, const std::string &device, const std::string &sig, int *set) {
  if (!path) return false;
  FILE *f = fopen(path, "r");
  if (!f) return false;
  char line[1 << 16];
  bool found = false;
  const std::string kd = "\"device\": \"" + device + "\"", ks = "\"signature\": \"" + sig + "\"";
  while (fgets(line, sizeof(line), f)) {
    const std::string l(line);
    if (l.find(kd) == std::string::npos || l.find(ks) == std::string::npos) continue;
    const size_t p = l.find("\"set\": ");
    if (p == std::string::npos) continue;
    const int v = atoi(l.c_str() + p + 7);
    if (v >= 0 && v < pct::kTileSets) {
      *set = v;
      found = true;  // the last matching line wins
    }
  }
  fclose(f);
  return found;
}

void cache_store(const char *path, const std::string &device, const std::string &sig, int set,
                 const double *ms) {
  if (!path) return;
  FILE *f = fopen(path, "a");
  if (!f) return;
  fprintf(f, "{\"device\": \"%s\", \"signature\": \"%s\", \"set\": %d, \"ms\": [", device.c_str(),
          sig.c_str(), set);
  for (int k = 0; k < pct::kTileSets; ++k) fprintf(f, "%s%.4f", k ? ", " : "", ms[k]);
  fprintf(f, "]}\n");
  fclose(f);
}

}  // namespace

extern "C" {

int pct_tile_sets(void) { return pct::kTileSets; }

int pct_set_tile_set(pct_handle *h, int set) {
  if (!h) return PCT_ERR_INVALID_ARG;
  if (set < 0 || set >= pct::kTileSets) return fail(h, PCT_ERR_INVALID_ARG, "no such tile set");
  h->tile_set = set;
  return PCT_OK;
}

int pct_get_tile_set(const pct_handle *h) { return h ? h->tile_set : PCT_ERR_INVALID_ARG; }

int pct_synthesize_batch(pct_handle *h, const pct_subject *subjects, int n, void *stream) {
  if (!h) return PCT_ERR_INVALID_ARG;
  h->last_error.clear();
  return run_batch_once(h, subjects, n, h->tile_set, static_cast<cudaStream_t>(stream));
}

int pct_batch_create(pct_handle *h, const pct_subject *subjects, int n, void *stream,
                     pct_batch **out) {
  if (!h || !out) return PCT_ERR_INVALID_ARG;
  h->last_error.clear();
  *out = nullptr;
  std::vector<pct::Geometry> geo;
  int st = check_subjects(h, subjects, n, geo);
  if (st) return st;
  if ((st = select_device(h))) return st;
  pct_batch *b = new (std::nothrow) pct_batch();
  if (!b) return PCT_ERR_OUT_OF_MEMORY;
  b->h = h;
  // Capture on the handle's own (non-blocking) stream: the legacy default stream cannot be
  // captured, and the graph does not depend on the stream it was captured on. The caller's
  // stream is drained first so the batch sees the inputs it has enqueued.
  if (stream && cudaStreamSynchronize(static_cast<cudaStream_t>(stream)) != cudaSuccess) {
    delete b;
    return fail(h, PCT_ERR_CUDA, "cudaStreamSynchronize");
  }
  if (!stream) cudaDeviceSynchronize();
  cudaStream_t s = h->stream;
  auto cleanup = [&](int code) {
    pct_batch_destroy(b);
    return code;
  };
  // The batch owns its buffers, so the graph's pointers stay valid whatever the handle does next.
  if ((st = ensure(h, b->stage, batch_stage_bytes(subjects, n) + 256)) ||
      (st = ensure(h, b->meta, pct::batch_scratch_bytes(n))) || (st = ensure(h, b->err, 16)))
    return cleanup(st);
  b->bytes = b->stage.bytes + b->meta.bytes + b->err.bytes;
  std::vector<pct::BatchSubjectIn> in;
  pct::BatchSetup setup;
  // Subject table and tensor maps are uploaded once, before capture.
  {
    std::vector<pct::BatchSubjectIn> probe;
    if ((st = stage_batch(h, subjects, n, geo, b->stage.ptr, probe, s))) return cleanup(st);
    cudaError_t e = pct::prepare_batch(probe.data(), n, h->tile_set, b->meta.ptr,
                                       static_cast<int *>(b->err.ptr), s, &setup);
    if (e != cudaSuccess) return cleanup(cuda_fail(h, e, "prepare_batch"));
  }
  // Capture: repacks, status reset, the persistent kernel.
  cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return cleanup(cuda_fail(h, e, "cudaStreamBeginCapture"));
  st = stage_batch(h, subjects, n, geo, b->stage.ptr, in, s);
  if (!st) {
    e = cudaMemsetAsync(b->err.ptr, 0, sizeof(int), s);
    if (e == cudaSuccess) e = pct::launch_prepared_batch(setup, s);
  }
  cudaGraph_t g = nullptr;
  const cudaError_t ee = cudaStreamEndCapture(s, &g);
  if (st) {
    if (g) cudaGraphDestroy(g);
    return cleanup(st);
  }
  if (e != cudaSuccess || ee != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return cleanup(cuda_fail(h, e != cudaSuccess ? e : ee, "batch capture"));
  }
  b->graph = g;
  e = cudaGraphInstantiate(&b->exec, g, 0);
  if (e != cudaSuccess) return cleanup(cuda_fail(h, e, "cudaGraphInstantiate"));
  *out = b;
  return PCT_OK;
}

int pct_batch_launch(pct_batch *b, void *stream) {
  if (!b || !b->exec) return PCT_ERR_INVALID_ARG;
  if (cudaSetDevice(b->h->device) != cudaSuccess) return PCT_ERR_CUDA;
  const cudaError_t e = cudaGraphLaunch(b->exec, static_cast<cudaStream_t>(stream));
  return e == cudaSuccess ? PCT_OK : cuda_fail(b->h, e, "cudaGraphLaunch");
}

int pct_batch_status(pct_batch *b, void *stream) {
  if (!b) return PCT_ERR_INVALID_ARG;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int v = 0;
  if (cudaMemcpyAsync(&v, b->err.ptr, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return PCT_ERR_CUDA;
  return v ? PCT_ERR_TIMEOUT : PCT_OK;
}

int pct_batch_destroy(pct_batch *b) {
  if (!b) return PCT_ERR_INVALID_ARG;
  if (b->h) cudaSetDevice(b->h->device);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  for (DevBuf *d : {&b->stage, &b->meta, &b->err})
    if (d->ptr) {
      cudaFree(d->ptr);
      if (b->h) b->h->allocated -= d->bytes;
    }
  delete b;
  return PCT_OK;
}

int pct_autotune(pct_handle *h, const pct_subject *subjects, int n, const char *cache_path,
                 double *ms_per_set, int *chosen) {
  if (!h) return PCT_ERR_INVALID_ARG;
  h->last_error.clear();
  std::vector<pct::Geometry> geo;
  int st = check_subjects(h, subjects, n, geo);
  if (st) return st;
  if ((st = select_device(h))) return st;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, h->device) != cudaSuccess) return PCT_ERR_CUDA;
  const std::string device = prop.name, sig = batch_signature(subjects, n);
  int set = 0;
  if (cache_lookup(cache_path, device, sig, &set)) {
    h->tile_set = set;
    if (chosen) *chosen = set;
    if (ms_per_set)
      for (int k = 0; k < pct::kTileSets; ++k) ms_per_set[k] = -1.0;  // not re-measured
    return PCT_OK;
  }
  cudaStream_t s = h->stream;
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
    return fail(h, PCT_ERR_CUDA, "cudaEventCreate");
  double ms[pct::kTileSets];
  int best = 0;
  for (int k = 0; k < pct::kTileSets && !st; ++k) {
    st = run_batch_once(h, subjects, n, k, s);  // warm-up
    if (!st) cudaEventRecord(e0, s);
    for (int r = 0; r < 2 && !st; ++r) st = run_batch_once(h, subjects, n, k, s);
    if (!st) {
      cudaEventRecord(e1, s);
      cudaEventSynchronize(e1);
      float t = 0;
      cudaEventElapsedTime(&t, e0, e1);
      ms[k] = t / 2.0;
      if (ms[k] < ms[best]) best = k;
      st = read_device_status(h, s);
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st) return st;
  h->tile_set = best;
  if (chosen) *chosen = best;
  if (ms_per_set)
    for (int k = 0; k < pct::kTileSets; ++k) ms_per_set[k] = ms[k];
  cache_store(cache_path, device, sig, best, ms);
  return PCT_OK;
}

}  // extern "C"
