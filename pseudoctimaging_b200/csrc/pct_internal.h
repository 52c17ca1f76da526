// Internal declarations shared by the CUDA translation units of libpct_b200.so.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

struct pct_model;

namespace pct {

// Half window and interior of one subject, as in the reference (NewPatchedBrainPureC.cpp:1263-1265):
// a voxel is interior when every coordinate c satisfies hw+1 <= c < n-hw-1.
struct Geometry {
  int nx, ny, nz, num, nh, hw;
  int lo;                 // first interior index, hw + 1
  int ix, iy, iz;         // interior extents (may be <= 0: nothing to compute)
  long long nvox() const { return (long long)nx * ny * nz; }
};

bool make_geometry(int nx, int ny, int nz, int num, int nh, Geometry *g);

// Inputs of the TMA-staged kernel: the input MRI in the reference layout, and the atlas MRI and
// CT stacks [num][nz][nx][pitch] with pitch >= ny, pitch % 4 == 0 and 16-byte aligned bases
// (TMA needs 16-byte row strides).
struct SlabInputs {
  const float *img;
  const float *atlas;
  const float *label;
  int pitch;
};

// TMA-staged plain FP32 fusion. Writes interior voxels of out only. *err (device) is set to a
// non-zero code if a bounded wait gave up; the caller zeroes it beforehand. When the planner
// splits the atlases into groups (to fill the persistent grid), `partial` must point to
// fuse_tma_partial_bytes(g) bytes of device scratch; otherwise it may be null.
// Hooks of one fusion launch. Testing hook for the bounded waits: when timeout_ns != 0, the first
// CTA withholds its first copies, so its wait runs out after timeout_ns and the launch reports a
// timeout. Timing hook: non-null start / stop events are recorded on the stream right before and
// after the fusion kernel (not the group combine).
struct LaunchHooks {
  unsigned long long timeout_ns;
  cudaEvent_t start, stop;
};

// Tile-shape sets compiled into the library (chosen per handle, see pct_autotune).
constexpr int kTileSets = 5;
size_t fuse_tma_partial_bytes(const Geometry &g, int set);
struct FusePlanInfo {
  int groups, tiles, ctas, rx, tz;
  size_t partial_bytes;
  int tiles_z, tiles_xy;  // tiles are numbered z-major: tile t has z-tile t / tiles_xy
};
cudaError_t fuse_tma_plan(const Geometry &g, int set, FusePlanInfo *info);
cudaError_t launch_fuse_tma(const Geometry &g, const SlabInputs &in, float *out, double div,
                            float *partial, int *err, const LaunchHooks &wt, int set,
                            cudaStream_t stream);
// Pipelined form of the same (plans with 2 or more atlas groups only): the work items
// [item_begin, item_end) into the partial sums (item = group * tiles + tile);
// launch_fuse_tma_combine adds the groups into out once every item has run. Lets the host start
// on the first planes of the first group while the rest is uploaded.
cudaError_t launch_fuse_tma_items(const Geometry &g, const SlabInputs &in, double div,
                                  float *partial, int *err, int set, int item_begin, int item_end,
                                  cudaStream_t stream);
// Planes [0, n) of the input and atlas volumes that the items of z-tiles [0, ztiles) read.
int fuse_tma_planes_read(const Geometry &g, const FusePlanInfo &info, int ztiles);
// The combine of the output planes [z_begin, z_end) (clipped to the interior).
cudaError_t launch_fuse_tma_combine(const Geometry &g, const float *partial, int set, float *out,
                                    int z_begin, int z_end, cudaStream_t stream);

// Tiles of the plain kernel as the learned form's fallback sees them (NH = 11, tile set 0): tile
// t = (tz * tiles_x + tx) * tiles_y + ty covers interior y [30 ty, 30 ty + 30), x rows
// [xc tx, xc tx + xc) and z planes [zt tz, zt tz + zt), counted from the first interior voxel.
struct TileShape {
  int out_y, xc, zt;
  int tiles_y, tiles_x, tiles_z;
};
TileShape fuse_tile_shape(const Geometry &g);
// The plain full search (NH = 11) of the flagged (tile, atlas) pairs of up to 32 atlases: bit i
// of masks[t] flags atlas atlas_base + i for tile t. Lists one item per two flagged atlases of a
// tile in `items` (room for 16 per tile; its length in *count), runs them into `partial` (slot
// k of a tile holds its k-th pair's sums: 2 floats per voxel and slot, up to 16 slots), then adds
// the slots of every interior voxel of a flagged tile into acc_p / acc_w in pair order.
cudaError_t launch_fuse_masked(const Geometry &g, const SlabInputs &in, double div, int atlas_base,
                               const uint32_t *masks, int *items, int *count, float *partial,
                               float *acc_p, float *acc_w, int *err, cudaStream_t stream);

// Batched form: many subjects (NH 7/9/11), one persistent launch.
struct BatchSubjectIn {
  Geometry geom;
  SlabInputs in;   // pitched atlas stacks (TMA-ready)
  float *out;
  double div;
};
struct BatchSetup {
  bool params_ready = false;
  int items = 0, blocks = 0, smem = 0, set = 0;
  void *bp_subjects = nullptr;
  int bp_nsub = 0;
  int *bp_err = nullptr;
};
size_t batch_scratch_bytes(int n);
// Plans the batch and uploads its subject table and tensor maps to dev_scratch (synchronous).
cudaError_t prepare_batch(const BatchSubjectIn *subs, int n, int set, void *dev_scratch, int *err,
                          cudaStream_t stream, BatchSetup *setup);
// Enqueues the persistent batch kernel (graph-capturable: no host work beyond the launch).
cudaError_t launch_prepared_batch(const BatchSetup &setup, cudaStream_t stream);

// dst[r*pitch + c] = src[r*ny + c] for r < rows, c < ny.
cudaError_t launch_pitch_copy(const float *src, float *dst, long long rows, int ny, int pitch,
                              cudaStream_t stream);

inline int slab_pitch(int ny) { return (ny + 3) / 4 * 4; }

// Run-time compiled kernels (NVRTC; pct_jit.cpp): the entry point `entry_name` of `source`
// built for the current device with `options` (typically -D constants), cached per (context,
// source name, options, entry point). nullptr when NVRTC or the driver's module calls are
// unavailable, the build failed, or it is not built yet and `build` is false (a lookup only);
// callers then launch their ahead-of-time build.
namespace jit {
void *kernel(const char *source, const char *file_name, const std::vector<std::string> &options,
             const char *entry_name, bool build = true);
// 1-D launch of a kernel returned by kernel() (no dynamic shared memory).
cudaError_t launch(void *fn, unsigned grid, unsigned block, cudaStream_t stream, void **args);
}  // namespace jit

// cuTensorMapEncodeTiled of the driver (a PFN_cuTensorMapEncodeTiled_v12000), found through the
// runtime's entry-point query; NULL if the driver does not provide it.
void *tensor_map_encoder();

// NaN median fill (synchronous on `stream`: it reads back a counter after each round).
// scratch must hold regularize_scratch_bytes(nx*ny*nz) bytes.
size_t regularize_scratch_bytes(long long nvox);
cudaError_t launch_regularize(float *vol, int nx, int ny, int nz, int nh, void *scratch,
                              cudaStream_t stream, long long *fills_out, int *rounds_out);

cudaError_t launch_normalize_labels(float *label, size_t n, cudaStream_t stream);
cudaError_t launch_finalize_hu(float *vol, size_t n, cudaStream_t stream);

namespace learned {
// Learned-proposal inference (NH = 11). `weights` are the model's BF16 parameters on the device.
size_t infer_scratch_bytes(const Geometry &g);
// Two device counters: (voxel, atlas) pairs that fell back, offsets evaluated by warp rows.
unsigned long long *infer_counters(void *scratch, long long nvox);
// *err (device) is set to a non-zero code if a bounded wait of the convolution pipeline gives up.
// Rows of voxels share the proposal of their block's anchor row: blocks of `block` x `block`
// rows in (z, x) (1 = every row segment proposes for itself); the kept set of a proposal is the
// rank triples with i + j + k <= level (2, 3, 4: 10, 20, 32 offsets). The convolutions compute
// only the outputs the anchor rows need unless `every_voxel` (same result).
// With `streams` (an auxiliary stream and 5 events), each atlas's convolutions and proposal run
// on the auxiliary stream while the previous atlas is rescored on `s` (two proposal tables in
// the scratch); without it everything runs on `s`.
struct LearnedStreams {
  cudaStream_t aux;
  cudaEvent_t ev[5];  // fork, proposal ready [2], rescoring done [2]
};
// A confidence threshold > 0 sends the low-confidence voxels' tiles of the plain kernel to its
// full search (NH = 11, 16-byte aligned atlas rows) when `fb_partial` holds
// fallback_partial_bytes(g) of device memory; otherwise (or with other windows) the rescoring
// runs the whole window for low-confidence rows itself.
size_t fallback_partial_bytes(const Geometry &g);
cudaError_t launch_learned(const Geometry &g, const void *weights, const SlabInputs &in, float *out,
                           double div, float conf_thr, int block, int level, bool every_voxel,
                           void *scratch, float *fb_partial, int *err,
                           const LearnedStreams *streams, cudaStream_t s);
// The proposal baseline without a network (no convolutions, no proposal kernel): every voxel
// rescores the k offsets of the window nearest its centre (1 <= k <= 125), with the same exact
// FP32 rescoring as the learned form. Writes the interior of out.
cudaError_t launch_prior(const Geometry &g, const SlabInputs &in, float *out, double div, int k,
                         void *scratch, cudaStream_t s);
cudaError_t learned_probe(const Geometry &g, const void *weights, const float *img,
                          const float *atlas_a, void *scratch, const int64_t *voxels, int n,
                          float *features, signed char *top, float *conf, cudaStream_t s);
const void *model_weights(const pct_model *m);
int model_device(const pct_model *m);
}  // namespace learned

namespace tc {
// Tensor-core form (NH = 11): FP16 or BF16 correlation on tcgen05, top-16 per (voxel, atlas),
// exact FP32 rescoring. Writes interior voxels of out. *err (device) is set if a bounded wait
// gives up. dbg_top (optional, device [nvox][16]) receives atlas 0's survivors per voxel. The
// atlas stacks must be TMA-ready (pitch % 4 == 0, 16-byte aligned); scratch holds
// scratch_bytes(g) bytes (one atlas's 16-bit patch rows, the sums, the subject's offset).
size_t scratch_bytes(const Geometry &g);
cudaError_t launch_tc(const Geometry &g, const SlabInputs &in, float *out, double div, bool bf16,
                      int *err, int16_t *dbg_top, void *scratch, cudaStream_t s);
}  // namespace tc

}  // namespace pct
