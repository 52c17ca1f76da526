/*
 * pct_b200: B200-native (sm_100a) patch-based multi-atlas pseudo-CT synthesis.
 *
 * C ABI over libpct_b200.so. Plain pointers and sizes only; every call returns PCT_OK (0) or a
 * negative pct_status. Reference paths below are relative to the
 * EduardoAlcainBallesteros/PseudoCTImaging tree.
 *
 * Volume layout (unchanged from the reference, PatchBasedPseudoCT.cu:853-890): row-major
 * [atlas][z][x][y] with y contiguous; voxel (z,x,y) of atlas a is at a*N + z*nx*ny + x*ny + y,
 * N = nx*ny*nz. nx is MATLAB's first dimension (rows), ny its second (cols).
 *
 * Threading: a pct_handle is used by one host thread at a time. Different handles are
 * independent (no globals, unlike the reference's nx/ny/nz/num/nh).
 *
 * Streams: every `void *stream` argument is a cudaStream_t; NULL means the CUDA default stream.
 * A handle's device scratch is shared by its calls, so calls on one handle that may overlap on
 * the GPU (different streams without an ordering between them) race; order them, or use one
 * handle per stream.
 */
#ifndef PCT_B200_H
#define PCT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PCT_ABI_VERSION 1

typedef enum pct_status {
  PCT_OK = 0,
  PCT_ERR_INVALID_ARG = -1,   /* null pointer, bad size, even/too-small NH, ... */
  PCT_ERR_CUDA = -2,          /* a CUDA runtime call failed (see pct_last_error_message) */
  PCT_ERR_OUT_OF_MEMORY = -3, /* device allocation failed or exceeded the handle's cap */
  PCT_ERR_UNSUPPORTED = -4,   /* exec_choice or NH this build does not provide */
  PCT_ERR_NO_DEVICE = -5,     /* bad device index, or no sm_100 device */
  PCT_ERR_TIMEOUT = -6,       /* a bounded device-side wait gave up */
  PCT_ERR_INTERNAL = -7,
  PCT_ERR_TOO_LARGE = -8      /* input larger than a fixed-size entry point accepts */
} pct_status;

/*
 * EXEC_CHOICE values. 0/1/2 are the reference's GPU choices (PatchBasedPseudoCT.cu:71-78:
 * GM=0, GM2=1, SM=2, GpuTestTime=4); all three compute the same function, so this library runs
 * them on its plain FP32 kernel. The new choices sit in the slots the reference leaves free.
 */
typedef enum pct_exec_choice {
  PCT_EXEC_GM = 0,
  PCT_EXEC_GM2 = 1,
  PCT_EXEC_SM = 2,
  PCT_EXEC_B200_FP32 = 3, /* plain FP32 sm_100a kernel */
  PCT_EXEC_TC_FP16 = 5,   /* tensor-core FP16 correlation + top-k FP32 rescoring */
  PCT_EXEC_TC_BF16 = 6,   /* tensor-core BF16 correlation + top-k FP32 rescoring */
  PCT_EXEC_LEARNED = 7,   /* learned proposal + FP32 rescoring */
  PCT_EXEC_BATCHED = 8    /* many subjects in one persistent launch */
} pct_exec_choice;

typedef struct pct_handle pct_handle;

/* Library / error helpers. */
int pct_abi_version(void);
const char *pct_strerror(int status);
/* Message of the last failure on this handle ("" if none). Valid until the next call. */
const char *pct_last_error_message(const pct_handle *h);

/*
 * Handle lifecycle. Replaces the per-call cudaSetDevice/cudaMalloc/cudaFree of
 * MultiPatchBasedSegmentationGpu (PatchBasedPseudoCT.cu:1687-1693,1744 and main's
 * cudaSetDevice at :1988): device buffers are cached on the handle and reused across calls.
 */
int pct_create(int device, pct_handle **out);
int pct_destroy(pct_handle *h);
/* Stream used by the host-pointer calls (pct_synthesize, pct_run_pipeline); NULL restores the
 * handle's own stream. The calls still synchronise on it before returning. */
int pct_set_stream(pct_handle *h, void *stream);
/* Cap on the bytes the handle may allocate (0 = unlimited). Exceeding it returns
 * PCT_ERR_OUT_OF_MEMORY without calling the allocator. */
int pct_set_memory_limit(pct_handle *h, size_t bytes);

/*
 * Drop-in for MultiPatchBasedSegmentationGpu (PatchBasedPseudoCT.cu:1635-1750).
 * img [N], atlas [num*N], atlas_label [num*N] (already label-normalised, as the reference's
 * main does before the call, PatchBasedPseudoCT.cu:2009-2020) and label_segmentation [N] are
 * HOST buffers owned by the caller. The sizes come in as arguments instead of the reference's
 * globals nx, ny, nz, num, nh (PatchBasedPseudoCT.cu:652-654). div = 2*27*beta*sigma^2
 * (PatchBasedPseudoCT.cu:2154). As in the reference, the whole output volume is written:
 * interior voxels get product/sum_weight or NaN, border voxels 0 (the reference zeroes its
 * device buffer, :1693, and copies all of it back, :1742). Synchronous.
 */
int pct_synthesize(pct_handle *h, const float *img, const float *atlas, const float *atlas_label,
                   float *label_segmentation, int nx, int ny, int nz, int num_atlas, int nh,
                   double div, int exec_choice);

/*
 * Same computation on DEVICE buffers already resident on the handle's device, enqueued on
 * `stream` (a cudaStream_t; NULL = the CUDA default stream, as everywhere in this header). Only
 * interior voxels of d_out are written; border voxels keep whatever the caller put there. Asynchronous: errors from the
 * launch are returned, errors during execution surface at the next synchronising call.
 */
int pct_synthesize_device(pct_handle *h, const float *d_img, const float *d_atlas,
                          const float *d_atlas_label, float *d_out, int nx, int ny, int nz,
                          int num_atlas, int nh, double div, int exec_choice, void *stream);

/*
 * Waits for `stream` to drain, then reports (and clears) the status of this handle's
 * asynchronous kernels: PCT_OK, or PCT_ERR_TIMEOUT if a bounded device-side wait gave up (the
 * kernel then stopped early and its output is incomplete). pct_synthesize and pct_run_pipeline
 * check this themselves.
 */
int pct_device_status(pct_handle *h, void *stream);

/*
 * How pct_synthesize_device would run a given shape on `device` (no work is done): the kernel
 * launches it issues (fusion, pitched repack copies when ny % 4 != 0 or buffers are not 16-byte
 * aligned — assumed aligned here —, the atlas-group combine), the number of atlas groups, the
 * register tile and the persistent grid.
 */
typedef struct pct_plan {
  int launches;        /* kernel launches per call */
  int groups;          /* atlas groups (work items per tile) */
  int tiles;           /* output tiles */
  int ctas;            /* persistent CTAs launched */
  int tile_rows;       /* RX: x rows per warp */
  int tile_planes;     /* TZ: z planes per half-tile */
  size_t scratch_bytes;/* device scratch for the group partial sums */
} pct_plan;
int pct_query_plan(int device, int nx, int ny, int nz, int num_atlas, int nh, pct_plan *plan);

/*
 * Z-slab sharding of one subject over `parts` GPUs (or passes). No counterpart in the reference,
 * which runs one subject on one device. The interior planes [hw+1, nz-hw-1) (hw = (nh-1)/2) are
 * split into `parts` contiguous slabs of near-equal size; part `part` owns output planes
 * [*z_begin, *z_end) and needs input planes [*src_begin, *src_end) = the slab plus hw+1 planes on
 * each side, of the input MRI and of every atlas MRI and CT. Running pct_synthesize(_device) on
 * that sub-volume (nz' = src_end - src_begin planes) gives the slab's output planes exactly
 * where the sub-volume's interior lies, planes [z_begin - src_begin, z_end - src_begin) of the
 * sub-volume; the slabs' outputs are disjoint and together cover the whole interior. A part with
 * no planes gets z_begin == z_end and an empty source range. Pure host arithmetic.
 */
int pct_slab_plan(int nz, int nh, int parts, int part, int *z_begin, int *z_end, int *src_begin,
                  int *src_end);

/*
 * Batched form (EXEC_CHOICE 8): many subjects of uneven size, atlas count and NH in one
 * persistent kernel launch. Each subject's buffers are DEVICE buffers in the reference layout
 * (labels already normalised); only interior voxels of `out` are written. NH must be 7, 9 or 11.
 * The reference processes one subject per call (MultiPatchBasedSegmentationGpu); this has no
 * direct counterpart there.
 */
typedef struct pct_subject {
  const float *img;          /* [nz][nx][ny] */
  const float *atlas;        /* [num_atlas][nz][nx][ny] */
  const float *atlas_label;  /* [num_atlas][nz][nx][ny], normalised */
  float *out;                /* [nz][nx][ny] */
  int nx, ny, nz, num_atlas, nh;
  double div;
} pct_subject;

/* One persistent launch over all subjects, enqueued on `stream` (asynchronous; errors of the
 * bounded waits surface through pct_device_status). */
int pct_synthesize_batch(pct_handle *h, const pct_subject *subjects, int n, void *stream);

/* The same batch captured once into a CUDA graph (pitched staging copies, status reset, the
 * persistent kernel) for repeated execution on the same buffers: pct_batch_launch replays it on
 * `stream`, pct_batch_status drains `stream` and reports PCT_OK or PCT_ERR_TIMEOUT.
 * pct_batch_create drains `stream` (NULL: the device) before it captures on the handle's own
 * stream. The batch owns its device buffers; it must be destroyed before its handle. */
typedef struct pct_batch pct_batch;
int pct_batch_create(pct_handle *h, const pct_subject *subjects, int n, void *stream,
                     pct_batch **out);
int pct_batch_launch(pct_batch *b, void *stream);
int pct_batch_status(pct_batch *b, void *stream);
int pct_batch_destroy(pct_batch *b);

/*
 * Register-tile sets compiled into the library (x rows and z planes per warp for each NH). The
 * autotuner times every set on the given batch (one warm-up and two timed runs each), keeps the
 * fastest on the handle (used by every later call on it) and appends the result to the JSON-lines
 * cache `cache_path` (NULL: no cache) keyed by device name and batch shape; a cached entry is
 * reused without timing (ms_per_set then reads -1). ms_per_set has pct_tile_sets() entries.
 */
int pct_tile_sets(void);
int pct_set_tile_set(pct_handle *h, int set);
int pct_get_tile_set(const pct_handle *h);
int pct_autotune(pct_handle *h, const pct_subject *subjects, int n, const char *cache_path,
                 double *ms_per_set, int *chosen);

/*
 * Device time of the plain path's fusion kernel (EXEC_CHOICE 0-3 through pct_synthesize_device,
 * or pct_synthesize when it uploads in one piece): while timing is on, CUDA events are recorded
 * on the call's stream right before and after each fusion launch (the group combine and the
 * repack are outside). pct_kernel_time waits for the last of them and returns the launches
 * timed since the previous read and their summed device time in milliseconds, then starts over.
 * At most 4096 launches are kept between reads; later ones run untimed. No counterpart in the
 * reference (its timing is host wall clock around the whole call).
 */
int pct_set_kernel_timing(pct_handle *h, int on);
int pct_kernel_time(pct_handle *h, double *ms_total, int *launches);

/*
 * Learned-proposal form (EXEC_CHOICE 7), training side. The model is a small 3D CNN over the
 * co-located 9x9x9 patches of the input MRI and one atlas MRI (conv 2->16, 3 x conv 16->16, all
 * 3x3x3 valid + ReLU, then three linear heads 16->11 scoring dw, du and dv); it proposes, per
 * (voxel, atlas), the 32 offsets of the 11^3 window with the largest p_w*p_u*p_v. No counterpart
 * in the reference. Weights are BF16 for the forward pass, with FP32 master weights and Adam.
 *
 * A training set is a list of samples (subject, atlas, voxel) over device-resident subjects; its
 * targets are computed on the GPU from the plain method: the exact FP32 SSD of all 11^3 offsets,
 * the 32 smallest, turned into one distribution per axis (the share of the 32 with each dw, du,
 * dv). Every sample voxel must be at least 6 voxels from each face of its volume.
 */
typedef struct pct_model pct_model;
typedef struct pct_train_set pct_train_set;
typedef struct pct_train_subject {
  const float *img;    /* device [nz][nx][ny] input MRI */
  const float *atlas;  /* device [num_atlas][nz][nx][ny] atlas MRIs */
  int nx, ny, nz, num_atlas;
} pct_train_subject;

int pct_model_num_params(void);
/* Deterministic He-normal initialisation from `seed`. */
int pct_model_create(int device, uint64_t seed, pct_model **out);
int pct_model_destroy(pct_model *m);
const char *pct_model_last_error(const pct_model *m);
/* FP32 master weights in and out (pct_model_num_params floats); setting resets Adam. With
 * inference_precision != 0 the BF16 weights the kernels use are returned (as floats). */
int pct_model_set_params(pct_model *m, const float *params);
int pct_model_get_params(pct_model *m, float *params, int inference_precision);
/* Checkpoint files: a 16-byte header ("PCTLRN01", uint32 parameter count, uint32 0) and the FP32
 * master weights, little-endian, in the flat parameter order. Loading resets Adam. */
int pct_model_load_file(pct_model *m, const char *path);
int pct_model_save_file(pct_model *m, const char *path);

/* samples: host array [n][3] of (subject index, atlas index, flat voxel index). */
int pct_train_set_create(int device, const pct_train_subject *subjects, int nsub,
                         const int *samples, int n, pct_train_set **out);
/* Per-axis targets [n][33] and the plain method's top-32 offsets [n][32] (index
 * (dw+5)*121 + (du+5)*11 + (dv+5)); either pointer may be NULL. */
int pct_train_set_targets(pct_train_set *ts, float *targets, int16_t *top);
int pct_train_set_destroy(pct_train_set *ts);

/* Mean gradient and loss of samples [begin, begin+count) without updating the model. */
int pct_model_gradients(pct_model *m, pct_train_set *ts, int begin, int count, float *grad,
                        float *loss);
/* `steps` Adam steps on consecutive batches of the (caller-shuffled) samples, wrapping around
 * at the end of the set; *mean_loss receives the mean per-sample loss over those steps. */
int pct_model_train(pct_model *m, pct_train_set *ts, int batch, int steps, float lr,
                    float *mean_loss);

/*
 * Learned-proposal form, inference side. pct_attach_model makes EXEC_CHOICE 7 available on the
 * handle's pct_synthesize / pct_synthesize_device / pct_run_pipeline calls (NH 7, 9 or 11; the
 * model must live on the handle's device and outlive its use; m = NULL detaches). Per atlas and
 * per row segment of 30 interior voxels along y, the network's per-axis offset probabilities
 * of the segment's voxels are summed (for NH 7 and 9 each axis's softmax runs over the offsets
 * inside the window only); the 4 most probable offsets per axis are kept and, of their
 * 64 combinations, the 32 whose per-axis ranks sum to at most 4 (ties: lower offset first). Only
 * those 32 offsets get the exact FP32 SSD and a weight. A voxel whose own probability mass
 * (p_w*p_u*p_v summed over the 32) is below `conf_threshold` falls back to all NH^3 offsets for
 * that atlas. conf_threshold = 0 never falls back; a threshold above 1 always does (every
 * candidate, as the plain method). Output: the same interior, border and NaN rule as the plain
 * method (voxels (NH+1)/2 or more from every face). No counterpart in the reference.
 */
int pct_attach_model(pct_handle *h, pct_model *m, float conf_threshold);
/* Proposal sharing (default 4): row segments share the proposal of their block's anchor row,
 * blocks of `block` x `block` rows in (z, x) anchored at their middle row; the network's heads
 * and the proposal run only on anchor rows (each convolution only on the rows, planes and y its
 * successors need for them), and a voxel's confidence is that of the anchor-row voxel at the
 * same y. 1 = every
 * row segment proposes for itself. Blocks start at the volume's first interior plane and row, so
 * z-slab shards reproduce the whole volume's result when their boundaries are multiples of
 * `block` interior planes apart. */
int pct_set_learned_block(pct_handle *h, int block);
/* Diagnostic (default 0): 1 = the learned form's convolutions compute every voxel of the volume
 * instead of only the outputs the anchor rows need (conv4 on the anchor rows, conv(4 - r) within
 * r rows and planes of them, interior y widened by r). The result is bit-identical; this is the
 * check of the restricted plan. No counterpart in the reference. */
int pct_set_learned_convs(pct_handle *h, int every_voxel);
/* Size of the kept set (default 32): from the 4 most probable offsets per axis, the rank triples
 * (i, j, k) with i + j + k <= 4 (k = 32), <= 3 (k = 20) or <= 2 (k = 10) are rescored exactly;
 * the confidence test uses the probability mass of the same set. Fewer offsets trade accuracy
 * for speed. No counterpart in the reference. */
int pct_set_learned_k(pct_handle *h, int k);

/*
 * The proposal baseline without a network, for measuring what the network gains: with k > 0,
 * EXEC_CHOICE 7 runs no convolutions and no proposal kernel and needs no attached model; every
 * voxel rescores the same k offsets, those of the NH^3 window nearest its centre (by squared
 * distance, ties in (dw, du, dv) order), with the learned form's exact FP32 rescoring; no
 * confidence fallback. k = 0 (the default) uses the attached network. 0 <= k <= 125. No
 * counterpart in the reference (its search is always the full window,
 * NewPatchedBrainPureC.cpp:1283-1331).
 */
int pct_set_learned_prior(pct_handle *h, int k);

/*
 * Tensor-core form (EXEC_CHOICE 5 = FP16, 6 = BF16; NH = 11) runs through pct_synthesize /
 * pct_synthesize_device / pct_run_pipeline. Per (voxel, atlas) the SSD of all 11^3 positions is
 * ranked by a tcgen05 correlation of 16-bit patches (the tile's mean removed, scaled by 1/64,
 * FP32 accumulation, |b|^2/2 of the rounded patch folded in as 16-bit parts), the 16 best are
 * rescored with the exact FP32 SSD and only they are weighted. Same interior, border and NaN rule
 * as the plain method. No counterpart in the reference (its GPU kernels are FP64).
 *
 * Testing hook: one atlas (num_atlas = 1) through the tensor-core form, writing d_out as above and
 * the 16 survivors of every interior voxel, best first, into d_top (device int16 [nz*nx*ny][16],
 * offset index (dw+5)*121 + (du+5)*11 + (dv+5)). Synchronous on `stream`.
 */
int pct_tc_survivors(pct_handle *h, int exec_choice, const float *d_img, const float *d_atlas,
                     const float *d_label, float *d_out, int nx, int ny, int nz, double div,
                     int16_t *d_top, void *stream);
/* Counters of the handle's last learned run (synchronises the stream that run used): the
 * (voxel, atlas) pairs that took the full search, and the offsets evaluated summed over warp
 * rows (one row = 30 output voxels of one atlas; the plain method evaluates 1331 per row).
 * Either pointer may be NULL. */
int pct_learned_stats(pct_handle *h, uint64_t *fallback_pairs, uint64_t *row_offsets);
/* Testing hook: for one (input, atlas) pair (d_img, d_atlas: one device volume each,
 * [nz][nx][ny]) at n voxels given by flat index, the 16 conv4 features (after ReLU, as the
 * inference kernels keep them in BF16) into features [n][16], the proposal's 4 offsets per axis
 * in rank order (dw, du, dv; values -5..5) into top [n][12], and its confidence into conf [n].
 * Any output pointer may be NULL. Synchronous. */
int pct_model_probe(pct_model *m, const float *d_img, const float *d_atlas, int nx, int ny, int nz,
                    const int64_t *voxels, int n, float *features, int8_t *top, float *conf);

/* In-place CT -> label scale L' = 255*((L+1024)/4095) on a device buffer of n floats
 * (PatchBasedPseudoCT.cu:2009-2020, NewPatchedBrainPureC.cpp:1583-1593). */
int pct_normalize_labels_device(pct_handle *h, float *d_label, size_t n, void *stream);

/*
 * Post-processing after the path, on a device volume in label scale:
 * RegularizationStep (NewPatchedBrainPureC.cpp:1059-1106; PatchBasedPseudoCT.cu:1501-1595):
 * every interior NaN becomes the median of the non-NaN values of its 3x3x3 neighbourhood,
 * filled in the reference's sequential z,x,y order (a voxel sees the fills of voxels before it).
 * nh gives the interior, as in the reference. *fills (optional) receives the number of fills.
 */
int pct_regularize_device(pct_handle *h, float *d_vol, int nx, int ny, int nz, int nh,
                          int64_t *fills, void *stream);

/*
 * Allocation-free variant of pct_regularize_device, for callers that may not allocate GPU memory
 * while running (for example applications whose device memory belongs to their own pool
 * allocator, or latency-critical loops that forbid allocation after start-up). No counterpart in
 * the reference. Same result as pct_regularize_device; needs no handle and calls no allocator:
 * its scratch is a fixed 64 MiB array inside the library, held by every GPU that loads the
 * library until the process exits. Volumes of more than 2^23 voxels (8,388,608) are rejected
 * with PCT_ERR_TOO_LARGE. Runs on the current device. CUDA loads the library's device code
 * lazily, so the array is reserved on a device by the first call of this entry point (or of any
 * other kernel of the library) there: make that first call at start-up, before the caller's pool
 * takes the device memory and before any stream capture, or set CUDA_MODULE_LOADING=EAGER. Every
 * call looks up the array's device address on the current device. Calls share the array: calls
 * whose work overlaps on the GPU race and must be issued one after another.
 * Synchronous on `stream`.
 */
int pct_regularize_device_noalloc(float *d_vol, int nx, int ny, int nz, int nh, int64_t *fills,
                                  void *stream);

/* RoundMatrix then the HU map round(4095*(v/255)) - 1024 over all n voxels
 * (NewPatchedBrainPureC.cpp:1221-1227,1732-1738; PatchBasedPseudoCT.cu:2173-2179). */
int pct_finalize_hu_device(pct_handle *h, float *d_vol, size_t n, void *stream);

/*
 * The reference's main() flow for one subject (PatchBasedPseudoCT.cu:2009-2020,2152-2180), on
 * host buffers: label normalisation of atlas_ct_hu (copied, not modified), the path
 * (exec_choice), then, if `regularize` is non-zero, RegularizationStep, RoundMatrix and the
 * map back to HU. out receives N floats (HU if regularize, else label scale).
 */
int pct_run_pipeline(pct_handle *h, const float *img, const float *atlas_mri,
                     const float *atlas_ct_hu, float *out, int nx, int ny, int nz, int num_atlas,
                     int nh, double sigma, double beta, int exec_choice, int regularize);

/*
 * FP64 comparison of two device volumes over the interior of an NH window, in HU
 * (HU = v*4095/255 - 1024 applied to both). NaN in exactly one of the two counts as a mask
 * mismatch and is excluded from the error sums; NaN in both is skipped.
 */
typedef struct pct_error_stats {
  double mae_hu;          /* mean |a-b| in HU over voxels finite in both */
  double max_abs_hu;      /* max |a-b| in HU */
  double max_rel;         /* max |a-b| / max(|b|, 1e-30), label scale */
  int64_t compared;       /* voxels finite in both */
  int64_t nan_mismatch;   /* NaN in exactly one */
  int64_t nan_both;       /* NaN in both */
} pct_error_stats;
int pct_error_stats_device(pct_handle *h, const float *d_a, const float *d_b, int nx, int ny,
                           int nz, int nh, pct_error_stats *stats, void *stream);

/*
 * Volume files of the drop-in command line (host, no GPU). MatrixIO text format of the reference
 * (MatrixIO<T>::Read/Store, PatchBasedPseudoCT.cu:679-809): header lines num, rows (nx), cols
 * (ny), depth (nz), then the values in [num][depth][rows][cols] order. dims[] = {num, rows, cols,
 * depth}. pct_matrixio_read expects n = the product of the header. The raw form is a plain
 * float32 dump of the same layout.
 */
int pct_matrixio_dims(const char *path, int dims[4]);
int pct_matrixio_read(const char *path, float *out, size_t n);
int pct_matrixio_write(const char *path, const float *data, int num, int rows, int cols, int depth);
int pct_raw_read(const char *path, float *out, size_t n);
int pct_raw_write(const char *path, const float *data, size_t n);

/*
 * MATLAB level-5 MAT-files, the reference's data and result files (ReadMatFile / FindDimension /
 * WriteOutputMatFile, PatchBasedPseudoCT.cu:1047-1370; read there through MATLAB's libmat).
 * A data file holds `img` ([nx ny nz] single) and the structs `atlas` and `atlas_label` whose
 * fields are the atlases' [nx ny nz] single volumes, atlas i = field i. pct_mat_dims gives
 * {num, nx, ny, nz}; pct_mat_read fills img (n_img = nx*ny*nz) and the atlas MRI and CT stacks
 * (n_atlas = num*nx*ny*nz) in this library's [atlas][z][x][y] layout (x = MATLAB dimension 1,
 * y = dimension 2, as the reference's ConvertToRowBased). Compressed (level-7) elements are
 * read; little-endian files only. pct_mat_write stores one [nx ny nz] single variable named
 * `variable` (uncompressed), from the [z][x][y] layout. PCT_ERR_INVALID_ARG for unreadable or
 * malformed files and for sizes that do not match.
 */
int pct_mat_dims(const char *path, int dims[4]);
int pct_mat_read(const char *path, float *img, float *atlas_mri, float *atlas_ct, size_t n_img,
                 size_t n_atlas);
int pct_mat_write(const char *path, const char *variable, const float *vol, int nx, int ny,
                  int nz);

/*
 * Normalised cross-correlation of two device volumes over the interior of an NH window, counting
 * only voxels finite in both (FP64 sums); the quality measure the reference reports for its
 * pseudo-CTs against the real CT (imgs/Correlation.png). *ncc is NaN if fewer than two voxels
 * qualify or either volume is constant there. *count (optional) receives the voxels used.
 */
int pct_ncc_device(pct_handle *h, const float *d_a, const float *d_b, int nx, int ny, int nz,
                   int nh, double *ncc, int64_t *count, void *stream);

/*
 * Testing hook for failure detection (no GPU fault involved): the next fusion launch on this
 * handle has its first CTA withhold the copies its first wait expects, so that bounded wait runs
 * out after timeout_ms; the CTA records the timeout and stops, and the call reports
 * PCT_ERR_TIMEOUT (pct_device_status for the asynchronous entry point). One-shot. The device
 * context stays usable.
 */
int pct_test_wait_timeout(pct_handle *h, double timeout_ms);

/*
 * Seeded synthetic subject (host). Input MRI = sum of n_blobs Gaussian blobs (amplitude
 * U[amp_lo,amp_hi], isotropic std U[std_lo,std_hi] voxels) + N(0, mri_noise). Atlas a: the
 * noise-free input resampled (trilinear) through a smooth random displacement field whose
 * largest displacement is max_disp voxels, + fresh N(0, mri_noise); its CT is a fixed
 * piecewise-linear MRI->HU map of that resampled image, clipped to [-1000, 2000], + N(0,
 * ct_noise). Deterministic in `seed` regardless of thread count. Any output pointer may be NULL.
 */
typedef struct pct_synth_params {
  int nx, ny, nz, num_atlas;
  int n_blobs;
  float amp_lo, amp_hi;
  float std_lo, std_hi;
  float mri_noise;
  float ct_noise;
  float max_disp;
  uint64_t seed;
} pct_synth_params;
int pct_synth_default_params(pct_synth_params *p, int nx, int ny, int nz, int num_atlas,
                             int n_blobs, uint64_t seed);
int pct_synth_generate(const pct_synth_params *p, float *img, float *atlas_mri,
                       float *atlas_ct_hu);

#ifdef __cplusplus
}
#endif

#endif /* PCT_B200_H */
