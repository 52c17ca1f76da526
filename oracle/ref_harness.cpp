// C entry points over the reference's own CPU implementation, for use as the parity oracle.
//
// TEST INFRASTRUCTURE ONLY. This file is compiled together with the UNMODIFIED reference source
// src/CPU/NewPatchedBrainPureC.cpp (read in place from the reference checkout by oracle/Makefile,
// never copied) into oracle/_ref/libpctref.so. Only tests/, the smoke check and bench.py's CPU
// baseline arm load that library, and only as the checker or the timed CPU baseline.
//
// The reference routines take their volume sizes and the input image from globals
// (NewPatchedBrainPureC.cpp:76-82) and read the global `im`, not their `img` parameter
// (NewPatchedBrainPureC.cpp:1316,1428), so each entry point sets those globals first. The
// globals make the library non-reentrant: callers must serialise calls.
#include <omp.h>

#include <iostream>
#include <sstream>

// Globals and routines defined by NewPatchedBrainPureC.cpp (C++ linkage).
extern float *im;
extern float *atlas;
extern float *label;
extern int nx, ny, nz;
extern int num, nh;
void MultiAtlasPatchBasedSegmentation(const float *img, const float *atlas, const float *atlas_label,
                                      float *labeled_img, const double div);
void MultiAtlasPatchBasedSegmentationOpenMP(const float *img, const float *atlas,
                                            const float *atlas_label, float *labeled_img,
                                            const double div);
void RegularizationStep(const int half_window, const int half_patch, const int nx, const int ny,
                        const int nz, float *segmentationArray);
void RoundMatrix(float *mat, const int size);

namespace {
// The reference prints progress lines on std::cout; keep them out of test output.
struct QuietCout {
  std::ostringstream sink;
  std::streambuf *saved;
  explicit QuietCout(bool quiet) : saved(quiet ? std::cout.rdbuf(sink.rdbuf()) : nullptr) {}
  ~QuietCout() {
    if (saved) std::cout.rdbuf(saved);
  }
};
}  // namespace

extern "C" {

// Runs MultiAtlasPatchBasedSegmentation[OpenMP] (NewPatchedBrainPureC.cpp:1238-1337 / 1350-1449)
// on caller-owned buffers in the reference layout [atlas][z][x][y]. `atlas_ct` must already be
// label-normalised (NewPatchedBrainPureC.cpp:1583-1593). Only interior voxels of `out` are
// written; the caller pre-fills the rest. threads <= 0 keeps OpenMP's default.
int pctref_fuse(const float *img, const float *atlas_mri, const float *atlas_ct, float *out, int nx_,
                int ny_, int nz_, int num_, int nh_, double div, int multicore, int threads,
                int quiet) {
  if (!img || !atlas_mri || !atlas_ct || !out || nx_ <= 0 || ny_ <= 0 || nz_ <= 0 || num_ <= 0 ||
      nh_ < 1 || (nh_ % 2) == 0)
    return -1;
  QuietCout q(quiet != 0);
  im = const_cast<float *>(img);
  atlas = const_cast<float *>(atlas_mri);
  label = const_cast<float *>(atlas_ct);
  nx = nx_;
  ny = ny_;
  nz = nz_;
  num = num_;
  nh = nh_;
  if (multicore) {
    if (threads > 0) omp_set_num_threads(threads);
    MultiAtlasPatchBasedSegmentationOpenMP(img, atlas_mri, atlas_ct, out, div);
  } else {
    MultiAtlasPatchBasedSegmentation(img, atlas_mri, atlas_ct, out, div);
  }
  im = nullptr;
  atlas = nullptr;
  label = nullptr;
  return 0;
}

// RegularizationStep (NewPatchedBrainPureC.cpp:1059-1106): in-place NaN median fill.
int pctref_regularize(int half_window, int half_patch, int nx_, int ny_, int nz_, float *arr,
                      int quiet) {
  if (!arr) return -1;
  QuietCout q(quiet != 0);
  RegularizationStep(half_window, half_patch, nx_, ny_, nz_, arr);
  return 0;
}

// RoundMatrix (NewPatchedBrainPureC.cpp:1221-1227).
int pctref_round(float *arr, int size) {
  if (!arr || size < 0) return -1;
  RoundMatrix(arr, size);
  return 0;
}

int pctref_max_threads(void) { return omp_get_max_threads(); }
}
