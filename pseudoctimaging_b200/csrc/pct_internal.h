// Internal declarations shared by the CUDA translation units of libpct_b200.so.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

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

// Plain FP32 fusion (the path's hot loop). Writes interior voxels of out only.
cudaError_t launch_fuse_plain(const Geometry &g, const float *img, const float *atlas,
                              const float *label, float *out, double div, cudaStream_t stream);

// Number of kernel launches launch_fuse_plain issues for this geometry.
int fuse_plain_launches(const Geometry &g);

// NaN median fill (synchronous on `stream`: it reads back a counter after each round).
// scratch must hold regularize_scratch_bytes(nx*ny*nz) bytes.
size_t regularize_scratch_bytes(long long nvox);
cudaError_t launch_regularize(float *vol, int nx, int ny, int nz, int nh, void *scratch,
                              cudaStream_t stream, long long *fills_out, int *rounds_out);

cudaError_t launch_normalize_labels(float *label, size_t n, cudaStream_t stream);
cudaError_t launch_finalize_hu(float *vol, size_t n, cudaStream_t stream);

}  // namespace pct
