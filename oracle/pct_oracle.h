/*
 * CPU restatement of the reference's patch-based multi-atlas pseudo-CT path.
 *
 * TEST INFRASTRUCTURE ONLY: the parity checker and the timed CPU baseline. Nothing in the
 * product library links or calls it. Each function cites the reference code it restates
 * (paths relative to the EduardoAlcainBallesteros/PseudoCTImaging tree).
 *
 * Layout everywhere: [atlas][z][x][y], y fastest, index a*N + z*nx*ny + x*ny + y.
 */
#ifndef PCT_ORACLE_H
#define PCT_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* div = 2*27*beta*sigma^2 (NewPatchedBrainPureC.cpp:1630). */
double pct_oracle_div(double sigma, double beta);

/* In-place CT->label scale L' = 255*((L+1024)/4095) in float (NewPatchedBrainPureC.cpp:1583-1593). */
void pct_oracle_normalize_labels(float *label, size_t n);

/* PatchSimilarity (NewPatchedBrainPureC.cpp:1184-1212) for the 3x3x3 patches centred at
 * (z,x,y) in img and (w,u,v) in atlas volume `at`: exp(-SSD/div), in double. */
double pct_oracle_patch_weight(const float *img, const float *atlas, int nx, int ny, int nz, int at,
                               int z, int x, int y, int w, int u, int v, double div);

/* MultiAtlasPatchBasedSegmentation[OpenMP] (NewPatchedBrainPureC.cpp:1238-1337, 1350-1449).
 * Writes only interior voxels of `out` (the rest is left as the caller set it). If `prod` /
 * `sumw` are non-NULL they receive the double accumulators per voxel (interior only).
 * threads <= 0 uses the OpenMP default. Returns the number of NaN voxels, or -1 on bad args. */
int64_t pct_oracle_fuse(const float *img, const float *atlas, const float *label, float *out,
                        int nx, int ny, int nz, int num, int nh, double div, double *prod,
                        double *sumw, int threads);

/* Same arithmetic for an explicit list of voxel indices (z*nx*ny + x*ny + y). Voxels outside
 * the interior get out = 0 and prod = sumw = 0. */
int pct_oracle_fuse_voxels(const float *img, const float *atlas, const float *label, int nx, int ny,
                           int nz, int num, int nh, double div, const int64_t *voxels, int64_t n,
                           float *out, double *prod, double *sumw, int threads);

/* RegularizationStep + Median (NewPatchedBrainPureC.cpp:1024-1047, 1059-1106): in-place
 * Gauss-Seidel NaN fill with the median of the non-NaN 3x3x3 neighbourhood, repeated until no
 * NaN remains in the interior. Returns the number of fills performed. */
int64_t pct_oracle_regularize(int half_window, int half_patch, int nx, int ny, int nz, float *arr);

/* RoundMatrix (NewPatchedBrainPureC.cpp:1221-1227). */
void pct_oracle_round(float *arr, size_t n);

/* Label scale back to HU: round(4095*(v/255)) - 1024 in float (NewPatchedBrainPureC.cpp:1732-1738). */
void pct_oracle_to_hu(float *arr, size_t n);

#ifdef __cplusplus
}
#endif

#endif /* PCT_ORACLE_H */
