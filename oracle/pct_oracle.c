/*
 * Oracle: CPU restatement of the reference's patch-based multi-atlas pseudo-CT path.
 *
 * TEST INFRASTRUCTURE ONLY (parity checker and timed CPU baseline); never linked into or called
 * by the product library. The arithmetic follows the reference CPU code step for step in double
 * precision, in the same loop and summation order, so that with -ffp-contract=off it reproduces
 * the compiled reference bit for bit (checked by tests/test_oracle.py against
 * oracle/_ref/libpctref.so and against tests/golden/).
 */
#include "pct_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

double pct_oracle_div(double sigma, double beta) {
  /* NewPatchedBrainPureC.cpp:1630: div = (2 * 27 * beta*pow(sigma, 2)); */
  return 2 * 27 * beta * pow(sigma, 2);
}

void pct_oracle_normalize_labels(float *label, size_t n) {
  /* NewPatchedBrainPureC.cpp:1588-1589, float arithmetic. */
  for (size_t i = 0; i < n; ++i) label[i] = 255.0f * ((label[i] + 1024.0f) / 4095.0f);
}

double pct_oracle_patch_weight(const float *img, const float *atlas, int nx, int ny, int nz, int at,
                               int z, int x, int y, int w, int u, int v, double div) {
  /* NewPatchedBrainPureC.cpp:1184-1212. Patch order: z (k), then x rows (i), then y cols (j);
   * each tap is a double difference of two floats, squared exactly as pow(d, 2). */
  const size_t pitch = (size_t)nx * ny;
  const size_t offset = pitch * (size_t)nz * (size_t)at;
  double sum = 0.0;
  for (int k = -1; k <= 1; ++k) {
    for (int i = -1; i <= 1; ++i) {
      for (int j = -1; j <= 1; ++j) {
        const double p = img[(size_t)(z + k) * pitch + (size_t)(x + i) * ny + (size_t)(y + j)];
        const double pa =
            atlas[offset + (size_t)(w + k) * pitch + (size_t)(u + i) * ny + (size_t)(v + j)];
        const double d = p - pa;
        sum += d * d;
      }
    }
  }
  return exp(-(sum / div));
}

/* One interior voxel: the body of the z/x/y loop, NewPatchedBrainPureC.cpp:1283-1331. */
static float fuse_one(const float *img, const float *atlas, const float *label, int nx, int ny,
                      int nz, int num, int hw, int z, int x, int y, double div, double *prod_out,
                      double *sumw_out) {
  const size_t pitch = (size_t)nx * ny;
  const size_t nvox = pitch * (size_t)nz;
  double product = 0.0, sum_weight = 0.0;
  for (int at = 0; at < num; ++at) {
    const size_t offset = nvox * (size_t)at;
    for (int w = z - hw; w <= z + hw; ++w) {
      for (int u = x - hw; u <= x + hw; ++u) {
        for (int v = y - hw; v <= y + hw; ++v) {
          const double lab = label[offset + (size_t)w * pitch + (size_t)u * ny + (size_t)v];
          const double weight =
              pct_oracle_patch_weight(img, atlas, nx, ny, nz, at, z, x, y, w, u, v, div);
          product += weight * lab;
          sum_weight += weight;
        }
      }
    }
  }
  if (prod_out) *prod_out = product;
  if (sumw_out) *sumw_out = sum_weight;
  /* NewPatchedBrainPureC.cpp:1325-1331 */
  if (fabs(product) > DBL_EPSILON && fabs(sum_weight) > DBL_EPSILON)
    return (float)(product / sum_weight);
  return NAN;
}

static int valid_args(int nx, int ny, int nz, int num, int nh) {
  return nx > 0 && ny > 0 && nz > 0 && num > 0 && nh >= 1 && (nh % 2) == 1;
}

int64_t pct_oracle_fuse(const float *img, const float *atlas, const float *label, float *out,
                        int nx, int ny, int nz, int num, int nh, double div, double *prod,
                        double *sumw, int threads) {
  if (!img || !atlas || !label || !out || !valid_args(nx, ny, nz, num, nh)) return -1;
  const int hp = 1, hw = (nh - 1) / 2;
  const int lo = hw + hp;
  const size_t pitch = (size_t)nx * ny;
  int64_t nan_count = 0;
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#else
  (void)threads;
#endif
  /* NewPatchedBrainPureC.cpp:1374: parallel over z planes. */
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : nan_count)
  for (int z = lo; z < nz - lo; ++z) {
    for (int x = lo; x < nx - lo; ++x) {
      for (int y = lo; y < ny - lo; ++y) {
        const size_t i = (size_t)z * pitch + (size_t)x * ny + (size_t)y;
        double p, s;
        const float o = fuse_one(img, atlas, label, nx, ny, nz, num, hw, z, x, y, div, &p, &s);
        out[i] = o;
        if (prod) prod[i] = p;
        if (sumw) sumw[i] = s;
        if (isnan(o)) ++nan_count;
      }
    }
  }
  return nan_count;
}

int pct_oracle_fuse_voxels(const float *img, const float *atlas, const float *label, int nx, int ny,
                           int nz, int num, int nh, double div, const int64_t *voxels, int64_t n,
                           float *out, double *prod, double *sumw, int threads) {
  if (!img || !atlas || !label || !voxels || !out || n < 0 || !valid_args(nx, ny, nz, num, nh))
    return -1;
  const int hw = (nh - 1) / 2, lo = hw + 1;
  const int64_t pitch = (int64_t)nx * ny;
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#else
  (void)threads;
#endif
#pragma omp parallel for schedule(dynamic, 4)
  for (int64_t k = 0; k < n; ++k) {
    const int64_t i = voxels[k];
    const int z = (int)(i / pitch);
    const int x = (int)((i % pitch) / ny);
    const int y = (int)(i % ny);
    double p = 0.0, s = 0.0;
    float o = 0.0f;
    if (i >= 0 && z >= lo && z < nz - lo && x >= lo && x < nx - lo && y >= lo && y < ny - lo)
      o = fuse_one(img, atlas, label, nx, ny, nz, num, hw, z, x, y, div, &p, &s);
    out[k] = o;
    if (prod) prod[k] = p;
    if (sumw) sumw[k] = s;
  }
  return 0;
}

/* Median (NewPatchedBrainPureC.cpp:1024-1047): median of the non-NaN entries, averaged in double
 * for an even count. A stable insertion sort stands in for std::stable_sort (same order). */
static double median_non_nan(const float *v, int length, int *count) {
  float buf[27];
  int cnt = 0;
  for (int j = 0; j < length; ++j)
    if (!isnan(v[j])) buf[cnt++] = v[j];
  for (int i = 1; i < cnt; ++i) {
    const float key = buf[i];
    int j = i - 1;
    while (j >= 0 && buf[j] > key) {
      buf[j + 1] = buf[j];
      --j;
    }
    buf[j + 1] = key;
  }
  *count = cnt;
  if (cnt <= 0) return NAN; /* the reference reads out of bounds here (UB); see below */
  if (cnt % 2 == 0) {
    const double a = buf[cnt / 2 - 1];
    const double b = buf[cnt / 2];
    return (a + b) / 2;
  }
  return (double)buf[cnt / 2];
}

int64_t pct_oracle_regularize(int half_window, int half_patch, int nx, int ny, int nz, float *arr) {
  /* NewPatchedBrainPureC.cpp:1059-1106. Sweeps z, x, y over the interior, replacing each NaN in
   * place (so later voxels of the same sweep see earlier fills), until a sweep leaves no NaN.
   * With a non-NaN border every NaN has an already-visited non-NaN neighbour, so the all-NaN
   * branch (undefined behaviour in the reference) is never reached; here it leaves the NaN for
   * the next sweep, and a sweep that fills nothing ends the loop instead of spinning. */
  if (!arr) return -1;
  const int lo = half_window + half_patch;
  const size_t level1 = (size_t)nx * ny;
  int64_t fills = 0;
  int nan_flag = 1;
  while (nan_flag) {
    nan_flag = 0;
    int64_t sweep_fills = 0;
    for (int z = lo; z < nz - lo; ++z) {
      for (int x = lo; x < nx - lo; ++x) {
        for (int y = lo; y < ny - lo; ++y) {
          float *c = &arr[(size_t)z * level1 + (size_t)x * ny + (size_t)y];
          if (!isnan(*c)) continue;
          float patch[27];
          int cnt = 0;
          for (int r = z - half_patch; r <= z + half_patch; ++r)
            for (int s = x - half_patch; s <= x + half_patch; ++s)
              for (int t = y - half_patch; t <= y + half_patch; ++t)
                patch[cnt++] = arr[(size_t)r * level1 + (size_t)s * ny + (size_t)t];
          int nn;
          const double m = median_non_nan(patch, cnt, &nn);
          if (nn > 0) {
            *c = (float)m;
            ++fills;
            ++sweep_fills;
          }
          if (isnan(*c)) nan_flag = 1;
        }
      }
    }
    if (sweep_fills == 0) break;
  }
  return fills;
}

void pct_oracle_round(float *arr, size_t n) {
  /* NewPatchedBrainPureC.cpp:1221-1227: round half away from zero. */
  for (size_t i = 0; i < n; ++i) arr[i] = roundf(arr[i]);
}

void pct_oracle_to_hu(float *arr, size_t n) {
  /* NewPatchedBrainPureC.cpp:1732-1738 with maxLabels = 4095.0f, minLabels = 1024.0f. */
  for (size_t i = 0; i < n; ++i) arr[i] = roundf(4095.0f * (arr[i] / 255.0f)) - 1024.0f;
}
