// Seeded synthetic subjects: input MRI, atlas MRIs and atlas CTs in the reference layout.
//
// The reference's real subject data (.mat files of an MRI plus atlas MRI/CT pairs) is not
// public, and its own test mode fills volumes with time-seeded uniform noise
// (PatchBasedPseudoCT.cu:1429-1450), which is neither reproducible nor image-like. This
// generator makes image-like volumes from a seed:
//   input   I = sum of Gaussian blobs + N(0, mri_noise)
//   atlas a MRI = blobs resampled through a smooth random displacement (max |u| = max_disp
//                 voxels, trilinear) + fresh N(0, mri_noise)
//   atlas a CT  = clip(piecewise-linear MRI->HU map of the resampled blobs, -1000, 2000)
//                 + N(0, ct_noise)
// Every random number is a hash of (seed, stream, index), so the result does not depend on the
// number of threads.
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <thread>
#include <vector>

#include "pct_b200.h"

namespace {

inline uint64_t mix64(uint64_t z) {  // splitmix64 finaliser
  z += 0x9e3779b97f4a7c15ULL;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

struct Rng {
  uint64_t key;
  Rng(uint64_t seed, uint64_t stream) : key(mix64(seed ^ mix64(stream * 0x632be59bd9b4e019ULL))) {}
  // Uniform in (0,1), 24-bit resolution, for counter i.
  double uniform(uint64_t i) const { return ((mix64(key + i) >> 40) + 0.5) * (1.0 / 16777216.0); }
  double uniform(uint64_t i, double lo, double hi) const { return lo + (hi - lo) * uniform(i); }
  // Standard normal for counter i (Box-Muller on two derived uniforms).
  float normal(uint64_t i) const {
    const double u1 = uniform(2 * i), u2 = uniform(2 * i + 1);
    return (float)(sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2));
  }
};

// Streams of the counter-based generator.
enum : uint64_t { kBlobs = 1, kInputNoise = 2, kField = 3, kAtlasNoise = 4, kCtNoise = 5 };

template <class F>
void parallel_planes(int nz, F &&f) {
  unsigned nt = std::max(1u, std::thread::hardware_concurrency());
  nt = std::min<unsigned>(nt, (unsigned)nz);
  std::vector<std::thread> ts;
  for (unsigned t = 0; t < nt; ++t)
    ts.emplace_back([&, t] {
      for (int z = (int)t; z < nz; z += (int)nt) f(z);
    });
  for (auto &th : ts) th.join();
}

// Piecewise-linear MRI intensity -> HU map (fixed knots), clipped to [-1000, 2000].
float mri_to_hu(float m) {
  static const float km[] = {0.f, 60.f, 250.f, 450.f, 700.f, 900.f, 1200.f};
  static const float kh[] = {-1000.f, -1000.f, -100.f, 40.f, 80.f, 1000.f, 2000.f};
  constexpr int n = 7;
  float hu;
  if (m <= km[0]) hu = kh[0];
  else if (m >= km[n - 1]) hu = kh[n - 1];
  else {
    int k = 1;
    while (m > km[k]) ++k;
    const float t = (m - km[k - 1]) / (km[k] - km[k - 1]);
    hu = kh[k - 1] + t * (kh[k] - kh[k - 1]);
  }
  return std::min(2000.f, std::max(-1000.f, hu));
}

struct Mode {
  double fz, fx, fy, phase, amp;
};

}  // namespace

extern "C" {

int pct_synth_default_params(pct_synth_params *p, int nx, int ny, int nz, int num_atlas,
                             int n_blobs, uint64_t seed) {
  if (!p) return PCT_ERR_INVALID_ARG;
  memset(p, 0, sizeof(*p));
  p->nx = nx;
  p->ny = ny;
  p->nz = nz;
  p->num_atlas = num_atlas;
  p->n_blobs = n_blobs;
  p->amp_lo = 100.f;
  p->amp_hi = 1000.f;
  p->std_lo = 2.f;
  p->std_hi = 8.f;
  p->mri_noise = 2.5f;
  p->ct_noise = 20.f;
  p->max_disp = 2.f;
  p->seed = seed;
  return PCT_OK;
}

int pct_synth_generate(const pct_synth_params *p, float *img, float *atlas_mri, float *atlas_ct_hu) {
  if (!p || p->nx <= 0 || p->ny <= 0 || p->nz <= 0 || p->num_atlas < 0 || p->n_blobs < 0 ||
      !(p->std_lo > 0.f) || p->std_hi < p->std_lo || p->amp_hi < p->amp_lo || p->max_disp < 0.f)
    return PCT_ERR_INVALID_ARG;
  const int nx = p->nx, ny = p->ny, nz = p->nz;
  const size_t nxy = (size_t)nx * ny, nvox = nxy * nz;

  // Noise-free blob image C.
  std::vector<float> clean(nvox, 0.f);
  {
    const Rng rb(p->seed, kBlobs);
    struct Blob {
      double cz, cx, cy, amp, inv2s2;
      int r;
    };
    std::vector<Blob> blobs(p->n_blobs);
    for (int b = 0; b < p->n_blobs; ++b) {
      const uint64_t c = (uint64_t)b * 8;
      Blob &bl = blobs[b];
      bl.cz = rb.uniform(c + 0, 0.0, nz - 1.0);
      bl.cx = rb.uniform(c + 1, 0.0, nx - 1.0);
      bl.cy = rb.uniform(c + 2, 0.0, ny - 1.0);
      bl.amp = rb.uniform(c + 3, p->amp_lo, p->amp_hi);
      const double sd = rb.uniform(c + 4, p->std_lo, p->std_hi);
      bl.inv2s2 = 1.0 / (2.0 * sd * sd);
      bl.r = (int)ceil(5.0 * sd);  // exp(-12.5) ~ 4e-6 of the amplitude beyond this radius
    }
    parallel_planes(nz, [&](int z) {
      std::vector<double> ex(nx), ey(ny);
      for (const Blob &bl : blobs) {
        const double dz = z - bl.cz;
        if (fabs(dz) > bl.r) continue;
        const double ez = bl.amp * exp(-dz * dz * bl.inv2s2);
        const int x0 = std::max(0, (int)floor(bl.cx) - bl.r), x1 = std::min(nx - 1, (int)ceil(bl.cx) + bl.r);
        const int y0 = std::max(0, (int)floor(bl.cy) - bl.r), y1 = std::min(ny - 1, (int)ceil(bl.cy) + bl.r);
        for (int x = x0; x <= x1; ++x) ex[x] = exp(-(x - bl.cx) * (x - bl.cx) * bl.inv2s2);
        for (int y = y0; y <= y1; ++y) ey[y] = exp(-(y - bl.cy) * (y - bl.cy) * bl.inv2s2);
        float *plane = clean.data() + (size_t)z * nxy;
        for (int x = x0; x <= x1; ++x) {
          const double ezx = ez * ex[x];
          float *row = plane + (size_t)x * ny;
          for (int y = y0; y <= y1; ++y) row[y] += (float)(ezx * ey[y]);
        }
      }
    });
  }

  if (img) {
    const Rng rn(p->seed, kInputNoise);
    parallel_planes(nz, [&](int z) {
      const size_t b = (size_t)z * nxy;
      for (size_t i = b; i < b + nxy; ++i) img[i] = clean[i] + p->mri_noise * rn.normal(i);
    });
  }

  const double two_pi = 6.283185307179586;
  for (int a = 0; a < p->num_atlas; ++a) {
    // Smooth displacement: per component, 4 Fourier modes of 0..2 cycles per volume extent.
    const Rng rf(p->seed, kField + 16 * (uint64_t)(a + 1));
    Mode modes[3][4];
    for (int c = 0; c < 3; ++c)
      for (int k = 0; k < 4; ++k) {
        const uint64_t base = (uint64_t)(c * 4 + k) * 8;
        Mode &m = modes[c][k];
        do {
          m.fz = floor(rf.uniform(base + 0) * 3.0);
          m.fx = floor(rf.uniform(base + 1) * 3.0);
          m.fy = floor(rf.uniform(base + 2) * 3.0);
          if (m.fz + m.fx + m.fy == 0) m.fy = 1;  // no constant mode
        } while (0);
        m.phase = rf.uniform(base + 3) * two_pi;
        m.amp = rf.uniform(base + 4, 0.5, 1.0);
      }
    auto disp = [&](int z, int x, int y, double *u) {
      for (int c = 0; c < 3; ++c) {
        double v = 0.0;
        for (int k = 0; k < 4; ++k) {
          const Mode &m = modes[c][k];
          v += m.amp * sin(two_pi * (m.fz * z / nz + m.fx * x / nx + m.fy * y / ny) + m.phase);
        }
        u[c] = v;
      }
    };
    // Scale so that the largest displacement magnitude is max_disp.
    std::vector<double> plane_max(nz, 0.0);
    parallel_planes(nz, [&](int z) {
      double m = 0.0, u[3];
      for (int x = 0; x < nx; ++x)
        for (int y = 0; y < ny; ++y) {
          disp(z, x, y, u);
          m = std::max(m, sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]));
        }
      plane_max[z] = m;
    });
    const double umax = *std::max_element(plane_max.begin(), plane_max.end());
    const double scale = umax > 0.0 ? p->max_disp / umax : 0.0;

    const Rng ra(p->seed, kAtlasNoise + 16 * (uint64_t)(a + 1));
    const Rng rc(p->seed, kCtNoise + 16 * (uint64_t)(a + 1));
    float *am = atlas_mri ? atlas_mri + (size_t)a * nvox : nullptr;
    float *ac = atlas_ct_hu ? atlas_ct_hu + (size_t)a * nvox : nullptr;
    if (!am && !ac) continue;
    parallel_planes(nz, [&](int z) {
      double u[3];
      for (int x = 0; x < nx; ++x)
        for (int y = 0; y < ny; ++y) {
          disp(z, x, y, u);
          const double sz = std::min(nz - 1.0, std::max(0.0, z + scale * u[0]));
          const double sx = std::min(nx - 1.0, std::max(0.0, x + scale * u[1]));
          const double sy = std::min(ny - 1.0, std::max(0.0, y + scale * u[2]));
          const int z0 = std::min(nz - 2, (int)floor(sz)), x0 = std::min(nx - 2, (int)floor(sx)),
                    y0 = std::min(ny - 2, (int)floor(sy));
          const int z0c = std::max(0, z0), x0c = std::max(0, x0), y0c = std::max(0, y0);
          const int z1 = std::min(nz - 1, z0c + 1), x1 = std::min(nx - 1, x0c + 1),
                    y1 = std::min(ny - 1, y0c + 1);
          const double fz = sz - z0c, fx = sx - x0c, fy = sy - y0c;
          auto C = [&](int zz, int xx, int yy) { return (double)clean[(size_t)zz * nxy + (size_t)xx * ny + yy]; };
          const double c00 = C(z0c, x0c, y0c) * (1 - fy) + C(z0c, x0c, y1) * fy;
          const double c01 = C(z0c, x1, y0c) * (1 - fy) + C(z0c, x1, y1) * fy;
          const double c10 = C(z1, x0c, y0c) * (1 - fy) + C(z1, x0c, y1) * fy;
          const double c11 = C(z1, x1, y0c) * (1 - fy) + C(z1, x1, y1) * fy;
          const double m = (c00 * (1 - fx) + c01 * fx) * (1 - fz) + (c10 * (1 - fx) + c11 * fx) * fz;
          const size_t i = (size_t)z * nxy + (size_t)x * ny + y;
          if (am) am[i] = (float)m + p->mri_noise * ra.normal(i);
          if (ac) ac[i] = mri_to_hu((float)m) + p->ct_noise * rc.normal(i);
        }
    });
  }
  return PCT_OK;
}

}  // extern "C"
