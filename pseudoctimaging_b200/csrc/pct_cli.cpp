// PatchBasedPseudoCT_b200: drop-in command line for the reference's GPU executable.
//
//   PatchBasedPseudoCT_b200 <data> <output name> <EXEC_CHOICE> <NH> [sigma beta] [device]
//
// Same positional arguments as the reference (PatchBasedPseudoCT.cu:1970-1983): sigma and beta
// are read when at least 7 arguments are given, the device when 8 are (defaults sigma=1, beta=1,
// device 0, as in the reference). EXEC_CHOICE 0/1/2/3 run the path (the reference's GM, GM2, SM
// and this library's plain FP32 kernel, which compute the same function); 4 times it like the
// reference's GpuTestTime (10 samples of 10 calls); 5/6 run the tensor-core FP16/BF16 form and 7
// the learned proposal (NH = 7, 9 or 11; the network from $PCT_LEARNED_MODEL, else the checkpoint
// shipped beside the program, with the fallback threshold $PCT_LEARNED_CONF, default 0).
//
// <data> is the reference's MATLAB data file (a name ending in .mat: variables img, atlas and
// atlas_label, ReadMatFile, PatchBasedPseudoCT.cu:1047-1169; the result goes to
// <output name>.mat as one single variable named after the result, WriteOutputMatFile,
// :1310-1370), or its non-MATLAB configuration file (PatchBasedPseudoCT.cu:1376-1488):
//   line 1: 0 -> lines 2-4: atlas MRI, atlas CT, input MRI as MatrixIO text files
//           1 -> lines 2-5: num, nx, ny, nz; volumes of uniform [0,10) values (the reference's
//                test mode; seeded here, so runs are reproducible)
//   and two forms of this library's:
//           2 -> lines 2-5: num, nx, ny, nz; lines 6-8: atlas MRI, atlas CT, input MRI as raw
//                float32 files in the [atlas][z][x][y] layout
//           3 -> lines 2-7: num, nx, ny, nz, n_blobs, seed; a synthetic subject from the seeded
//                generator
// After the path the label volume is regularised, rounded and mapped back to HU as the reference's
// main does (:2166-2180) and written to <output name>.txt (MatrixIO) or, for forms 2 and 3,
// <output name>.f32 (raw).
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <chrono>
#include <fstream>
#include <string>
#include <vector>

#include "pct_b200.h"

namespace {

struct Subject {
  int nx = 0, ny = 0, nz = 0, num = 0;
  std::vector<float> img, atlas, ct;
  bool raw_output = false;
  bool mat_output = false;
};

bool ends_with(const std::string &s, const char *suffix) {
  const size_t n = strlen(suffix);
  return s.size() >= n && s.compare(s.size() - n, n, suffix) == 0;
}

std::vector<std::string> read_lines(const char *path) {
  std::vector<std::string> lines;
  std::ifstream in(path);
  std::string l;
  while (std::getline(in, l)) {
    while (!l.empty() && (l.back() == '\r' || l.back() == ' ')) l.pop_back();
    lines.push_back(l);
  }
  return lines;
}

int to_int(const std::string &s, int *v) {
  char *end = nullptr;
  const long x = strtol(s.c_str(), &end, 10);
  if (end == s.c_str() || x <= 0 || x > (1L << 30)) return -1;
  *v = (int)x;
  return 0;
}

bool load_matrixio(const std::string &path, std::vector<float> &out, int dims[4]) {
  if (pct_matrixio_dims(path.c_str(), dims) != PCT_OK) return false;
  out.resize((size_t)dims[0] * dims[1] * dims[2] * dims[3]);
  return pct_matrixio_read(path.c_str(), out.data(), out.size()) == PCT_OK;
}

bool load_subject(const char *config, Subject *s, std::string *err) {
  if (ends_with(config, ".mat") || ends_with(config, ".MAT")) {
    // the reference's MATLAB data file: img, atlas, atlas_label (ReadMatFile)
    int d[4];
    if (pct_mat_dims(config, d) != PCT_OK) {
      *err = std::string("cannot read the MAT data file ") + config +
             " (img, atlas and atlas_label of equal [nx ny nz] single volumes)";
      return false;
    }
    s->num = d[0];
    s->nx = d[1];
    s->ny = d[2];
    s->nz = d[3];
    const size_t n = (size_t)s->nx * s->ny * s->nz;
    s->img.resize(n);
    s->atlas.resize(n * s->num);
    s->ct.resize(n * s->num);
    if (pct_mat_read(config, s->img.data(), s->atlas.data(), s->ct.data(), n, n * s->num) !=
        PCT_OK) {
      *err = std::string("cannot read the MAT data file ") + config;
      return false;
    }
    s->mat_output = true;
    return true;
  }
  const std::vector<std::string> L = read_lines(config);
  if (L.empty()) {
    *err = std::string("cannot read configuration file ") + config;
    return false;
  }
  int mode = -1;
  if (to_int(L[0], &mode) != 0 && L[0] != "0") {
    *err = "first line must be 0, 1, 2 or 3";
    return false;
  }
  if (L[0] == "0") mode = 0;
  if (mode == 0) {
    if (L.size() < 4) {
      *err = "mode 0 needs three MatrixIO paths (atlas MRI, atlas CT, input MRI)";
      return false;
    }
    int da[4], dl[4], di[4];
    if (!load_matrixio(L[1], s->atlas, da) || !load_matrixio(L[2], s->ct, dl) ||
        !load_matrixio(L[3], s->img, di)) {
      *err = "cannot read a MatrixIO volume";
      return false;
    }
    // dims = num, rows (nx), cols (ny), depth (nz); the check of PatchBasedPseudoCT.cu:1464-1482
    if (memcmp(da, dl, sizeof(da)) != 0 || da[1] != di[1] || da[2] != di[2] || da[3] != di[3] ||
        di[0] != 1) {
      *err = "Dimensions do not match";
      return false;
    }
    s->num = da[0];
    s->nx = da[1];
    s->ny = da[2];
    s->nz = da[3];
    return true;
  }
  if (mode < 1 || mode > 3 || L.size() < 5 || to_int(L[1], &s->num) || to_int(L[2], &s->nx) ||
      to_int(L[3], &s->ny) || to_int(L[4], &s->nz)) {
    *err = "modes 1-3 need num, nx, ny, nz on lines 2-5";
    return false;
  }
  const size_t n = (size_t)s->nx * s->ny * s->nz;
  s->img.resize(n);
  s->atlas.resize(n * s->num);
  s->ct.resize(n * s->num);
  if (mode == 1) {
    // Uniform [0,10) like the reference's random mode, from a fixed-seed generator.
    uint64_t state = 0x2545F4914F6CDD1DULL;
    auto next = [&state]() {
      state ^= state << 13;
      state ^= state >> 7;
      state ^= state << 17;
      return (float)((state >> 40) * (1.0 / 16777216.0) * 10.0);
    };
    for (auto &v : s->atlas) v = next();
    for (auto &v : s->ct) v = next();
    for (auto &v : s->img) v = next();
    return true;
  }
  s->raw_output = true;
  if (mode == 2) {
    if (L.size() < 8 || pct_raw_read(L[5].c_str(), s->atlas.data(), s->atlas.size()) ||
        pct_raw_read(L[6].c_str(), s->ct.data(), s->ct.size()) ||
        pct_raw_read(L[7].c_str(), s->img.data(), s->img.size())) {
      *err = "mode 2 needs three raw float32 volumes of the stated sizes on lines 6-8";
      return false;
    }
    return true;
  }
  int blobs = 0, seed = 0;
  if (L.size() < 7 || to_int(L[5], &blobs) || (to_int(L[6], &seed) && L[6] != "0")) {
    *err = "mode 3 needs n_blobs and seed on lines 6-7";
    return false;
  }
  if (L[6] == "0") seed = 0;
  pct_synth_params p;
  pct_synth_default_params(&p, s->nx, s->ny, s->nz, s->num, blobs, (uint64_t)seed);
  if (pct_synth_generate(&p, s->img.data(), s->atlas.data(), s->ct.data()) != PCT_OK) {
    *err = "synthetic generator rejected the sizes";
    return false;
  }
  return true;
}

void usage() {
  printf(
      "Usage: PatchBasedPseudoCT_b200 <data> <output name> <EXEC_CHOICE> <NH> [sigma beta] "
      "[device]\n"
      "  EXEC_CHOICE {GM=0, GM2=1, SM=2, B200 FP32=3: the path; GpuTestTime=4: timing;\n"
      "               5/6: tensor-core FP16/BF16 form; 7: learned proposal}\n"
      "  NH {3,5,7,9,11} (11 for 5 and 6; 7, 9 or 11 for 7); sigma, beta default 1; device 0\n"
      "  EXEC_CHOICE 7 reads the network from $PCT_LEARNED_MODEL (default: the checkpoint\n"
      "  shipped beside this program, ../checkpoints/learned_nh11.pctl) and the full-search\n"
      "  confidence threshold from $PCT_LEARNED_CONF (default 0)\n");
}

}  // namespace

int main(int argc, char **argv) {
  if (argc < 5) {
    usage();
    return 0;
  }
  double sigma = 1.0, beta = 1.0;
  int device = 0;
  if (argc >= 8) device = atoi(argv[7]);
  if (argc >= 7) {
    sigma = atof(argv[5]);
    beta = atof(argv[6]);
  }
  const std::string out_name = argv[2];
  const int choice = atoi(argv[3]);
  const int nh = atoi(argv[4]);

  Subject s;
  std::string err;
  if (!load_subject(argv[1], &s, &err)) {
    fprintf(stderr, "%s\n", err.c_str());
    return EXIT_FAILURE;
  }
  printf("nx=%d ny=%d nz=%d num=%d NH=%d sigma=%g beta=%g device=%d choice=%d\n", s.nx, s.ny, s.nz,
         s.num, nh, sigma, beta, device, choice);

  pct_handle *h = nullptr;
  int st = pct_create(device, &h);
  if (st != PCT_OK) {
    fprintf(stderr, "pct_create: %s\n", pct_strerror(st));
    return EXIT_FAILURE;
  }
  const size_t n = (size_t)s.nx * s.ny * s.nz;
  std::vector<float> out(n, 0.0f);
  const double div = 2 * 27 * beta * sigma * sigma;

  if (choice == 4) {
    // Timing of the path alone, 10 samples of 10 calls (the reference's GpuTestTime loop).
    std::vector<float> label(s.ct);
    for (auto &v : label) v = 255.0f * ((v + 1024.0f) / 4095.0f);
    for (int i = 0; i < 10 && st == PCT_OK; ++i) {
      const auto t0 = std::chrono::steady_clock::now();
      for (int j = 0; j < 10 && st == PCT_OK; ++j)
        st = pct_synthesize(h, s.img.data(), s.atlas.data(), label.data(), out.data(), s.nx, s.ny,
                            s.nz, s.num, nh, div, PCT_EXEC_B200_FP32);
      const double ms =
          std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count() / 10;
      printf("Iter %d Atlas %d Nh %d Elapsed Time %f ms %f voxels/s\n", i, s.num, nh, ms,
             n / (ms / 1e3));
    }
  } else if ((choice >= 0 && choice <= 3) || choice == 5 || choice == 6 || choice == 7) {
    pct_model *model = nullptr;
    if (choice == PCT_EXEC_LEARNED) {
      std::string path;
      if (const char *e = getenv("PCT_LEARNED_MODEL")) {
        path = e;
      } else {
        std::string exe = argv[0];
        const size_t slash = exe.rfind('/');
        path = (slash == std::string::npos ? std::string(".") : exe.substr(0, slash)) +
               "/../checkpoints/learned_nh11.pctl";
      }
      const char *c = getenv("PCT_LEARNED_CONF");
      const float conf = c ? (float)atof(c) : 0.0f;
      if ((st = pct_model_create(device, 0, &model)) != PCT_OK ||
          (st = pct_model_load_file(model, path.c_str())) != PCT_OK ||
          (st = pct_attach_model(h, model, conf)) != PCT_OK) {
        fprintf(stderr, "learned model %s: %s %s\n", path.c_str(), pct_strerror(st),
                model ? pct_model_last_error(model) : "");
        if (model) pct_model_destroy(model);
        pct_destroy(h);
        return EXIT_FAILURE;
      }
    }
    const auto t0 = std::chrono::steady_clock::now();
    st = pct_run_pipeline(h, s.img.data(), s.atlas.data(), s.ct.data(), out.data(), s.nx, s.ny,
                          s.nz, s.num, nh, sigma, beta, choice, /*regularize=*/1);
    const double ms =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    if (st == PCT_OK) {
      const std::string file =
          out_name + (s.mat_output ? ".mat" : s.raw_output ? ".f32" : ".txt");
      // a MAT result holds one variable named after the result, as the reference's
      // WriteOutputMatFile; a directory part of the name is not part of the variable's name
      const size_t slash = out_name.find_last_of("/\\");
      const std::string var = slash == std::string::npos ? out_name : out_name.substr(slash + 1);
      const int wst =
          s.mat_output ? pct_mat_write(file.c_str(), var.c_str(), out.data(), s.nx, s.ny, s.nz)
          : s.raw_output ? pct_raw_write(file.c_str(), out.data(), n)
                         : pct_matrixio_write(file.c_str(), out.data(), 1, s.nx, s.ny, s.nz);
      if (wst != PCT_OK) {
        fprintf(stderr, "cannot write %s\n", file.c_str());
        st = wst;
      } else {
        printf("File %s written\n", file.c_str());
      }
      printf("Elapsed Time %f ms (transfers, path, regularisation, HU map) %f voxels/s\n", ms,
             n / (ms / 1e3));
    }
    if (model) {
      pct_attach_model(h, nullptr, 0.f);
      pct_model_destroy(model);
    }
  } else {
    st = PCT_ERR_INVALID_ARG;
  }
  if (st != PCT_OK)
    fprintf(stderr, "error: %s: %s\n", pct_strerror(st), pct_last_error_message(h));
  pct_destroy(h);
  return st == PCT_OK ? EXIT_SUCCESS : EXIT_FAILURE;
}
