// Volume files of the drop-in command line.
//
// MatrixIO text format (the reference's MatrixIO<T>::Read/Store, PatchBasedPseudoCT.cu:679-809):
// four header lines num, rows, cols, depth, then num*rows*cols*depth whitespace-separated values
// in the row-based layout [num][depth][rows][cols] (rows = nx, cols = ny, depth = nz). The
// reference writes values with the stream's default 6 significant digits; this writer uses 9 so
// that a float round-trips exactly, and the reader accepts either.
//
// Raw format (this library's addition for large volumes): a sidecar-free little-endian float32
// dump of the same layout; the sizes come from the config file.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <fstream>
#include <sstream>
#include <string>

#include "pct_b200.h"

namespace {

bool read_header(std::istream &in, int dims[4]) {
  std::string line;
  for (int i = 0; i < 4; ++i) {
    if (!std::getline(in, line)) return false;
    char *end = nullptr;
    const long v = strtol(line.c_str(), &end, 10);
    if (end == line.c_str() || v <= 0 || v > (1L << 30)) return false;
    dims[i] = (int)v;
  }
  return true;
}

}  // namespace

extern "C" {

int pct_matrixio_dims(const char *path, int dims[4]) {
  if (!path || !dims) return PCT_ERR_INVALID_ARG;
  std::ifstream in(path);
  if (!in.is_open()) return PCT_ERR_INVALID_ARG;
  return read_header(in, dims) ? PCT_OK : PCT_ERR_INVALID_ARG;
}

int pct_matrixio_read(const char *path, float *out, size_t n) {
  if (!path || (!out && n)) return PCT_ERR_INVALID_ARG;
  std::ifstream in(path);
  if (!in.is_open()) return PCT_ERR_INVALID_ARG;
  int dims[4];
  if (!read_header(in, dims)) return PCT_ERR_INVALID_ARG;
  const size_t expect = (size_t)dims[0] * dims[1] * dims[2] * dims[3];
  if (expect != n) return PCT_ERR_INVALID_ARG;
  // Values may be split over any number of lines (the reference writes them on one line).
  std::string tok;
  size_t i = 0;
  while (i < n && (in >> tok)) {
    char *end = nullptr;
    const float v = strtof(tok.c_str(), &end);
    if (end == tok.c_str()) return PCT_ERR_INVALID_ARG;
    out[i++] = v;
  }
  return i == n ? PCT_OK : PCT_ERR_INVALID_ARG;
}

int pct_matrixio_write(const char *path, const float *data, int num, int rows, int cols,
                       int depth) {
  if (!path || !data || num <= 0 || rows <= 0 || cols <= 0 || depth <= 0)
    return PCT_ERR_INVALID_ARG;
  FILE *f = fopen(path, "w");
  if (!f) return PCT_ERR_INVALID_ARG;
  fprintf(f, "%d\n%d\n%d\n%d\n", num, rows, cols, depth);
  const size_t n = (size_t)num * rows * cols * depth;
  for (size_t i = 0; i < n; ++i) fprintf(f, "%.9g ", (double)data[i]);
  fputc('\n', f);
  const int bad = ferror(f);
  return (fclose(f) == 0 && !bad) ? PCT_OK : PCT_ERR_INVALID_ARG;
}

int pct_raw_read(const char *path, float *out, size_t n) {
  if (!path || (!out && n)) return PCT_ERR_INVALID_ARG;
  FILE *f = fopen(path, "rb");
  if (!f) return PCT_ERR_INVALID_ARG;
  const size_t got = fread(out, sizeof(float), n, f);
  const int extra = fgetc(f);
  fclose(f);
  return (got == n && extra == EOF) ? PCT_OK : PCT_ERR_INVALID_ARG;
}

int pct_raw_write(const char *path, const float *data, size_t n) {
  if (!path || (!data && n)) return PCT_ERR_INVALID_ARG;
  FILE *f = fopen(path, "wb");
  if (!f) return PCT_ERR_INVALID_ARG;
  const size_t put = fwrite(data, sizeof(float), n, f);
  return (fclose(f) == 0 && put == n) ? PCT_OK : PCT_ERR_INVALID_ARG;
}

}  // extern "C"
