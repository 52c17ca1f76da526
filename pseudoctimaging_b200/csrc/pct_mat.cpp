// MATLAB level-5 MAT-files: the reference's data and result files, without MATLAB's libmat.
//
// Data file (ReadMatFile and FindDimension, PatchBasedPseudoCT.cu:1047-1300): a variable `img`
// ([nx ny nz] single), and `atlas` and `atlas_label`, 1x1 structs whose fields are the atlases'
// [nx ny nz] single volumes; atlas i is the struct's i-th field, so num = the number of fields.
// As in the reference, a numeric variable that is not a struct is taken as the input MRI
// (Choice / the else branch of ReadMatFile), structs named neither atlas nor atlas_label are
// ignored, and fields that are not real single arrays are skipped (AnalyzeStructArray). Every
// volume must have the same three dimensions.
// Result file (WriteOutputMatFile, :1310-1370): one [nx ny nz] single variable named after the
// result, uncompressed.
// MATLAB stores arrays column-major; the reference converts them to its layout [z][x][y] with
// x = dimension 1 and y = dimension 2 (ConvertToRowBased, :851-889, and ConvertMatrixMatlab for
// the way back), and so does this file.
//
// Format (MathWorks, "MAT-File Format", level 5): a 128-byte header (text, subsystem offset,
// version 0x0100, endian indicator "IM" for little-endian files), then data elements, each an
// 8-byte tag (type, byte count; or the 4-byte "small" form with the count in the upper half of
// the type word) and data padded to 8 bytes. miCOMPRESSED elements hold one zlib-deflated element.
// A miMATRIX holds array flags (class in the low byte), dimensions, a name and, for numeric
// classes, the real part in any numeric storage type (MATLAB may store single data as smaller
// integer types); a struct holds the field-name length, the names, then one miMATRIX per element
// and field. Little-endian files only.
#include <stdint.h>
#include <stdio.h>
#include <string.h>
#include <zlib.h>

#include <string>
#include <vector>

#include "pct_b200.h"

namespace {

enum : uint32_t {
  miINT8 = 1, miUINT8 = 2, miINT16 = 3, miUINT16 = 4, miINT32 = 5, miUINT32 = 6, miSINGLE = 7,
  miDOUBLE = 9, miINT64 = 12, miUINT64 = 13, miMATRIX = 14, miCOMPRESSED = 15
};
enum : uint32_t { mxSTRUCT = 2, mxDOUBLE = 6, mxSINGLE = 7 };

struct Element {
  uint32_t type = 0;
  const unsigned char *data = nullptr;
  size_t bytes = 0;
};

// Reads the element at *pos of [buf, buf + n); advances *pos past it (and its padding).
bool next_element(const unsigned char *buf, size_t n, size_t *pos, Element *e, bool pad = true) {
  if (*pos + 8 > n) return false;
  uint32_t w0, w1;
  memcpy(&w0, buf + *pos, 4);
  memcpy(&w1, buf + *pos + 4, 4);
  if (w0 >> 16) {  // small data element: up to 4 bytes in the tag's second word
    e->type = w0 & 0xFFFF;
    e->bytes = w0 >> 16;
    if (e->bytes > 4) return false;
    e->data = buf + *pos + 4;
    *pos += 8;
    return true;
  }
  e->type = w0;
  e->bytes = w1;
  if (*pos + 8 + e->bytes > n) return false;
  e->data = buf + *pos + 8;
  *pos += 8 + e->bytes;
  if (pad) *pos = (*pos + 7) & ~(size_t)7;
  return true;
}

size_t type_size(uint32_t t) {
  switch (t) {
    case miINT8: case miUINT8: return 1;
    case miINT16: case miUINT16: return 2;
    case miINT32: case miUINT32: case miSINGLE: return 4;
    case miDOUBLE: case miINT64: case miUINT64: return 8;
    default: return 0;
  }
}

template <typename T>
T load(const unsigned char *p) {
  T v;
  memcpy(&v, p, sizeof(T));
  return v;
}

double value_at(const Element &e, size_t i) {
  const unsigned char *p = e.data + i * type_size(e.type);
  switch (e.type) {
    case miINT8: return (double)load<int8_t>(p);
    case miUINT8: return (double)load<uint8_t>(p);
    case miINT16: return (double)load<int16_t>(p);
    case miUINT16: return (double)load<uint16_t>(p);
    case miINT32: return (double)load<int32_t>(p);
    case miUINT32: return (double)load<uint32_t>(p);
    case miSINGLE: return (double)load<float>(p);
    case miDOUBLE: return load<double>(p);
    case miINT64: return (double)load<int64_t>(p);
    case miUINT64: return (double)load<uint64_t>(p);
    default: return 0.0;
  }
}

// One parsed array: class, dimensions, name; numeric data (the real part) or struct fields.
struct Array {
  uint32_t cls = 0;
  bool complex = false;
  std::vector<int64_t> dims;
  std::string name;
  Element real;
  std::vector<std::string> fields;
  std::vector<Array> members;  // element-major: members[e * fields + f]
};

bool parse_matrix(const unsigned char *buf, size_t n, Array *a, int depth);

// The body of a miMATRIX element.
bool parse_matrix(const unsigned char *buf, size_t n, Array *a, int depth) {
  if (depth > 8) return false;
  if (n == 0) return true;  // an empty array (e.g. an unset struct field)
  size_t pos = 0;
  Element e;
  if (!next_element(buf, n, &pos, &e) || e.type != miUINT32 || e.bytes < 8) return false;
  const uint32_t flags = load<uint32_t>(e.data);
  a->cls = flags & 0xFF;
  a->complex = (flags & 0x800) != 0;
  if (!next_element(buf, n, &pos, &e) || e.type != miINT32 || e.bytes % 4 || e.bytes == 0)
    return false;
  int64_t count = 1;
  for (size_t i = 0; i < e.bytes / 4; ++i) {
    const int32_t d = load<int32_t>(e.data + 4 * i);
    if (d < 0) return false;
    a->dims.push_back(d);
    count *= d;
    if (count > ((int64_t)1 << 40)) return false;  // larger than any file this reads
  }
  if (!next_element(buf, n, &pos, &e) || (e.type != miINT8 && e.type != miUINT8)) return false;
  a->name.assign(reinterpret_cast<const char *>(e.data), e.bytes);
  if (a->cls == mxSTRUCT) {
    if (!next_element(buf, n, &pos, &e) || e.type != miINT32 || e.bytes != 4) return false;
    const int32_t len = load<int32_t>(e.data);
    if (!next_element(buf, n, &pos, &e) || (e.type != miINT8 && e.type != miUINT8) || len <= 0 ||
        e.bytes % (size_t)len)
      return false;
    for (size_t f = 0; f < e.bytes / (size_t)len; ++f)
      a->fields.emplace_back(reinterpret_cast<const char *>(e.data) + f * len,
                             strnlen(reinterpret_cast<const char *>(e.data) + f * len, len));
    for (int64_t m = 0; m < count * (int64_t)a->fields.size(); ++m) {
      if (!next_element(buf, n, &pos, &e) || e.type != miMATRIX) return false;
      Array member;
      if (!parse_matrix(e.data, e.bytes, &member, depth + 1)) return false;
      a->members.push_back(std::move(member));
    }
    return true;
  }
  if (a->cls >= mxDOUBLE && a->cls <= 15) {  // numeric classes
    if (!next_element(buf, n, &pos, &e) || type_size(e.type) == 0 ||
        e.bytes != (size_t)count * type_size(e.type))
      return false;
    a->real = e;
  }
  return true;  // other classes (cell, char, sparse, ...) are carried but never used
}

// Every top-level variable of the file; `store` keeps the inflated bodies alive.
bool parse_file(const std::vector<unsigned char> &file, std::vector<Array> *vars,
                std::vector<std::vector<unsigned char>> *store, std::string *why) {
  if (file.size() < 128) {
    *why = "shorter than the 128-byte MAT header";
    return false;
  }
  if (file[126] != 'I' || file[127] != 'M') {
    *why = "not a little-endian level-5 MAT-file";
    return false;
  }
  if (file[125] != 0x01 || file[124] != 0x00) {  // 0x0200: a version 7.3 (HDF5) file
    *why = "not a level-5 MAT-file (version 7.3 files are HDF5; save with -v7 or -v6)";
    return false;
  }
  size_t pos = 128;
  while (pos + 8 <= file.size()) {
    Element e;
    const uint32_t t = load<uint32_t>(file.data() + pos);
    if (!next_element(file.data(), file.size(), &pos, &e, t != miCOMPRESSED)) {
      *why = "truncated data element";
      return false;
    }
    if (e.type == miCOMPRESSED) {
      // the inflated size is unknown: grow the output until the stream ends
      std::vector<unsigned char> out(e.bytes * 4 + 1024);
      z_stream zs{};
      if (inflateInit(&zs) != Z_OK) {
        *why = "zlib initialisation failed";
        return false;
      }
      zs.next_in = const_cast<unsigned char *>(e.data);
      zs.avail_in = (uInt)e.bytes;
      int rc = Z_OK;
      while (rc == Z_OK) {
        if (zs.total_out == out.size()) out.resize(out.size() * 2);
        zs.next_out = out.data() + zs.total_out;
        zs.avail_out = (uInt)(out.size() - zs.total_out);
        rc = inflate(&zs, Z_NO_FLUSH);
      }
      const size_t got = zs.total_out;
      inflateEnd(&zs);
      if (rc != Z_STREAM_END) {
        *why = "corrupt compressed element";
        return false;
      }
      out.resize(got);
      store->push_back(std::move(out));
      const std::vector<unsigned char> &body = store->back();
      size_t ip = 0;
      Element inner;
      if (!next_element(body.data(), body.size(), &ip, &inner)) {
        *why = "corrupt compressed element";
        return false;
      }
      e = inner;
    }
    if (e.type != miMATRIX) continue;  // other top-level elements carry no variables
    Array a;
    if (!parse_matrix(e.data, e.bytes, &a, 0)) {
      *why = "malformed array";
      return false;
    }
    vars->push_back(std::move(a));
  }
  return true;
}

bool read_file(const char *path, std::vector<unsigned char> *buf) {
  FILE *f = fopen(path, "rb");
  if (!f) return false;
  bool ok = fseek(f, 0, SEEK_END) == 0;
  const long size = ok ? ftell(f) : -1;
  ok = ok && size >= 0 && fseek(f, 0, SEEK_SET) == 0;
  if (ok) {
    buf->resize((size_t)size);
    ok = fread(buf->data(), 1, buf->size(), f) == buf->size();
  }
  fclose(f);
  return ok;
}

bool is_volume(const Array &a) {
  return a.cls == mxSINGLE && !a.complex && a.dims.size() == 3 && a.real.data;
}

// The subject in a data file: img, and the atlas and label volumes in field order.
struct MatSubject {
  const Array *img = nullptr;
  std::vector<const Array *> atlas, label;
  int64_t nx = -1, ny = -1, nz = -1;
};

int find_subject(const std::vector<Array> &vars, MatSubject *s) {
  for (const Array &v : vars) {
    if (v.cls == mxSTRUCT) {
      std::vector<const Array *> *dst =
          v.name == "atlas" ? &s->atlas : v.name == "atlas_label" ? &s->label : nullptr;
      if (!dst) continue;
      // field f is atlas f; of a struct array's elements the last one is kept, as the
      // reference's loop over them overwrites the same slot
      dst->clear();
      const size_t nf = v.fields.size();
      const size_t elements = nf ? v.members.size() / nf : 0;
      for (size_t f = 0; f < nf; ++f) {
        const Array *last = nullptr;
        for (size_t e = 0; e < elements; ++e)
          if (is_volume(v.members[e * nf + f])) last = &v.members[e * nf + f];
        if (last) dst->push_back(last);
      }
    } else if (v.cls >= mxDOUBLE && v.cls <= 15) {
      s->img = &v;
    }
  }
  if (!s->img || !is_volume(*s->img) || s->atlas.empty() || s->atlas.size() != s->label.size())
    return PCT_ERR_INVALID_ARG;
  s->nx = s->img->dims[0];
  s->ny = s->img->dims[1];
  s->nz = s->img->dims[2];
  if (s->nx <= 0 || s->ny <= 0 || s->nz <= 0 || s->nx * s->ny * s->nz > (int64_t)1 << 31)
    return PCT_ERR_INVALID_ARG;
  for (const auto *list : {&s->atlas, &s->label})
    for (const Array *a : *list)
      if (a->dims[0] != s->nx || a->dims[1] != s->ny || a->dims[2] != s->nz)
        return PCT_ERR_INVALID_ARG;
  return PCT_OK;
}

// Column-major [nx ny nz] (x fastest) -> [z][x][y] (y fastest).
void to_row_based(const Array &a, float *out) {
  const int64_t nx = a.dims[0], ny = a.dims[1], nz = a.dims[2];
  for (int64_t z = 0; z < nz; ++z)
    for (int64_t x = 0; x < nx; ++x)
      for (int64_t y = 0; y < ny; ++y)
        out[(z * nx + x) * ny + y] = (float)value_at(a.real, (size_t)(z * nx * ny + y * nx + x));
}

int load_subject(const char *path, std::vector<unsigned char> *file, std::vector<Array> *vars,
                 std::vector<std::vector<unsigned char>> *store, MatSubject *s) {
  if (!path) return PCT_ERR_INVALID_ARG;
  if (!read_file(path, file)) return PCT_ERR_INVALID_ARG;
  std::string why;
  if (!parse_file(*file, vars, store, &why)) {
    fprintf(stderr, "pct_b200: %s: %s\n", path, why.c_str());
    return PCT_ERR_INVALID_ARG;
  }
  return find_subject(*vars, s);
}

void put_tag(std::string &out, uint32_t type, uint32_t bytes) {
  out.append(reinterpret_cast<const char *>(&type), 4);
  out.append(reinterpret_cast<const char *>(&bytes), 4);
}

void pad8(std::string &out) { out.append((8 - out.size() % 8) % 8, '\0'); }

}  // namespace

extern "C" {

int pct_mat_dims(const char *path, int dims[4]) {
  if (!dims) return PCT_ERR_INVALID_ARG;
  std::vector<unsigned char> file;
  std::vector<Array> vars;
  std::vector<std::vector<unsigned char>> store;
  MatSubject s;
  const int st = load_subject(path, &file, &vars, &store, &s);
  if (st != PCT_OK) return st;
  dims[0] = (int)s.atlas.size();
  dims[1] = (int)s.nx;
  dims[2] = (int)s.ny;
  dims[3] = (int)s.nz;
  return PCT_OK;
}

int pct_mat_read(const char *path, float *img, float *atlas_mri, float *atlas_ct, size_t n_img,
                 size_t n_atlas) {
  if (!img || !atlas_mri || !atlas_ct) return PCT_ERR_INVALID_ARG;
  std::vector<unsigned char> file;
  std::vector<Array> vars;
  std::vector<std::vector<unsigned char>> store;
  MatSubject s;
  const int st = load_subject(path, &file, &vars, &store, &s);
  if (st != PCT_OK) return st;
  const size_t n = (size_t)(s.nx * s.ny * s.nz);
  if (n_img != n || n_atlas != n * s.atlas.size()) return PCT_ERR_INVALID_ARG;
  to_row_based(*s.img, img);
  for (size_t a = 0; a < s.atlas.size(); ++a) {
    to_row_based(*s.atlas[a], atlas_mri + a * n);
    to_row_based(*s.label[a], atlas_ct + a * n);
  }
  return PCT_OK;
}

int pct_mat_write(const char *path, const char *variable, const float *vol, int nx, int ny,
                  int nz) {
  if (!path || !variable || !vol || nx <= 0 || ny <= 0 || nz <= 0 ||
      (int64_t)nx * ny * nz * 4 > 0x7FFFFFF0LL || !*variable || strlen(variable) > 63)
    return PCT_ERR_INVALID_ARG;
  const size_t n = (size_t)nx * ny * nz;
  std::string body;
  put_tag(body, miUINT32, 8);
  const uint32_t flags[2] = {mxSINGLE, 0};
  body.append(reinterpret_cast<const char *>(flags), 8);
  put_tag(body, miINT32, 12);
  const int32_t d[3] = {nx, ny, nz};
  body.append(reinterpret_cast<const char *>(d), 12);
  pad8(body);
  const size_t name_len = strlen(variable);
  put_tag(body, miINT8, (uint32_t)name_len);
  body.append(variable, name_len);
  pad8(body);
  put_tag(body, miSINGLE, (uint32_t)(n * 4));
  const size_t data_at = body.size();
  body.resize(data_at + n * 4);
  float *col = reinterpret_cast<float *>(&body[data_at]);
  for (int z = 0; z < nz; ++z)
    for (int x = 0; x < nx; ++x)
      for (int y = 0; y < ny; ++y)
        col[(size_t)z * nx * ny + (size_t)y * nx + x] = vol[((size_t)z * nx + x) * ny + y];
  pad8(body);
  std::string header(128, ' ');
  const char text[] = "MATLAB 5.0 MAT-file, written by pct_b200";
  memcpy(&header[0], text, sizeof(text) - 1);
  memset(&header[116], 0, 8);  // no subsystem data
  header[124] = 0x00;
  header[125] = 0x01;  // version 0x0100
  header[126] = 'I';
  header[127] = 'M';
  std::string tag;
  put_tag(tag, miMATRIX, (uint32_t)body.size());
  FILE *f = fopen(path, "wb");
  if (!f) return PCT_ERR_INVALID_ARG;
  const bool ok = fwrite(header.data(), 1, header.size(), f) == header.size() &&
                  fwrite(tag.data(), 1, tag.size(), f) == tag.size() &&
                  fwrite(body.data(), 1, body.size(), f) == body.size();
  return (fclose(f) == 0 && ok) ? PCT_OK : PCT_ERR_INVALID_ARG;
}

}  // extern "C"
