// CFL volume IO and the b-table reader: the file formats of the reference's dataset builder
// (data_import.rs:67-145, 187-202) and output writer (lib.rs:353-362).
//
// A CFL data set is a pair of files: <name>.hdr, text, "# Dimensions" then one line of
// whitespace-separated sizes (column-major, first fastest), and <name>.cfl, raw little-endian
// complex64 (interleaved FP32 re, im) in that column-major order.  A b-table is whitespace-
// separated numbers, four per volume: b-value, gx, gy, gz (data_import.rs:110-145).
#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "llr_common.cuh"

using namespace llr;

namespace {

std::string strip_ext(const char* path) {
  std::string p(path);
  const size_t slash = p.find_last_of('/');
  const size_t dot = p.find_last_of('.');
  if (dot != std::string::npos && (slash == std::string::npos || dot > slash)) {
    const std::string ext = p.substr(dot);
    if (ext == ".cfl" || ext == ".hdr") p = p.substr(0, dot);
  }
  return p;
}

int read_dims(const std::string& base, std::vector<long long>& dims) {
  FILE* f = std::fopen((base + ".hdr").c_str(), "r");
  if (!f) return set_error(LLR_ERR_INVALID, "cannot open %s.hdr: %s", base.c_str(), std::strerror(errno));
  char line[4096];
  dims.clear();
  bool want = false;
  while (std::fgets(line, sizeof line, f)) {
    if (line[0] == '#') {
      want = std::strstr(line, "Dimensions") != nullptr;
      continue;
    }
    if (!want) continue;
    char* p = line;
    while (*p) {
      char* end = nullptr;
      const long long v = std::strtoll(p, &end, 10);
      if (end == p) break;
      dims.push_back(v);
      p = end;
    }
    break;
  }
  std::fclose(f);
  if (dims.empty()) return set_error(LLR_ERR_INVALID, "%s.hdr has no dimensions line", base.c_str());
  for (long long d : dims)
    if (d < 1) return set_error(LLR_ERR_INVALID, "%s.hdr has a non-positive dimension", base.c_str());
  return LLR_OK;
}

}  // namespace

extern "C" {

int llr_cfl_dims(const char* path, int64_t* dims, int32_t max_dims, int32_t* ndims) {
  if (!path || !dims || !ndims || max_dims < 1) return set_error(LLR_ERR_INVALID, "null pointer");
  std::vector<long long> d;
  LLR_TRY(read_dims(strip_ext(path), d));
  if ((int)d.size() > max_dims) return set_error(LLR_ERR_INVALID, "%s: %zu dimensions > %d", path, d.size(), max_dims);
  for (size_t i = 0; i < d.size(); ++i) dims[i] = d[i];
  *ndims = (int32_t)d.size();
  return LLR_OK;
}

int llr_cfl_read(const char* path, llr_cf32* dst, int64_t count) {
  if (!path || !dst || count < 0) return set_error(LLR_ERR_INVALID, "null pointer");
  const std::string base = strip_ext(path);
  std::vector<long long> d;
  LLR_TRY(read_dims(base, d));
  long long n = 1;
  for (long long v : d) n *= v;
  if (n != count) return set_error(LLR_ERR_INVALID, "%s holds %lld elements, %lld expected", path, n, (long long)count);
  FILE* f = std::fopen((base + ".cfl").c_str(), "rb");
  if (!f) return set_error(LLR_ERR_INVALID, "cannot open %s.cfl: %s", base.c_str(), std::strerror(errno));
  const size_t got = std::fread(dst, sizeof(llr_cf32), (size_t)n, f);
  std::fclose(f);
  if (got != (size_t)n) return set_error(LLR_ERR_INVALID, "%s.cfl is short (%zu of %lld elements)", base.c_str(), got, n);
  return LLR_OK;
}

int llr_cfl_write(const char* path, const int64_t* dims, int32_t ndims, const llr_cf32* src) {
  if (!path || !dims || !src || ndims < 1) return set_error(LLR_ERR_INVALID, "null pointer");
  const std::string base = strip_ext(path);
  long long n = 1;
  for (int i = 0; i < ndims; ++i) {
    if (dims[i] < 1) return set_error(LLR_ERR_INVALID, "non-positive dimension");
    n *= dims[i];
  }
  FILE* h = std::fopen((base + ".hdr").c_str(), "w");
  if (!h) return set_error(LLR_ERR_INVALID, "cannot create %s.hdr: %s", base.c_str(), std::strerror(errno));
  std::fprintf(h, "# Dimensions\n");
  for (int i = 0; i < ndims; ++i) std::fprintf(h, "%lld%s", (long long)dims[i], i + 1 < ndims ? " " : "\n");
  std::fclose(h);
  FILE* f = std::fopen((base + ".cfl").c_str(), "wb");
  if (!f) return set_error(LLR_ERR_INVALID, "cannot create %s.cfl: %s", base.c_str(), std::strerror(errno));
  const size_t put = std::fwrite(src, sizeof(llr_cf32), (size_t)n, f);
  const int rc = std::fclose(f);
  if (put != (size_t)n || rc != 0) return set_error(LLR_ERR_INVALID, "short write to %s.cfl", base.c_str());
  return LLR_OK;
}

int llr_read_b_table(const char* path, int32_t n_vols, float* b_vals, float* b_vecs) {
  if (!path || !b_vals || !b_vecs || n_vols < 1) return set_error(LLR_ERR_INVALID, "null pointer");
  std::string p(path);
  const size_t slash = p.find_last_of('/'), dot = p.find_last_of('.');
  if (dot == std::string::npos || (slash != std::string::npos && dot < slash)) p += ".txt";   // with_extension("txt")
  FILE* f = std::fopen(p.c_str(), "r");
  if (!f) return set_error(LLR_ERR_INVALID, "cannot open b-table %s: %s", p.c_str(), std::strerror(errno));
  std::vector<float> v;
  char tok[256];
  while (std::fscanf(f, "%255s", tok) == 1) {
    char* end = nullptr;
    const float x = std::strtof(tok, &end);
    if (end == tok || *end != '\0') {
      std::fclose(f);
      return set_error(LLR_ERR_INVALID, "failed to parse b-table at %s", tok);
    }
    v.push_back(x);
  }
  std::fclose(f);
  if (v.size() % 4 != 0) return set_error(LLR_ERR_INVALID, "b-table entries must be a multiple of 4 (b, gx, gy, gz)");
  if ((long long)v.size() / 4 != n_vols)
    return set_error(LLR_ERR_INVALID, "expected %d b-vectors, read %zu", n_vols, v.size() / 4);
  for (int i = 0; i < n_vols; ++i) {
    b_vals[i] = v[4 * i];
    for (int a = 0; a < 3; ++a) b_vecs[3 * i + a] = v[4 * i + 1 + a];
  }
  return LLR_OK;
}

int llr_read_affine_translation(const char* path, float multiplier, float* translation) {
  if (!path || !translation) return set_error(LLR_ERR_INVALID, "null pointer");
  FILE* f = std::fopen(path, "r");
  if (!f) return set_error(LLR_ERR_INVALID, "failed to open %s: %s", path, std::strerror(errno));
  std::string line;
  char buf[4096];
  bool found = false;
  std::vector<float> v;
  while (!found && std::fgets(buf, sizeof buf, f)) {
    line = buf;
    if (line.find("Parameters:") == std::string::npos) continue;
    found = true;
    // every whitespace-separated token that parses completely as a number
    size_t i = 0;
    while (i < line.size()) {
      while (i < line.size() && std::isspace((unsigned char)line[i])) ++i;
      size_t j = i;
      while (j < line.size() && !std::isspace((unsigned char)line[j])) ++j;
      if (j > i) {
        const std::string tok = line.substr(i, j - i);
        char* end = nullptr;
        const float x = std::strtof(tok.c_str(), &end);
        if (end && *end == '\0') v.push_back(x);
      }
      i = j;
    }
  }
  std::fclose(f);
  if (!found) return set_error(LLR_ERR_INVALID, "failed to find Parameter field in affine file %s", path);
  if (v.size() != 12) return set_error(LLR_ERR_INVALID, "expected 12 matrix entries in %s, read %zu", path, v.size());
  for (int a = 0; a < 3; ++a) translation[a] = v[9 + a] * multiplier;   // signal_model.rs:148-176
  return LLR_OK;
}

int llr_b0_mask(const float* b_vecs, int32_t n_vols, float tol, uint8_t* is_b0) {
  if (!b_vecs || !is_b0 || n_vols < 0) return set_error(LLR_ERR_INVALID, "null pointer");
  if (!(tol >= 0.f)) return set_error(LLR_ERR_INVALID, "vector magnitude tolerance must be non-negative");
  for (int i = 0; i < n_vols; ++i) {
    const float* g = b_vecs + 3 * i;
    is_b0[i] = std::sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]) <= tol ? 1 : 0;   // data_import.rs:322-328
  }
  return LLR_OK;
}

}  // extern "C"
