// llr-dti-scalars: DTI scalar maps of reconstructed volumes (diffusion_models.rs:21-129,
// calc_scalars) on the GPU through the C ABI.
//
//   llr-dti-scalars <input_cfl_dir> <cfl_pattern> <b_table[.txt]> <output_dir> <n_expected_vols>
//
// Reads the volumes matched by the pattern (sorted), splits b0 and diffusion-weighted sets with
// the gradient-norm tolerance 1e-6 (as there), fits the tensor per voxel and writes b0av, e1,
// e2, e3, md, rd and fa as (nx, ny, nz) CFL volumes (real values, zero imaginary part).
#include <glob.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "../../include/llr_b200.h"

namespace {

[[noreturn]] void die(const std::string& msg) {
  std::fprintf(stderr, "llr-dti-scalars: %s\n", msg.c_str());
  std::exit(1);
}

void check(int st, const char* what) {
  if (st != LLR_OK) die(std::string(what) + ": " + llr_last_error());
}

std::string with_ext(const std::string& p, const char* ext) {
  const size_t slash = p.find_last_of('/'), dot = p.find_last_of('.');
  if (dot != std::string::npos && (slash == std::string::npos || dot > slash)) return p.substr(0, dot) + ext;
  return p + ext;
}

std::string join(const std::string& dir, const std::string& name) {
  if (dir.empty() || dir.back() == '/') return dir + name;
  return dir + "/" + name;
}

std::vector<int64_t> squeezed_dims(const std::string& path) {
  int64_t d[16];
  int32_t nd = 0;
  check(llr_cfl_dims(path.c_str(), d, 16, &nd), "cfl header");
  std::vector<int64_t> out;
  for (int i = 0; i < nd; ++i)
    if (d[i] != 1) out.push_back(d[i]);
  return out;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc != 6) die("usage: llr-dti-scalars <input_cfl_dir> <cfl_pattern> <b_table> <output_dir> <n_expected_vols>");
  const std::string in_dir = argv[1], pattern = argv[2], btab = argv[3], out_dir = argv[4];
  const long expected = std::strtol(argv[5], nullptr, 10);
  glob_t gl;
  const std::string full = with_ext(join(in_dir, pattern), ".cfl");
  if (glob(full.c_str(), 0, nullptr, &gl) != 0 || gl.gl_pathc == 0) die("no files found for " + full);
  std::vector<std::string> files(gl.gl_pathv, gl.gl_pathv + gl.gl_pathc);
  globfree(&gl);
  std::sort(files.begin(), files.end());
  if ((long)files.size() != expected) die("unexpected number of files found");
  const auto vd = squeezed_dims(files[0]);
  if (vd.size() != 3) die("expecting n volume dims to be 3");
  for (const auto& f : files)
    if (squeezed_dims(f) != vd) die("mismatch between first volume dims and volume " + f);
  const int n_all = (int)files.size();
  const long long V = vd[0] * vd[1] * vd[2];
  std::vector<float> bval(n_all), bvec(3 * (size_t)n_all);
  check(llr_read_b_table(btab.c_str(), n_all, bval.data(), bvec.data()), "b-table");
  std::vector<uint8_t> is_b0(n_all);
  check(llr_b0_mask(bvec.data(), n_all, 1e-6f, is_b0.data()), "b0 mask");
  std::vector<llr_cf32> dwi, b0;
  std::vector<float> b, g;
  std::vector<llr_cf32> vol((size_t)V);
  for (int i = 0; i < n_all; ++i) {
    check(llr_cfl_read(files[i].c_str(), vol.data(), V), "volume");
    auto& dst = is_b0[i] ? b0 : dwi;
    dst.insert(dst.end(), vol.begin(), vol.end());
    if (!is_b0[i]) {
      b.push_back(bval[i]);
      g.insert(g.end(), bvec.begin() + 3 * i, bvec.begin() + 3 * i + 3);
    }
  }
  const int nq = (int)b.size(), nb0 = n_all - nq;
  std::vector<float> out((size_t)V * 7);
  check(llr_dti_fit(dwi.data(), nq, nb0 ? b0.data() : nullptr, nb0, V, b.data(), g.data(), out.data()), "DTI fit");
  const char* names[7] = {"b0av", "e1", "e2", "e3", "md", "rd", "fa"};
  const int64_t dims[3] = {vd[0], vd[1], vd[2]};
  for (int k = 0; k < 7; ++k) {
    for (long long v = 0; v < V; ++v) vol[(size_t)v] = llr_cf32{out[(size_t)k * V + v], 0.f};
    check(llr_cfl_write(join(out_dir, names[k]).c_str(), dims, 3, vol.data()), "write");
  }
  std::printf("wrote b0av, e1, e2, e3, md, rd, fa to %s\n", out_dir.c_str());
  return 0;
}
