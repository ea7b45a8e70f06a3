// llr-recon: the reference's command-line driver (bin/llr-recon.rs:6-25 with
// llr_recon_exec, lib.rs:113-363) on the B200 library, through the C ABI only.
//
//   llr-recon <recon_params[.toml]> <input_cfl_dir> <input_cfl_pattern> <output_cfl_dir>
//             <output_cfl_prefix> <b_table[.txt]> [--b0-null-vec-tol T] [--sample-mask-cfl PATH]
//             [--expected-volumes N] [--is-image] [--recon-b0] [--device D]
//
// Same inputs and outputs as the reference (DataSetParams, lib.rs:84-111): volumes matched by
// the glob pattern (sorted), the b-table selects the b0 or the diffusion-weighted set
// (data_import.rs:147-270), an optional (ny, nz, n_volumes) sampling mask zeroes unsampled
// x-lines (data_import.rs:416-438), linear k-space corrections are estimated per volume
// (signal_model.rs:100-106), the recon runs on the GPU, and every reconstructed volume is
// written as <prefix><index> with the index zero-padded to the digits of the volume count, plus
// error_history.json (relative data-consistency error per iteration).
//
// The parameter file uses the reference's LlrReconParams keys (lib.rs:47-81): llr_block_size,
// max_rand_shift, fft_max_batch_size, cas_mat_max_batch_size, llr_block_rank,
// wavelet_shrink_factor, n_iter, subspace_projection_mat; this driver also reads prox_mode
// ("hard" | "soft"), lambda_rel (soft threshold = lambda_rel * largest block singular value of
// the zero-filled image at shift 0) and seed.
#include <glob.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/llr_b200.h"

namespace {

[[noreturn]] void die(const std::string& msg) {
  std::fprintf(stderr, "llr-recon: %s\n", msg.c_str());
  std::exit(1);
}

void check(int st, const char* what) {
  if (st != LLR_OK) die(std::string(what) + ": " + llr_last_error());
}

std::string trim(const std::string& s) {
  const size_t a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
  return a == std::string::npos ? "" : s.substr(a, b - a + 1);
}

// key = value lines of a TOML file (scalars, strings, flat arrays); tables and comments skipped
std::map<std::string, std::string> read_toml(const std::string& path) {
  FILE* f = std::fopen(path.c_str(), "r");
  if (!f) die("failed to open config file: " + path);
  std::map<std::string, std::string> kv;
  char line[4096];
  while (std::fgets(line, sizeof line, f)) {
    std::string s(line);
    bool in_str = false;
    for (size_t i = 0; i < s.size(); ++i) {   // strip comments outside strings
      if (s[i] == '"') in_str = !in_str;
      if (s[i] == '#' && !in_str) { s = s.substr(0, i); break; }
    }
    s = trim(s);
    if (s.empty() || s[0] == '[') continue;
    const size_t eq = s.find('=');
    if (eq == std::string::npos) die("failed to parse recon params line: " + s);
    kv[trim(s.substr(0, eq))] = trim(s.substr(eq + 1));
  }
  std::fclose(f);
  return kv;
}

std::vector<double> toml_array(const std::string& v) {
  std::vector<double> out;
  std::string s = v;
  if (!s.empty() && s.front() == '[') s = s.substr(1);
  if (!s.empty() && s.back() == ']') s.pop_back();
  char* p = &s[0];
  while (*p) {
    while (*p == ' ' || *p == ',') ++p;
    if (!*p) break;
    char* end = nullptr;
    const double d = std::strtod(p, &end);
    if (end == p) die("bad array value: " + v);
    out.push_back(d);
    p = end;
  }
  return out;
}

std::string toml_string(const std::string& v) {
  if (v.size() >= 2 && v.front() == '"' && v.back() == '"') return v.substr(1, v.size() - 2);
  return v;
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
  std::vector<std::string> pos;
  float b0_tol = 0.f;
  std::string mask_path;
  long expected = -1;
  bool is_image = false, recon_b0 = false;
  int device = 0;
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    auto next = [&]() -> std::string {
      if (i + 1 >= argc) die("missing value after " + a);
      return argv[++i];
    };
    if (a == "--b0-null-vec-tol") b0_tol = std::strtof(next().c_str(), nullptr);
    else if (a == "--sample-mask-cfl") mask_path = next();
    else if (a == "--expected-volumes") expected = std::strtol(next().c_str(), nullptr, 10);
    else if (a == "--is-image") is_image = true;
    else if (a == "--recon-b0") recon_b0 = true;
    else if (a == "--device") device = (int)std::strtol(next().c_str(), nullptr, 10);
    else if (a == "-h" || a == "--help") {
      std::printf("usage: llr-recon <recon_params> <input_cfl_dir> <input_cfl_pattern> <output_cfl_dir> "
                  "<output_cfl_prefix> <b_table> [--b0-null-vec-tol T] [--sample-mask-cfl PATH] "
                  "[--expected-volumes N] [--is-image] [--recon-b0] [--device D]\n");
      return 0;
    } else pos.push_back(a);
  }
  if (pos.size() != 6) die("expected 6 positional arguments (see --help)");
  const std::string params_path = with_ext(pos[0], ".toml"), in_dir = pos[1], pattern = pos[2], out_dir = pos[3],
                    prefix = pos[4], btab = pos[5];

  // recon parameters (LlrReconParams, lib.rs:47-81)
  llr_config cfg;
  check(llr_config_default(&cfg), "config");
  cfg.device = device;
  const auto kv = read_toml(params_path);
  std::string subspace_path;
  double lambda_rel = 0.02;
  for (const auto& [k, v] : kv) {
    if (k == "llr_block_size") {
      const auto a = toml_array(v);
      if (a.size() != 3) die("llr_block_size needs 3 values");
      for (int i = 0; i < 3; ++i) cfg.block_size[i] = (int)a[i];
    } else if (k == "max_rand_shift") {
      const auto a = toml_array(v);
      if (a.size() != 3) die("max_rand_shift needs 3 values");
      for (int i = 0; i < 3; ++i) cfg.max_rand_shift[i] = (int)a[i];
    } else if (k == "fft_max_batch_size") cfg.fft_max_batch_size = std::atoi(v.c_str());
    else if (k == "cas_mat_max_batch_size") cfg.cas_mat_max_batch_size = std::atoi(v.c_str());
    else if (k == "llr_block_rank") cfg.rank = std::atoi(v.c_str());
    else if (k == "wavelet_shrink_factor") cfg.wavelet_alpha = std::strtof(v.c_str(), nullptr);
    else if (k == "n_iter") cfg.n_iter = std::atoi(v.c_str());
    else if (k == "subspace_projection_mat") subspace_path = toml_string(v);
    else if (k == "prox_mode") {
      const std::string m = toml_string(v);
      if (m == "hard") cfg.prox_mode = LLR_PROX_HARD_RANK;
      else if (m == "soft") cfg.prox_mode = LLR_PROX_SOFT_THRESH;
      else die("prox_mode must be \"hard\" or \"soft\"");
    } else if (k == "lambda_rel") lambda_rel = std::strtod(v.c_str(), nullptr);
    else if (k == "seed") cfg.seed = std::strtoull(v.c_str(), nullptr, 10);
    else die("unknown recon parameter: " + k);
  }

  // volumes (data_import.rs:67-108)
  glob_t gl;
  const std::string full = with_ext(join(in_dir, pattern), ".cfl");
  if (glob(full.c_str(), 0, nullptr, &gl) != 0 || gl.gl_pathc == 0) die("no files found for " + full);
  std::vector<std::string> files(gl.gl_pathv, gl.gl_pathv + gl.gl_pathc);
  globfree(&gl);
  std::sort(files.begin(), files.end());
  if (expected >= 0 && (long)files.size() != expected) die("unexpected number of files found");
  const auto vd = squeezed_dims(files[0]);
  if (vd.size() != 3) die("expecting n volume dims to be 3");
  for (const auto& f : files)
    if (squeezed_dims(f) != vd) die("mismatch between first volume dims and volume " + f);
  const int nx = (int)vd[0], ny = (int)vd[1], nz = (int)vd[2], n_all = (int)files.size();
  const long long V = (long long)nx * ny * nz;

  // b-table and the volume set (data_import.rs:110-145, 256-268)
  std::vector<float> bval(n_all), bvec(3 * n_all);
  check(llr_read_b_table(btab.c_str(), n_all, bval.data(), bvec.data()), "b-table");
  std::vector<uint8_t> is_b0(n_all);
  check(llr_b0_mask(bvec.data(), n_all, b0_tol, is_b0.data()), "b0 mask");
  std::vector<int> idx;
  for (int i = 0; i < n_all; ++i)
    if ((bool)is_b0[i] == recon_b0) idx.push_back(i);
  const int nq = (int)idx.size();
  if (nq == 0) die(recon_b0 ? "no b0 volumes" : "no diffusion-weighted volumes");

  std::vector<llr_cf32> data((size_t)V * nq);
  for (int q = 0; q < nq; ++q)
    check(llr_cfl_read(files[idx[q]].c_str(), data.data() + (size_t)V * q, V), "volume");
  if (is_image) {   // image -> k-space with zero corrections (lib.rs:153-167)
    const size_t sz[3] = {(size_t)nx, (size_t)ny, (size_t)nz};
    check(llr_signal_model(data.data(), sz, (size_t)nq, nullptr, nullptr, LLR_FORWARD), "forward model");
  }
  if (!mask_path.empty()) {   // under_sample_kspace (data_import.rs:416-438)
    const auto md = squeezed_dims(mask_path);
    if (md.size() != 3 || md[0] != ny || md[1] != nz || md[2] != n_all) die("sample mask must be (ny, nz, n_volumes)");
    std::vector<llr_cf32> mask((size_t)ny * nz * n_all);
    check(llr_cfl_read(mask_path.c_str(), mask.data(), (int64_t)mask.size()), "sample mask");
    for (int q = 0; q < nq; ++q)
      for (long long yz = 0; yz < (long long)ny * nz; ++yz) {
        const llr_cf32 mv = mask[(size_t)idx[q] * ny * nz + yz];
        if (mv.re == 0.f && mv.im == 0.f)
          for (int x = 0; x < nx; ++x) data[(size_t)V * q + (size_t)yz * nx + x] = llr_cf32{0.f, 0.f};
      }
  }

  // subspace matrix (lib.rs:212-222)
  std::vector<llr_cf32> S;
  if (!subspace_path.empty()) {
    const auto sd = squeezed_dims(subspace_path);
    if (sd.size() != 2 || sd[0] != nq) die("subspace matrix must be (nq, rank)");
    S.resize((size_t)sd[0] * sd[1]);
    check(llr_cfl_read(subspace_path.c_str(), S.data(), (int64_t)S.size()), "subspace matrix");
    cfg.subspace_rank = (int)sd[1];
  }

  cfg.vol_size[0] = nx; cfg.vol_size[1] = ny; cfg.vol_size[2] = nz;
  cfg.nq = nq;
  check(llr_config_validate(&cfg), "recon params");
  std::vector<float> lin_ksp(3 * (size_t)nq), lin_img(3 * (size_t)nq, 0.f);
  const int32_t vs[3] = {nx, ny, nz};
  check(llr_estimate_linear_corrections(data.data(), vs, nq, lin_ksp.data()), "linear corrections");

  llr_ctx* ctx = nullptr;
  check(llr_ctx_create(&cfg, &ctx), "context");
  check(llr_set_linear_corrections(ctx, lin_ksp.data(), lin_img.data()), "linear corrections");
  check(llr_upload_kspace(ctx, data.data()), "k-space");
  if (!S.empty()) check(llr_upload_subspace(ctx, S.data()), "subspace");
  double energy = 0.0, us = 0.0;
  check(llr_measurement_stats(ctx, &energy, &us), "measurement stats");
  std::printf("under sampling factor: %.03f\n", us);
  check(llr_init_zero_filled(ctx), "zero-filled image");
  if (cfg.prox_mode == LLR_PROX_SOFT_THRESH) {
    const int32_t zero[3] = {0, 0, 0};
    double smax = 0.0;
    check(llr_sigma_max(ctx, zero, &smax), "sigma_max");
    check(llr_set_lambda(ctx, (float)(lambda_rel * smax)), "lambda");
  }
  std::vector<double> hist((size_t)std::max(cfg.n_iter, 1));
  check(llr_iterate(ctx, cfg.n_iter, hist.data()), "iterate");
  check(llr_download_image(ctx, data.data()), "download");
  check(llr_ctx_destroy(ctx), "destroy");

  // error_history.json and the volumes (lib.rs:345-362)
  {
    FILE* f = std::fopen(join(out_dir, "error_history.json").c_str(), "w");
    if (!f) die("failed to create json file");
    std::fprintf(f, "[\n");
    for (int i = 0; i < cfg.n_iter; ++i)
      std::fprintf(f, "  %.17g%s\n", energy > 0 ? hist[i] / energy : hist[i], i + 1 < cfg.n_iter ? "," : "");
    std::fprintf(f, "]\n");
    std::fclose(f);
  }
  const int width = (int)std::to_string(n_all).size();
  for (int q = 0; q < nq; ++q) {
    char name[64];
    std::snprintf(name, sizeof name, "%0*d", width, idx[q]);
    const int64_t dims[3] = {nx, ny, nz};
    check(llr_cfl_write(join(out_dir, prefix + name).c_str(), dims, 3, data.data() + (size_t)V * q), "write volume");
  }
  std::printf("wrote %d volumes to %s\n", nq, out_dir.c_str());
  return 0;
}
