// C ABI: library-level entry points, counter RNG, masks, filters, device-pointer operators
// and host-slice entry points that keep the reference's argument order.
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <cmath>
#include <complex>
#include <vector>
#include <algorithm>

#include "llr_internal.h"

namespace llr {

namespace {
thread_local char g_err[1024] = "";
}

int set_error(int status, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return status;
}

int cuda_error(cudaError_t e, const char* what, const char* file, int line) {
  const char* base = strrchr(file, '/');
  set_error(e == cudaErrorMemoryAllocation ? LLR_ERR_NOMEM
            : (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) ? LLR_ERR_NO_DEVICE
                                                                           : LLR_ERR_CUDA,
            "%s failed: %s (%s:%d)", what, cudaGetErrorString(e), base ? base + 1 : file, line);
  if (e == cudaErrorMemoryAllocation) return LLR_ERR_NOMEM;
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return LLR_ERR_NO_DEVICE;
  return LLR_ERR_CUDA;
}

// Daubechies scaling filter (reconstruction order, sum = sqrt 2) by spectral factorisation
// of P(y) = sum_k C(N-1+k, k) y^k (Daubechies 1992, sec. 6.1); roots by Durand-Kerner.
int daubechies_host(int order, double* h) {
  if (order < 1 || order > 10) return set_error(LLR_ERR_INVALID, "Daubechies order %d outside [1, 10]", order);
  const int N = order;
  typedef std::complex<double> cd;
  std::vector<cd> poly(1, cd(1.0, 0.0));  // coefficients, highest degree first
  auto conv = [](const std::vector<cd>& a, const std::vector<cd>& b) {
    std::vector<cd> c(a.size() + b.size() - 1, cd(0, 0));
    for (size_t i = 0; i < a.size(); ++i)
      for (size_t j = 0; j < b.size(); ++j) c[i + j] += a[i] * b[j];
    return c;
  };
  for (int k = 0; k < N; ++k) poly = conv(poly, {cd(1, 0), cd(1, 0)});
  if (N > 1) {
    // P coefficients p_k = C(N-1+k, k), k = 0..N-1; monic in y after dividing by p_{N-1}
    std::vector<double> p(N);
    for (int k = 0; k < N; ++k) {
      double c = 1.0;
      for (int i = 1; i <= k; ++i) c = c * (N - 1 + i) / i;
      p[k] = c;
    }
    const int deg = N - 1;
    std::vector<cd> roots(deg);
    const cd seed(0.4, 0.9);
    for (int i = 0; i < deg; ++i) roots[i] = std::pow(seed, i);
    auto evalP = [&](cd y) {
      cd v(0, 0);
      for (int k = deg; k >= 0; --k) v = v * y + p[k];
      return v / p[deg];
    };
    for (int it = 0; it < 2000; ++it) {
      double delta = 0;
      for (int i = 0; i < deg; ++i) {
        cd den(1, 0);
        for (int j = 0; j < deg; ++j)
          if (j != i) den *= (roots[i] - roots[j]);
        const cd step = evalP(roots[i]) / den;
        roots[i] -= step;
        delta = std::max(delta, std::abs(step));
      }
      if (delta < 1e-15) break;
    }
    for (int i = 0; i < deg; ++i) {
      // z + 1/z = 2 - 4y  ->  z^2 - (2 - 4y) z + 1 = 0; keep |z| < 1
      const cd b = -(2.0 - 4.0 * roots[i]);
      const cd disc = std::sqrt(b * b - 4.0);
      cd z1 = (-b + disc) / 2.0, z2 = (-b - disc) / 2.0;
      const cd z = std::abs(z1) < std::abs(z2) ? z1 : z2;
      poly = conv(poly, {cd(1, 0), -z});
    }
  }
  double sum = 0;
  for (size_t i = 0; i < poly.size(); ++i) sum += poly[i].real();
  const double sc = std::sqrt(2.0) / sum;
  for (int i = 0; i < 2 * N; ++i) h[i] = poly[i].real() * sc;
  return LLR_OK;
}

int signal_model_dev(float2* d_x, const int dims[3], int batch, const float* lin_ksp, const float* lin_img,
                     int direction, cudaStream_t s);
int launch_lift(const float2* vol, float2* mat, const int* vs, int nq, const int* bs, const int* sh, long long start,
                long long n, int dir, cudaStream_t s);
int launch_rhs_cdgmm(int m, int n, int batch, float2* a, const float* d, cudaStream_t s);
int launch_cgemm(int m, int k, int n, int batch, int broadcast_a, float2 alpha, float2 beta, int ta, int tb,
                 const float2* A, const float2* B, float2* C, cudaStream_t s);
int launch_dwt_axis_ref(const float2* vol, float2* dec, const uint32_t* vs, const uint32_t* ds, int axis,
                        const float* lo, const float* hi, int F, const int* sh, int inverse, cudaStream_t s,
                        const float* d_lo = nullptr, const float* d_hi = nullptr, const int* d_sh = nullptr);
int launch_hard_project(float2* x, const float2* y, long long n, double* partials, int nblocks, cudaStream_t s);
int launch_conj_transpose(const float2* in, float2* out, int m, int n, int batch, cudaStream_t s);
int launch_finalize(const double* partials, int np, double scale, double* hist, long long cap, long long* it,
                    int advance, double* out, cudaStream_t s);

// RAII device buffer for host-slice entry points.
struct DevBuf {
  void* p = nullptr;
  ~DevBuf() { if (p) cudaFree(p); }
  int alloc(size_t bytes) {
    cudaError_t e = cudaMalloc(&p, bytes ? bytes : 16);
    if (e != cudaSuccess) { p = nullptr; return cuda_error(e, "cudaMalloc", __FILE__, __LINE__); }
    return LLR_OK;
  }
  template <class T> T* as() { return reinterpret_cast<T*>(p); }
};

}  // namespace llr

using namespace llr;

extern "C" {

const char* llr_version(void) { return "llr-b200 0.1.0 (sm_100a)"; }
const char* llr_last_error(void) { return g_err; }

const char* llr_status_string(int s) {
  switch (s) {
    case LLR_OK: return "ok";
    case LLR_ERR_INVALID: return "invalid argument";
    case LLR_ERR_CUDA: return "CUDA error";
    case LLR_ERR_CUFFT: return "cuFFT error";
    case LLR_ERR_NOMEM: return "out of memory";
    case LLR_ERR_NOT_FINITE: return "non-finite objective";
    case LLR_ERR_STATE: return "call out of order";
    case LLR_ERR_UNSUPPORTED: return "unsupported shape";
    case LLR_ERR_NO_DEVICE: return "no CUDA device";
    default: return "unknown status";
  }
}

int llr_config_default(llr_config* c) {
  if (!c) return set_error(LLR_ERR_INVALID, "null config");
  memset(c, 0, sizeof(*c));
  for (int a = 0; a < 3; ++a) c->block_size[a] = 32;   // lib.rs:70
  c->prox_mode = LLR_PROX_HARD_RANK;
  c->rank = 6;                                          // lib.rs:74
  c->lambda = 0.f;
  c->wavelet_alpha = 0.005f;                            // lib.rs:75
  c->wavelet_moments = 2;                               // Daubechies2 (lib.rs:439)
  c->wavelet_levels = 0;
  c->subspace_rank = 0;
  c->fft_max_batch_size = 200;                          // lib.rs:72
  c->cas_mat_max_batch_size = 200;                      // lib.rs:73
  c->n_iter = 60;                                       // lib.rs:76
  c->seed = 0;
  c->device = 0;
  return LLR_OK;
}

int llr_config_validate(const llr_config* c) {
  if (!c) return set_error(LLR_ERR_INVALID, "null config");
  for (int a = 0; a < 3; ++a) {
    if (c->vol_size[a] < 1) return set_error(LLR_ERR_INVALID, "vol_size[%d] = %d must be >= 1", a, c->vol_size[a]);
    if (c->block_size[a] < 1 || c->block_size[a] > c->vol_size[a])
      return set_error(LLR_ERR_INVALID, "block dimension must be in [1, volume dimension] (block.rs:69-71)");
    if (c->max_rand_shift[a] < 0 || c->max_rand_shift[a] > c->vol_size[a])
      return set_error(LLR_ERR_INVALID, "max_rand_shift[%d] must be in [0, vol_size]", a);
  }
  if (c->nq < 1) return set_error(LLR_ERR_INVALID, "nq must be >= 1");
  const long long m = (long long)c->block_size[0] * c->block_size[1] * c->block_size[2];
  const int n = c->subspace_rank > 0 ? c->subspace_rank : c->nq;
  if (c->prox_mode != LLR_PROX_HARD_RANK && c->prox_mode != LLR_PROX_SOFT_THRESH)
    return set_error(LLR_ERR_INVALID, "unknown prox_mode %d", c->prox_mode);
  if (c->prox_mode == LLR_PROX_HARD_RANK) {
    if (c->rank < 1) return set_error(LLR_ERR_INVALID, "rank should not be less than 1 (lib.rs:207)");
    if (c->rank > n) return set_error(LLR_ERR_INVALID, "rank must not exceed n (lib.rs:205)");
  } else if (!(c->lambda >= 0.f)) {
    return set_error(LLR_ERR_INVALID, "lambda must be >= 0");
  }
  if (c->subspace_rank < 0 || c->subspace_rank > c->nq)
    return set_error(LLR_ERR_INVALID, "subspace rank must be in [0, nq] (lib.rs:215-217)");
  if (c->subspace_rank > 0 && c->prox_mode == LLR_PROX_HARD_RANK && c->rank > c->subspace_rank)
    return set_error(LLR_ERR_INVALID, "llr rank must be <= subspace rank (lib.rs:217)");
  if (!(c->wavelet_alpha >= 0.f)) return set_error(LLR_ERR_INVALID, "wavelet_alpha must be >= 0");
  if (c->eig_solver < 0 || c->eig_solver > 1) return set_error(LLR_ERR_INVALID, "eig_solver must be 0 or 1");
  if (c->gram_mode != 0 && c->gram_mode != 1) return set_error(LLR_ERR_INVALID, "gram_mode must be 0 or 1");
  if (c->fft_mode != 0 && c->fft_mode != 1) return set_error(LLR_ERR_INVALID, "fft_mode must be 0 or 1");
  if (c->wavelet_alpha > 0.f && (c->wavelet_moments < 1 || c->wavelet_moments > 10))
    return set_error(LLR_ERR_INVALID, "wavelet_moments must be in [1, 10]");
  if (c->wavelet_space != 0 && c->wavelet_space != 1) return set_error(LLR_ERR_INVALID, "wavelet_space must be 0 or 1");
  bool tiles = true, overlap = false;
  for (int a = 0; a < 3; ++a) {
    const int b = c->block_size[a], st = c->block_stride[a];
    if (st < 0 || st > b) return set_error(LLR_ERR_INVALID, "block_stride[%d] must be in [0, block size]", a);
    if (st > 0 && st < b) {
      overlap = true;
      if (b % st != 0) return set_error(LLR_ERR_INVALID, "block size must be a multiple of block_stride");
    }
    if (c->vol_size[a] % b != 0) tiles = false;
  }
  if (overlap && !tiles) return set_error(LLR_ERR_UNSUPPORTED, "overlapping blocks need a volume the blocks tile");
  if (overlap && c->subspace_rank > 0)
    return set_error(LLR_ERR_UNSUPPORTED, "overlapping blocks are not combined with a subspace");
  if (c->wavelet_space == 1 && c->subspace_rank > 0 && c->wavelet_alpha > 0.f && !tiles)
    return set_error(LLR_ERR_UNSUPPORTED, "subspace-coefficient wavelet needs a volume the blocks tile");
  if (m < 1) return set_error(LLR_ERR_INVALID, "empty block");
  const long long E = (long long)c->vol_size[0] * c->vol_size[1] * c->vol_size[2] * c->nq;
  if (E >= (1LL << 31) * 2) return set_error(LLR_ERR_UNSUPPORTED, "dataset of %lld elements too large", E);
  return LLR_OK;
}

int llr_rand_shift(uint64_t seed, int64_t it, const int32_t* mx, int32_t* out) {
  if (!mx || !out) return set_error(LLR_ERR_INVALID, "null pointer");
  for (int a = 0; a < 3; ++a) {
    if (mx[a] < 1) return set_error(LLR_ERR_INVALID, "max shift must be >= 1");
    out[a] = llr_shift_draw(seed, it, a, mx[a]);
  }
  return LLR_OK;
}

int llr_grid_dim(const int32_t* vs, const int32_t* bs, int32_t* out) {
  if (!vs || !bs || !out) return set_error(LLR_ERR_INVALID, "null pointer");
  for (int a = 0; a < 3; ++a) {
    if (bs[a] < 1) return set_error(LLR_ERR_INVALID, "block size must be >= 1");
    out[a] = vs[a] / bs[a];
  }
  return LLR_OK;
}

int llr_vd_mask(int32_t ny, int32_t nz, int32_t nq, double accel, int32_t centre, uint64_t seed, uint8_t* out) {
  if (ny < 1 || nz < 1 || nq < 1 || !(accel >= 1.0) || centre < 0 || !out)
    return set_error(LLR_ERR_INVALID, "bad mask arguments");
  const int cy = ny / 2, cz = nz / 2;
  std::vector<double> w((size_t)ny * nz);
  for (int j = 0; j < ny; ++j) {
    const double dy = ((double)j - cy) / (ny / 2.0);
    for (int k = 0; k < nz; ++k) {
      const double dz = ((double)k - cz) / (nz / 2.0);
      const double r = std::sqrt(dy * dy + dz * dz);
      const double t = 1.0 - (r < 1.0 ? r : 1.0);
      w[(size_t)j * nz + k] = t * t + 0.02;
    }
  }
  const int h0 = centre / 2;
  std::vector<char> inc((size_t)ny * nz, 0);
  long long n_inc = 0;
  for (int j = std::max(cy - h0, 0); j < std::min(cy - h0 + centre, ny); ++j)
    for (int k = std::max(cz - h0, 0); k < std::min(cz - h0 + centre, nz); ++k) {
      inc[(size_t)j * nz + k] = 1;
      ++n_inc;
    }
  const long long target = (long long)std::nearbyint((double)ny * nz / accel);
  const long long rest = std::max(target - n_inc, 0LL);
  const double TWO32 = 4294967296.0;
  auto quant_sum = [&](double a, std::vector<uint64_t>* qv) {
    unsigned long long s = 0;
    for (size_t i = 0; i < w.size(); ++i) {
      uint64_t v = 0;
      if (!inc[i]) {
        double p = a * w[i];
        p = p > 1.0 ? 1.0 : p;
        v = (uint64_t)std::floor(p * TWO32);
      }
      if (qv) (*qv)[i] = v;
      s += v;
    }
    return s;
  };
  const unsigned long long goal = (unsigned long long)rest << 32;
  double lo = 0.0, hi = 1.0;
  while (quant_sum(hi, nullptr) < goal && hi < 1e12) hi *= 2.0;
  for (int i = 0; i < 60; ++i) {
    const double mid = 0.5 * (lo + hi);
    if (quant_sum(mid, nullptr) < goal) lo = mid;
    else hi = mid;
  }
  std::vector<uint64_t> qv(w.size());
  quant_sum(hi, &qv);
  for (int q = 0; q < nq; ++q)
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j) {
        const size_t wi = (size_t)j * nz + k;
        uint8_t v;
        if (inc[wi]) v = 1;
        else {
          const uint64_t u = llr_rng_u64(seed, LLR_MASK_STREAM + ((uint64_t)q << 8), (uint64_t)(j + (long long)ny * k)) >> 32;
          v = u < qv[wi] ? 1 : 0;
        }
        out[(size_t)j + (size_t)ny * ((size_t)k + (size_t)nz * q)] = v;
      }
  return LLR_OK;
}

int llr_daubechies_filters(int32_t order, float* lo_d, float* hi_d, float* lo_r, float* hi_r) {
  double h[20];
  LLR_TRY(daubechies_host(order, h));
  const int F = 2 * order;
  for (int k = 0; k < F; ++k) {
    const double lr = h[k];
    const double hr = ((k & 1) ? -1.0 : 1.0) * h[F - 1 - k];
    if (lo_r) lo_r[k] = (float)lr;
    if (hi_r) hi_r[k] = (float)hr;
    if (lo_d) lo_d[F - 1 - k] = (float)lr;
    if (hi_d) hi_d[F - 1 - k] = (float)hr;
  }
  return LLR_OK;
}

int llr_estimate_linear_corrections(const llr_cf32* y, const int32_t* vs, int32_t nq, float* out) {
  if (!y || !vs || !out || nq < 1) return set_error(LLR_ERR_INVALID, "null pointer");
  const long long V = (long long)vs[0] * vs[1] * vs[2];
  for (int q = 0; q < nq; ++q) {
    const llr_cf32* v = y + V * q;
    long long best = 0;
    float bv = -1.f;
    for (long long i = 0; i < V; ++i) {  // last index among equal maxima (cufft.rs:332-335)
      const float e = v[i].re * v[i].re + v[i].im * v[i].im;
      if (e >= bv) { bv = e; best = i; }
    }
    const int ix = (int)(best % vs[0]);
    const int iy = (int)((best / vs[0]) % vs[1]);
    const int iz = (int)(best / ((long long)vs[0] * vs[1]));
    out[3 * q + 0] = (float)(ix - (vs[0] + 1) / 2);   // signal_model.rs:100-106
    out[3 * q + 1] = (float)(iy - (vs[1] + 1) / 2);
    out[3 * q + 2] = (float)(iz - (vs[2] + 1) / 2);
  }
  return LLR_OK;
}

// ---- device-pointer operators -------------------------------------------------------------
int llr_signal_model_dev(llr_cf32* d_x, const int32_t* is, int32_t batch, const float* lin_ksp, const float* lin_img,
                         int32_t direction, void* stream) {
  if (!d_x || !is || batch < 1) return set_error(LLR_ERR_INVALID, "bad signal_model arguments");
  if (direction != LLR_FORWARD && direction != LLR_INVERSE) return set_error(LLR_ERR_INVALID, "bad direction");
  int dims[3] = {is[0], is[1], is[2]};
  return signal_model_dev((float2*)d_x, dims, batch, lin_ksp, lin_img, direction, (cudaStream_t)stream);
}

int llr_lift_data_set_dev(const llr_cf32* d_vol, int32_t nq, llr_cf32* d_mat, const int32_t* vs, const int32_t* bs,
                          const int32_t* sh, int64_t start, int64_t n, void* stream) {
  if (!d_vol || !d_mat || !vs || !bs || !sh || nq < 1) return set_error(LLR_ERR_INVALID, "null pointer");
  for (int a = 0; a < 3; ++a)
    if (bs[a] < 1 || bs[a] > vs[a]) return set_error(LLR_ERR_INVALID, "block dimension must be <= volume dimension");
  return launch_lift((const float2*)d_vol, (float2*)d_mat, vs, nq, bs, sh, start, n, 0, (cudaStream_t)stream);
}

int llr_un_lift_data_set_dev(llr_cf32* d_vol, int32_t nq, const llr_cf32* d_mat, const int32_t* vs,
                             const int32_t* bs, const int32_t* sh, int64_t start, int64_t n, void* stream) {
  if (!d_vol || !d_mat || !vs || !bs || !sh || nq < 1) return set_error(LLR_ERR_INVALID, "null pointer");
  for (int a = 0; a < 3; ++a)
    if (bs[a] < 1 || bs[a] > vs[a]) return set_error(LLR_ERR_INVALID, "block dimension must be <= volume dimension");
  return launch_lift((const float2*)d_vol, (float2*)d_mat, vs, nq, bs, sh, start, n, 1, (cudaStream_t)stream);
}

static int g_batch_eig_solver = 0;

static int batch_prox(int m, int n, int mode, int rank, float lam, int batch, llr_cf32* d, void* stream) {
  if (!d || m < 1 || n < 1 || batch < 0) return set_error(LLR_ERR_INVALID, "bad matrix batch arguments");
  if (batch == 0) return LLR_OK;
  cudaStream_t s = (cudaStream_t)stream;
  BlockSource src;
  memset(&src, 0, sizeof(src));
  src.kind = 0;
  src.data = (float2*)d;
  src.nblocks = batch;
  ProxOp op;
  memset(&op, 0, sizeof(op));
  op.m = m; op.n = n; op.mode = mode; op.rank = rank; op.lambda = lam; op.block_stat = nullptr;
  op.eig_solver = g_batch_eig_solver;
  int* fb = nullptr;
  float2* gram = nullptr;
  // fallback list + count, then the per-block kept counts + queue counter
  LLR_CUDA_TRY(cudaMallocAsync((void**)&fb, sizeof(int) * (2 * (size_t)batch + 2), s));
  cudaError_t e = cudaMallocAsync((void**)&gram, sizeof(float2) * (size_t)batch * (size_t)prox_gram_stride(n), s);
  if (e != cudaSuccess) {
    cudaFreeAsync(fb, s);
    return cuda_error(e, "cudaMallocAsync", __FILE__, __LINE__);
  }
  op.fb_list = fb;
  op.fb_count = fb + batch;
  op.blk_ra = fb + batch + 1;
  op.gram = gram;
  op.gram_stride = prox_gram_stride(n);
  op.gram_mode = 0;
  op.err = nullptr;
  float2* vwide = nullptr;
  if ((n > 64 && n <= kProxMaxN) || prox_needs_wide_fallback(m, n)) {   // wide Jacobi kernel scratch
    op.vwide_ctas = wide_jacobi_ctas();
    e = cudaMallocAsync((void**)&vwide, sizeof(float2) * (size_t)op.vwide_ctas * (size_t)wide_v_stride(), s);
    if (e != cudaSuccess) {
      cudaFreeAsync(fb, s);
      cudaFreeAsync(gram, s);
      return cuda_error(e, "cudaMallocAsync", __FILE__, __LINE__);
    }
    op.vwide = vwide;
  }
  int st = launch_llr_prox(src, op, s);
  if (vwide) cudaFreeAsync(vwide, s);
  e = cudaFreeAsync(fb, s);
  cudaError_t e2 = cudaFreeAsync(gram, s);
  if (st == LLR_OK && e != cudaSuccess) st = cuda_error(e, "cudaFreeAsync", __FILE__, __LINE__);
  if (st == LLR_OK && e2 != cudaSuccess) st = cuda_error(e2, "cudaFreeAsync", __FILE__, __LINE__);
  return st;
}

int llr_low_rank_batch_dev(int32_t m, int32_t n, int32_t rank, int32_t batch, llr_cf32* d, void* stream) {
  if (rank < 1 || rank > n) return set_error(LLR_ERR_INVALID, "rank must be in [1, n] (lib.rs:205-207)");
  return batch_prox(m, n, LLR_PROX_HARD_RANK, rank, 0.f, batch, d, stream);
}

int llr_soft_threshold_batch_dev(int32_t m, int32_t n, float lam, int32_t batch, llr_cf32* d, void* stream) {
  if (!(lam >= 0.f)) return set_error(LLR_ERR_INVALID, "lambda must be >= 0");
  return batch_prox(m, n, LLR_PROX_SOFT_THRESH, 0, lam, batch, d, stream);
}

int llr_subspace_low_rank_batch_dev(int32_t m, int32_t nq, int32_t srank, int32_t mode, int32_t rank, float lam,
                                    const llr_cf32* d_S, int32_t batch, llr_cf32* d, void* stream) {
  if (!d || !d_S || m < 1 || nq < 1 || srank < 1 || srank > nq) return set_error(LLR_ERR_INVALID, "bad arguments");
  if (mode == LLR_PROX_HARD_RANK && (rank < 1 || rank > srank))
    return set_error(LLR_ERR_INVALID, "rank must be in [1, srank]");
  BlockSource src;
  memset(&src, 0, sizeof(src));
  src.kind = 0;
  src.data = (float2*)d;
  src.nblocks = batch;
  SubspaceOp op;
  op.m = m; op.nq = nq; op.srank = srank; op.mode = mode; op.rank = rank; op.lambda = lam;
  op.S = (const float2*)d_S;
  return launch_llr_prox_subspace(src, op, (cudaStream_t)stream);
}

int rhsCdgmmBatched(int m, int n, int batch, llr_cf32* d_matrix, float* d_diag) {
  // kernels.cu:49-67 contract: launch, synchronise, return the cudaError_t.
  if (m < 0 || n < 0 || batch < 0 || (m * (long long)n * batch > 0 && (!d_matrix || !d_diag)))
    return (int)cudaErrorInvalidValue;
  int st = launch_rhs_cdgmm(m, n, batch, (float2*)d_matrix, d_diag, 0);
  cudaError_t e = cudaDeviceSynchronize();
  if (st != LLR_OK && e == cudaSuccess) e = cudaGetLastError();
  return (int)e;
}

int llr_cgemm_strided_batched_dev(int32_t m, int32_t k, int32_t n, int32_t batch, int32_t bcast, llr_cf32 alpha,
                                  llr_cf32 beta, int32_t ta, int32_t tb, const llr_cf32* a, const llr_cf32* b,
                                  llr_cf32* c, void* stream) {
  if (m < 0 || k < 0 || n < 0 || batch < 0 || !a || !b || !c) return set_error(LLR_ERR_INVALID, "bad cgemm arguments");
  return launch_cgemm(m, k, n, batch, bcast, make_float2(alpha.re, alpha.im), make_float2(beta.re, beta.im), ta, tb,
                      (const float2*)a, (const float2*)b, (float2*)c, (cudaStream_t)stream);
}

int llr_dwt3_axis_dev(const llr_cf32* v, llr_cf32* d, const uint32_t* vs, const uint32_t* ds, uint32_t axis,
                      uint32_t F, const float* lo, const float* hi, const int32_t* sh, void* stream) {
  if (!v || !d || !vs || !ds || !lo || !hi || axis > 2) return set_error(LLR_ERR_INVALID, "bad dwt3_axis arguments");
  float hlo[20], hhi[20];
  if (F < 2 || F > 20) return set_error(LLR_ERR_INVALID, "filter length outside [2, 20]");
  LLR_CUDA_TRY(cudaMemcpy(hlo, lo, F * sizeof(float), cudaMemcpyDeviceToHost));
  LLR_CUDA_TRY(cudaMemcpy(hhi, hi, F * sizeof(float), cudaMemcpyDeviceToHost));
  return launch_dwt_axis_ref((const float2*)v, (float2*)d, vs, ds, (int)axis, hlo, hhi, (int)F, sh, 0,
                             (cudaStream_t)stream);
}

int llr_idwt3_axis_dev(llr_cf32* v, const llr_cf32* d, const uint32_t* vs, const uint32_t* ds, uint32_t axis,
                       uint32_t F, const float* lo, const float* hi, const int32_t* sh, void* stream) {
  if (!v || !d || !vs || !ds || !lo || !hi || axis > 2) return set_error(LLR_ERR_INVALID, "bad idwt3_axis arguments");
  float hlo[20], hhi[20];
  if (F < 2 || F > 20) return set_error(LLR_ERR_INVALID, "filter length outside [2, 20]");
  LLR_CUDA_TRY(cudaMemcpy(hlo, lo, F * sizeof(float), cudaMemcpyDeviceToHost));
  LLR_CUDA_TRY(cudaMemcpy(hhi, hi, F * sizeof(float), cudaMemcpyDeviceToHost));
  return launch_dwt_axis_ref((const float2*)v, (float2*)d, vs, ds, (int)axis, hlo, hhi, (int)F, sh, 1,
                             (cudaStream_t)stream);
}

// The reference's native launchers (kernels.cu:273-348) as its Rust code binds them
// (cudwt3.rs:97-100): host size arrays, device volume / decomposition / filter / shift
// pointers, default stream, synchronise, return the cudaError_t.  The circular shift wraps
// each axis by its own extent.
static int dwt3_axis_abi(llr_cf32* vol, llr_cf32* dec, const unsigned* vs, const unsigned* ds, unsigned axis,
                         unsigned F, const float* lo, const float* hi, const int* sh, int inverse) {
  if (!vol || !dec || !vs || !ds || !lo || !hi || !sh || axis > 2 || F < 2 || F > 20)
    return (int)cudaErrorInvalidValue;
  for (int a = 0; a < 3; ++a)
    if (vs[a] == 0 || ds[a] == 0) return (int)cudaErrorInvalidValue;
  const unsigned nc = (vs[axis] + F - 1) / 2;
  if ((!inverse && ds[axis] < 2 * nc) || (inverse && ds[axis] != 2 * nc)) return (int)cudaErrorInvalidValue;
  for (int a = 0; a < 3; ++a)
    if (a != (int)axis && vs[a] != ds[a]) return (int)cudaErrorInvalidValue;
  int st = launch_dwt_axis_ref((const float2*)vol, (float2*)dec, vs, ds, (int)axis, nullptr, nullptr, (int)F, nullptr,
                               inverse, 0, lo, hi, sh);
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e == cudaSuccess && st != LLR_OK) e = cudaErrorLaunchFailure;
  return (int)e;
}

int dwt3_axis(llr_cf32* vol_data, llr_cf32* decomp, unsigned int* vol_size, unsigned int* decomp_size,
              unsigned int axis, unsigned int filter_len, float* lo_d, float* hi_d, int* rand_shift) {
  return dwt3_axis_abi(vol_data, decomp, vol_size, decomp_size, axis, filter_len, lo_d, hi_d, rand_shift, 0);
}

int idwt3_axis(llr_cf32* vol_data, llr_cf32* decomp, unsigned int* vol_size, unsigned int* decomp_size,
               unsigned int axis, unsigned int filter_len, float* lo_r, float* hi_r, int* rand_shift) {
  return dwt3_axis_abi(vol_data, decomp, vol_size, decomp_size, axis, filter_len, lo_r, hi_r, rand_shift, 1);
}

int llr_wavelet_denoise_dev(llr_cf32* d_vols, const int32_t* vs, int32_t nvol, int32_t moments, int32_t levels,
                            float alpha, void* stream) {
  if (!d_vols || !vs || nvol < 1) return set_error(LLR_ERR_INVALID, "bad wavelet arguments");
  WaveletPlan p;
  LLR_TRY(wavelet_plan_init(&p, vs[0], vs[1], vs[2], moments, levels));
  if (p.levels == 0) return set_error(LLR_ERR_UNSUPPORTED, "volume too small for one wavelet level");
  const size_t per = wavelet_workspace_elems(p, 1);
  DevBuf w;
  LLR_TRY(w.alloc(per * sizeof(float2)));
  const long long V = (long long)vs[0] * vs[1] * vs[2];
  for (int v = 0; v < nvol; ++v)
    LLR_TRY(wavelet_denoise_strided(p, (float2*)d_vols + V * v, 1, vs[0], (long long)vs[0] * vs[1], V, 1, alpha,
                                    w.as<float2>(), (cudaStream_t)stream));
  LLR_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
  return LLR_OK;
}

int llr_hard_project_dev(llr_cf32* d_x, const llr_cf32* d_y, int64_t n, double* out, void* stream) {
  if (!d_x || !d_y || n < 0) return set_error(LLR_ERR_INVALID, "bad hard_project arguments");
  cudaStream_t s = (cudaStream_t)stream;
  const int nb = 296;
  DevBuf part;
  LLR_TRY(part.alloc(sizeof(double) * (nb + 1)));
  LLR_TRY(launch_hard_project((float2*)d_x, (const float2*)d_y, n, part.as<double>(), nb, s));
  LLR_TRY(launch_finalize(part.as<double>(), nb, 1.0, nullptr, 0, nullptr, 0, part.as<double>() + nb, s));
  double h = 0;
  LLR_CUDA_TRY(cudaMemcpyAsync(&h, part.as<double>() + nb, sizeof(double), cudaMemcpyDeviceToHost, s));
  LLR_CUDA_TRY(cudaStreamSynchronize(s));
  if (out) *out = h;
  return LLR_OK;
}

// ---- host-slice entry points ---------------------------------------------------------------
int llr_cu_low_rank_approx_batch(size_t m, size_t n, size_t rank, size_t batch, llr_cf32* data) {
  if (!data) return set_error(LLR_ERR_INVALID, "null matrix data");
  if (rank < 1 || rank > n) return set_error(LLR_ERR_INVALID, "rank must be in [1, n]");
  const size_t bytes = m * n * batch * sizeof(llr_cf32);
  DevBuf d;
  LLR_TRY(d.alloc(bytes));
  LLR_CUDA_TRY(cudaMemcpy(d.p, data, bytes, cudaMemcpyHostToDevice));
  LLR_TRY(llr_low_rank_batch_dev((int)m, (int)n, (int)rank, (int)batch, d.as<llr_cf32>(), nullptr));
  LLR_CUDA_TRY(cudaMemcpy(data, d.p, bytes, cudaMemcpyDeviceToHost));
  return LLR_OK;
}

int llr_signal_model(llr_cf32* x, const size_t* is, size_t batch, const float* lk, const float* li, int32_t dir) {
  if (!x || !is || batch < 1) return set_error(LLR_ERR_INVALID, "bad signal_model arguments");
  const size_t bytes = is[0] * is[1] * is[2] * batch * sizeof(llr_cf32);
  DevBuf d;
  LLR_TRY(d.alloc(bytes));
  LLR_CUDA_TRY(cudaMemcpy(d.p, x, bytes, cudaMemcpyHostToDevice));
  int32_t dims[3] = {(int32_t)is[0], (int32_t)is[1], (int32_t)is[2]};
  LLR_TRY(llr_signal_model_dev(d.as<llr_cf32>(), dims, (int32_t)batch, lk, li, dir, nullptr));
  LLR_CUDA_TRY(cudaMemcpy(x, d.p, bytes, cudaMemcpyDeviceToHost));
  return LLR_OK;
}

static int host_lift(llr_cf32* vols, size_t nvols, llr_cf32* mats, const size_t* vs, const size_t* bs,
                     const size_t* sh, size_t start, size_t n, int dir) {
  if (!vols || !mats || !vs || !bs || !sh) return set_error(LLR_ERR_INVALID, "null pointer");
  const size_t V = vs[0] * vs[1] * vs[2];
  const size_t m = bs[0] * bs[1] * bs[2];
  DevBuf dv, dm;
  LLR_TRY(dv.alloc(V * nvols * sizeof(llr_cf32)));
  LLR_TRY(dm.alloc(m * nvols * n * sizeof(llr_cf32)));
  LLR_CUDA_TRY(cudaMemcpy(dv.p, vols, V * nvols * sizeof(llr_cf32), cudaMemcpyHostToDevice));
  if (dir == 1) LLR_CUDA_TRY(cudaMemcpy(dm.p, mats, m * nvols * n * sizeof(llr_cf32), cudaMemcpyHostToDevice));
  int32_t v3[3] = {(int32_t)vs[0], (int32_t)vs[1], (int32_t)vs[2]};
  int32_t b3[3] = {(int32_t)bs[0], (int32_t)bs[1], (int32_t)bs[2]};
  int32_t s3[3] = {(int32_t)sh[0], (int32_t)sh[1], (int32_t)sh[2]};
  if (dir == 0) {
    LLR_TRY(llr_lift_data_set_dev(dv.as<llr_cf32>(), (int32_t)nvols, dm.as<llr_cf32>(), v3, b3, s3, start, n, nullptr));
    LLR_CUDA_TRY(cudaMemcpy(mats, dm.p, m * nvols * n * sizeof(llr_cf32), cudaMemcpyDeviceToHost));
  } else {
    LLR_TRY(llr_un_lift_data_set_dev(dv.as<llr_cf32>(), (int32_t)nvols, dm.as<llr_cf32>(), v3, b3, s3, start, n,
                                     nullptr));
    LLR_CUDA_TRY(cudaMemcpy(vols, dv.p, V * nvols * sizeof(llr_cf32), cudaMemcpyDeviceToHost));
  }
  return LLR_OK;
}

int llr_lift_data_set(const llr_cf32* vols, size_t nvols, llr_cf32* mats, const size_t* vs, const size_t* bs,
                      const size_t* sh, size_t start, size_t n) {
  return host_lift(const_cast<llr_cf32*>(vols), nvols, mats, vs, bs, sh, start, n, 0);
}

int llr_un_lift_data_set(llr_cf32* vols, size_t nvols, const llr_cf32* mats, const size_t* vs, const size_t* bs,
                         const size_t* sh, size_t start, size_t n) {
  return host_lift(vols, nvols, const_cast<llr_cf32*>(mats), vs, bs, sh, start, n, 1);
}

int llr_dti_project(const llr_cf32* S, const llr_cf32* X, llr_cf32* C, size_t batch, size_t nq, size_t nvox,
                    size_t srank) {
  if (!S || !X || !C) return set_error(LLR_ERR_INVALID, "null pointer");
  DevBuf dS, dX, dC;
  LLR_TRY(dS.alloc(nq * srank * sizeof(llr_cf32)));
  LLR_TRY(dX.alloc(nq * nvox * batch * sizeof(llr_cf32)));
  LLR_TRY(dC.alloc(srank * nvox * batch * sizeof(llr_cf32)));
  LLR_CUDA_TRY(cudaMemcpy(dS.p, S, nq * srank * sizeof(llr_cf32), cudaMemcpyHostToDevice));
  LLR_CUDA_TRY(cudaMemcpy(dX.p, X, nq * nvox * batch * sizeof(llr_cf32), cudaMemcpyHostToDevice));
  llr_cf32 one = {1.f, 0.f}, zero = {0.f, 0.f};
  // S^H * X^H : (srank x nq) (nq x nvox)  (dti_subspace.rs:156-160)
  LLR_TRY(llr_cgemm_strided_batched_dev((int)srank, (int)nq, (int)nvox, (int)batch, 1, one, zero, 1, 1,
                                        dS.as<llr_cf32>(), dX.as<llr_cf32>(), dC.as<llr_cf32>(), nullptr));
  LLR_CUDA_TRY(cudaMemcpy(C, dC.p, srank * nvox * batch * sizeof(llr_cf32), cudaMemcpyDeviceToHost));
  return LLR_OK;
}

int llr_dti_back_project(const llr_cf32* S, llr_cf32* X, const llr_cf32* C, size_t batch, size_t nq, size_t nvox,
                         size_t srank) {
  if (!S || !X || !C) return set_error(LLR_ERR_INVALID, "null pointer");
  DevBuf dS, dX, dC, dT;
  LLR_TRY(dS.alloc(nq * srank * sizeof(llr_cf32)));
  LLR_TRY(dX.alloc(nq * nvox * batch * sizeof(llr_cf32)));
  LLR_TRY(dT.alloc(nq * nvox * batch * sizeof(llr_cf32)));
  LLR_TRY(dC.alloc(srank * nvox * batch * sizeof(llr_cf32)));
  LLR_CUDA_TRY(cudaMemcpy(dS.p, S, nq * srank * sizeof(llr_cf32), cudaMemcpyHostToDevice));
  LLR_CUDA_TRY(cudaMemcpy(dC.p, C, srank * nvox * batch * sizeof(llr_cf32), cudaMemcpyHostToDevice));
  llr_cf32 one = {1.f, 0.f}, zero = {0.f, 0.f};
  // T = S * L^H : (nq x srank)(srank x nvox), then X = T^H  (dti_subspace.rs:190-206)
  LLR_TRY(llr_cgemm_strided_batched_dev((int)nq, (int)srank, (int)nvox, (int)batch, 1, one, zero, 0, 0,
                                        dS.as<llr_cf32>(), dC.as<llr_cf32>(), dT.as<llr_cf32>(), nullptr));
  // conjugate transpose (nq x nvox) -> (nvox x nq) per batch (dti_subspace.rs:389)
  LLR_TRY(launch_conj_transpose(dT.as<float2>(), dX.as<float2>(), (int)nq, (int)nvox, (int)batch, 0));
  LLR_CUDA_TRY(cudaMemcpy(X, dX.p, nq * nvox * batch * sizeof(llr_cf32), cudaMemcpyDeviceToHost));
  return LLR_OK;
}

int llr_cu_dwt_denoise(llr_cf32* vol, const size_t* vs, const float* lo_d, const float* hi_d, const float* lo_r,
                       const float* hi_r, size_t F, const int32_t* sh) {
  if (!vol || !vs || !lo_d || !hi_d || !lo_r || !hi_r) return set_error(LLR_ERR_INVALID, "null pointer");
  if (F < 2 || F > 20) return set_error(LLR_ERR_INVALID, "filter length outside [2, 20]");
  const uint32_t v0[3] = {(uint32_t)vs[0], (uint32_t)vs[1], (uint32_t)vs[2]};
  uint32_t nc[3];
  for (int a = 0; a < 3; ++a) nc[a] = (uint32_t)((vs[a] + F - 1) / 2);
  const uint32_t t1[3] = {2 * nc[0], v0[1], v0[2]};
  const uint32_t t2[3] = {2 * nc[0], 2 * nc[1], v0[2]};
  const uint32_t dd[3] = {2 * nc[0], 2 * nc[1], 2 * nc[2]};
  const size_t nV = (size_t)v0[0] * v0[1] * v0[2];
  DevBuf dv, d1, d2, dd_;
  LLR_TRY(dv.alloc(nV * sizeof(llr_cf32)));
  LLR_TRY(d1.alloc((size_t)t1[0] * t1[1] * t1[2] * sizeof(llr_cf32)));
  LLR_TRY(d2.alloc((size_t)t2[0] * t2[1] * t2[2] * sizeof(llr_cf32)));
  LLR_TRY(dd_.alloc((size_t)dd[0] * dd[1] * dd[2] * sizeof(llr_cf32)));
  LLR_CUDA_TRY(cudaMemcpy(dv.p, vol, nV * sizeof(llr_cf32), cudaMemcpyHostToDevice));
  const int zero[3] = {0, 0, 0};
  const int* s3 = sh ? sh : zero;
  // cudwt3.rs:146-219: analysis x, y, z then synthesis z, y, x.
  LLR_TRY(launch_dwt_axis_ref(dv.as<float2>(), d1.as<float2>(), v0, t1, 0, lo_d, hi_d, (int)F, s3, 0, 0));
  LLR_TRY(launch_dwt_axis_ref(d1.as<float2>(), d2.as<float2>(), t1, t2, 1, lo_d, hi_d, (int)F, s3, 0, 0));
  LLR_TRY(launch_dwt_axis_ref(d2.as<float2>(), dd_.as<float2>(), t2, dd, 2, lo_d, hi_d, (int)F, s3, 0, 0));
  LLR_TRY(launch_dwt_axis_ref(d2.as<float2>(), dd_.as<float2>(), t2, dd, 2, lo_r, hi_r, (int)F, s3, 1, 0));
  LLR_TRY(launch_dwt_axis_ref(d1.as<float2>(), d2.as<float2>(), t1, t2, 1, lo_r, hi_r, (int)F, s3, 1, 0));
  LLR_TRY(launch_dwt_axis_ref(dv.as<float2>(), d1.as<float2>(), v0, t1, 0, lo_r, hi_r, (int)F, s3, 1, 0));
  LLR_CUDA_TRY(cudaMemcpy(vol, dv.p, nV * sizeof(llr_cf32), cudaMemcpyDeviceToHost));
  return LLR_OK;
}

// ---- memory helpers -------------------------------------------------------------------------
int llr_host_alloc(size_t bytes, void** out) {
  if (!out) return set_error(LLR_ERR_INVALID, "null pointer");
  LLR_CUDA_TRY(cudaHostAlloc(out, bytes ? bytes : 16, cudaHostAllocDefault));
  return LLR_OK;
}
int llr_host_free(void* p) {
  if (p) LLR_CUDA_TRY(cudaFreeHost(p));
  return LLR_OK;
}
int llr_device_alloc(size_t bytes, void** out) {
  if (!out) return set_error(LLR_ERR_INVALID, "null pointer");
  LLR_CUDA_TRY(cudaMalloc(out, bytes ? bytes : 16));
  return LLR_OK;
}
int llr_device_free(void* p) {
  if (p) LLR_CUDA_TRY(cudaFree(p));
  return LLR_OK;
}
int llr_memcpy_h2d(void* dst, const void* src, size_t bytes, void* stream) {
  LLR_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, (cudaStream_t)stream));
  return LLR_OK;
}
int llr_memcpy_d2h(void* dst, const void* src, size_t bytes, void* stream) {
  LLR_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, (cudaStream_t)stream));
  return LLR_OK;
}
int llr_stream_sync(void* stream) {
  LLR_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
  return LLR_OK;
}
int llr_device_count(int32_t* n) {
  if (!n) return set_error(LLR_ERR_INVALID, "null pointer");
  int c = 0;
  cudaError_t e = cudaGetDeviceCount(&c);
  if (e != cudaSuccess) { *n = 0; return cuda_error(e, "cudaGetDeviceCount", __FILE__, __LINE__); }
  *n = c;
  return LLR_OK;
}

}  // extern "C"
