// Signal operator A / A^H (signal_model.rs:34-117, cufft.rs:124-337) and hard data
// consistency (lib.rs:392-406) on the device.
//
// Within the iteration the phase ramps and unitary scalings never get a pass of their
// own: the k-space DC pass works on raw cuFFT output against precomputed
// sqrt(N) e^{+i theta_img} y, and the image-domain ramp plus 1/N are applied inside the
// LLR gather/scatter.  For line-structured sampling (whole x-lines, as produced by
// under_sample_kspace, data_import.rs:416-438) the x-axis transform cancels exactly
// (A^H (1-M) A = I_x (x) A_yz^H (1-M) A_yz, A_x unitary), so only 2-D FFTs over (y, z) run
// and DC touches only sampled lines.
#include <cstdio>
#include <cstring>
#include <cmath>
#include <algorithm>
#include <map>
#include <tuple>

#include "llr_internal.h"

namespace llr {

// ---------------------------------------------------------------------------------------
// cuFFT plan cache for stand-alone calls
// ---------------------------------------------------------------------------------------
int cufft_error(cufftResult r, const char* what) {
  return set_error(LLR_ERR_CUFFT, "%s failed: cufftResult %d", what, (int)r);
}

namespace {
std::mutex g_plan_mu;
std::map<std::tuple<int, int, long long, long long, long long, long long>, cufftHandle> g_plans;
}  // namespace

int get_c2c_plan(int rank, const long long* n, long long batch, cufftHandle* out) {
  int dev = 0;
  LLR_CUDA_TRY(cudaGetDevice(&dev));
  auto key = std::make_tuple(dev, rank, n[0], rank > 1 ? n[1] : 0LL, rank > 2 ? n[2] : 0LL, batch);
  std::lock_guard<std::mutex> lk(g_plan_mu);
  auto it = g_plans.find(key);
  if (it != g_plans.end()) { *out = it->second; return LLR_OK; }
  cufftHandle h;
  cufftResult r = cufftCreate(&h);
  if (r != CUFFT_SUCCESS) return cufft_error(r, "cufftCreate");
  long long nn[3] = {n[0], rank > 1 ? n[1] : 1, rank > 2 ? n[2] : 1};
  long long dist = 1;
  for (int a = 0; a < rank; ++a) dist *= nn[a];
  size_t ws = 0;
  r = cufftMakePlanMany64(h, rank, nn, nullptr, 1, dist, nullptr, 1, dist, CUFFT_C2C, batch, &ws);
  if (r != CUFFT_SUCCESS) { cufftDestroy(h); return cufft_error(r, "cufftMakePlanMany64"); }
  g_plans[key] = h;
  *out = h;
  return LLR_OK;
}

// ---------------------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------------------
namespace {

__device__ __forceinline__ float2 apply_phase(float2 v, float2 p, int sign) {
  if (sign > 0) return cmul(v, p);
  if (sign < 0) return cmul_bc(v, p);
  return v;
}

// (nyz x nx) row-major per volume  <->  (nx x nyz) row-major per volume.
__global__ void transpose_kernel(const float2* __restrict__ in, float2* __restrict__ out, Geom g, int to_planar,
                                 float scale, PhaseTab ph, int sign) {
  __shared__ float2 tile[32][33];
  const int q = blockIdx.z;
  const long long base = (long long)q * g.V;
  // to_planar: input rows j (nyz) x cols ix (nx); output rows ix x cols j.
  const long long rows_in = to_planar ? g.nyz : g.nx;
  const long long cols_in = to_planar ? g.nx : g.nyz;
  const long long c0 = (long long)blockIdx.x * 32, r0 = (long long)blockIdx.y * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const long long r = r0 + k, c = c0 + threadIdx.x;
    if (r < rows_in && c < cols_in) tile[k][threadIdx.x] = in[base + r * cols_in + c];
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const long long orow = c0 + k, ocol = r0 + threadIdx.x;  // output row = input col
    if (orow < cols_in && ocol < rows_in) {
      float2 v = tile[threadIdx.x][k];
      long long ix, j;
      if (to_planar) { ix = orow; j = ocol; } else { ix = ocol; j = orow; }
      if (sign != 0 || scale != 1.f) {
        const int iy = (int)(j % g.ny), iz = (int)(j / g.ny);
        if (sign != 0) v = apply_phase(v, phase_at(ph, g, q, (int)ix, iy, iz), sign);
        v = cscale(v, scale);
      }
      out[base + orow * rows_in + ocol] = v;
    }
  }
}

// x *= scale * exp(sign * i * (theta_x + theta_y + theta_z)) on a reference-layout batch.
__global__ void phase_ref_kernel(float2* x, Geom g, int nvol, const float2* tx, const float2* ty, const float2* tz,
                                 int sign, float scale) {
  const long long tot = g.V * nvol;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < tot; i += (long long)gridDim.x * blockDim.x) {
    const int q = (int)(i / g.V);
    long long r = i - (long long)q * g.V;
    const int ix = (int)(r % g.nx);
    r /= g.nx;
    const int iy = (int)(r % g.ny);
    const int iz = (int)(r / g.ny);
    float2 p = cmul(cmul(tx[(long long)q * g.nx + ix], ty[(long long)q * g.ny + iy]), tz[(long long)q * g.nz + iz]);
    float2 v = x[i];
    v = (sign > 0) ? cmul(v, p) : cmul_bc(v, p);
    x[i] = cscale(v, scale);
  }
}

// phase along x only (reference layout), used by the hybrid set-up.
__global__ void phase_x_kernel(float2* x, Geom g, int nvol, const float2* tx, int sign, float scale) {
  const long long tot = g.V * nvol;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < tot; i += (long long)gridDim.x * blockDim.x) {
    const int q = (int)(i / g.V);
    const int ix = (int)((i - (long long)q * g.V) % g.nx);
    float2 v = apply_phase(x[i], tx[(long long)q * g.nx + ix], sign);
    x[i] = cscale(v, scale);
  }
}

template <int BS>
__device__ double block_reduce_d(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < BS / 32; ++i) s += sh[i];
  return s;
}

// Hybrid-space DC over sampled lines only.  u: planar raw 2-D spectra; yhat: per volume q a
// block of nx x L_q values (x-major) = sqrt(N_yz) e^{+i theta_img,yz} A_x^H y.
__global__ void __launch_bounds__(256) dc_hybrid_kernel(float2* __restrict__ u, const float2* __restrict__ yhat,
                                                        const int* __restrict__ pos, const long long* __restrict__ off,
                                                        Geom g, double* partials, int replace_only) {
  __shared__ double sh[8];
  const int q = blockIdx.y;
  const long long o0 = off[q], L = off[q + 1] - o0;
  const long long tot = L * g.nx;
  const float2* yq = yhat + o0 * g.nx;
  const int* pq = pos + o0;
  double err = 0.0;
  for (long long t = blockIdx.x * 256LL + threadIdx.x; t < tot; t += (long long)gridDim.x * 256) {
    const long long ix = t / L, s = t - ix * L;
    const long long a = (long long)pq[s] + g.nyz * (ix + (long long)g.nx * q);
    const float2 yv = yq[t];
    if (!replace_only) {
      const float2 uv = u[a];
      const double dx = (double)uv.x - (double)yv.x, dy = (double)uv.y - (double)yv.y;
      err += dx * dx + dy * dy;
    }
    u[a] = yv;
  }
  const double s = block_reduce_d<256>(err, sh);
  if (threadIdx.x == 0 && partials) partials[(long long)blockIdx.y * gridDim.x + blockIdx.x] = s;
}

// Element-wise DC (general sampling pattern): where yhat != 0, err += |u - yhat|^2, u = yhat.
__global__ void __launch_bounds__(256) dc_full_kernel(float2* __restrict__ u, const float2* __restrict__ yhat,
                                                      long long n, double* partials, int replace_only) {
  __shared__ double sh[8];
  double err = 0.0;
  for (long long i = blockIdx.x * 256LL + threadIdx.x; i < n; i += (long long)gridDim.x * 256) {
    const float2 yv = yhat[i];
    if (yv.x != 0.f || yv.y != 0.f) {
      if (!replace_only) {
        const float2 uv = u[i];
        const double dx = (double)uv.x - (double)yv.x, dy = (double)uv.y - (double)yv.y;
        err += dx * dx + dy * dy;
      }
      u[i] = yv;
    } else if (replace_only) {
      u[i] = make_float2(0.f, 0.f);
    }
  }
  const double s = block_reduce_d<256>(err, sh);
  if (threadIdx.x == 0 && partials) partials[blockIdx.x] = s;
}

// Reference hard_project on reference-layout buffers (lib.rs:392-406).
__global__ void __launch_bounds__(256) hard_project_kernel(float2* __restrict__ x, const float2* __restrict__ y,
                                                           long long n, double* partials) {
  __shared__ double sh[8];
  double err = 0.0;
  for (long long i = blockIdx.x * 256LL + threadIdx.x; i < n; i += (long long)gridDim.x * 256) {
    const float2 yv = y[i];
    if (yv.x != 0.f || yv.y != 0.f) {
      const float2 xv = x[i];
      const float dx = xv.x - yv.x, dy = xv.y - yv.y;
      err += (double)(dx * dx + dy * dy);
      x[i] = yv;
    }
  }
  const double s = block_reduce_d<256>(err, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

// Deterministic final reduction: hist[*it] = scale * sum(partials); optionally ++*it.
__global__ void __launch_bounds__(256) finalize_kernel(const double* partials, int np, double scale, double* hist,
                                                       long long cap, long long* it, int advance, double* out) {
  __shared__ double sh[8];
  double v = 0.0;
  for (int i = threadIdx.x; i < np; i += 256) v += partials[i];
  const double s = block_reduce_d<256>(v, sh) * scale;
  if (threadIdx.x == 0) {
    if (out) *out = s;
    if (it) {
      const long long k = *it;
      if (hist && k >= 0 && k < cap) hist[k] = s;
      if (advance) *it = k + 1;
    }
  }
}

// Objective of the iterate the prox just produced: 0.5 ||M A x - y||^2 (the residual the
// finalize kernel stored for iteration k = *it - 1) plus lambda times the blocks' nuclear norms,
// summed in FP64 in a fixed order.  blk_nuc null: the data term alone.
__global__ void __launch_bounds__(256) objective_kernel(const double* blk_nuc, long long nb, double lam,
                                                        const double* hist, double* obj, long long cap,
                                                        const long long* it) {
  __shared__ double sh[8];
  double v = 0.0;
  if (blk_nuc)
    for (long long i = threadIdx.x; i < nb; i += 256) v += blk_nuc[i];
  const double nuc = block_reduce_d<256>(v, sh);
  if (threadIdx.x == 0) {
    const long long k = *it - 1;
    if (k >= 0 && k < cap) obj[k] = 0.5 * hist[k] + (blk_nuc ? lam * nuc : 0.0);
  }
}

// sum |a - b|^2 and sum |b|^2 in FP64, one pair of partials per block
__global__ void __launch_bounds__(256) diff_norm_kernel(const float2* __restrict__ a, const float2* __restrict__ b,
                                                        long long n, double* part_d, double* part_b) {
  __shared__ double sh[8];
  double d = 0.0, r = 0.0;
  for (long long i = blockIdx.x * 256LL + threadIdx.x; i < n; i += (long long)gridDim.x * 256) {
    const float2 u = a[i], v = b[i];
    const double dx = (double)u.x - v.x, dy = (double)u.y - v.y;
    d += dx * dx + dy * dy;
    r += (double)v.x * v.x + (double)v.y * v.y;
  }
  double s = block_reduce_d<256>(d, sh);
  __syncthreads();
  double t = block_reduce_d<256>(r, sh);
  if (threadIdx.x == 0) { part_d[blockIdx.x] = s; part_b[blockIdx.x] = t; }
}

// Per-line non-zero count along x (reference layout): one warp per (ky, kz, q) line.
__global__ void line_nnz_kernel(const float2* __restrict__ y, long long nlines, int nx, int* cnt) {
  const long long warp = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= nlines) return;
  const float2* l = y + warp * nx;
  int c = 0;
  for (int i = lane; i < nx; i += 32) c += (l[i].x != 0.f || l[i].y != 0.f);
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if (lane == 0) cnt[warp] = c;
}

// sum |y|^2 and nnz (lib.rs:409-417).
__global__ void __launch_bounds__(256) energy_kernel(const float2* __restrict__ y, long long n, double* part_e,
                                                     double* part_n) {
  __shared__ double sh[8];
  double e = 0.0, c = 0.0;
  for (long long i = blockIdx.x * 256LL + threadIdx.x; i < n; i += (long long)gridDim.x * 256) {
    const float2 v = y[i];
    e += (double)(v.x * v.x + v.y * v.y);
    c += (v.x != 0.f || v.y != 0.f) ? 1.0 : 0.0;
  }
  double s = block_reduce_d<256>(e, sh);
  __syncthreads();
  double t = block_reduce_d<256>(c, sh);
  if (threadIdx.x == 0) { part_e[blockIdx.x] = s; part_n[blockIdx.x] = t; }
}

// Gather sampled lines of planar hybrid-space data into the compact yhat layout, applying
// sqrt(N_yz) e^{+i theta_img,yz}.
__global__ void gather_lines_kernel(const float2* __restrict__ yh, float2* __restrict__ yhat,
                                    const int* __restrict__ pos, const long long* __restrict__ off, Geom g,
                                    PhaseTab ph_img, float scale) {
  const int q = blockIdx.y;
  const long long o0 = off[q], L = off[q + 1] - o0;
  const long long tot = L * g.nx;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot; t += (long long)gridDim.x * blockDim.x) {
    const long long ix = t / L, s = t - ix * L;
    const int p = pos[o0 + s];
    const int ky = p % g.ny, kz = p / g.ny;
    const float2 v = yh[(long long)p + g.nyz * (ix + (long long)g.nx * q)];
    float2 w = cmul(v, phase_at(ph_img, g, q, 0, ky, kz));
    yhat[o0 * g.nx + t] = cscale(w, scale);
  }
}

// Element-wise yhat = scale * e^{+i theta_img} y on planar data (general path).
__global__ void prep_full_kernel(float2* y, Geom g, PhaseTab ph_img, float scale) {
  const long long tot = g.V * g.nq;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < tot; i += (long long)gridDim.x * blockDim.x) {
    const int q = (int)(i / g.V);
    long long r = i - (long long)q * g.V;
    const int iy = (int)(r % g.ny);
    r /= g.ny;
    const int iz = (int)(r % g.nz);
    const int ix = (int)(r / g.nz);
    const float2 v = y[i];
    if (v.x != 0.f || v.y != 0.f) y[i] = cscale(cmul(v, phase_at(ph_img, g, q, ix, iy, iz)), scale);
  }
}

// Voxels outside the shifted block grid: value = raw * scale (* conj(phase) if requested).
__global__ void uncovered_kernel(float2* data, Geom g, int cx, int cy, int cz, const long long* it_ptr,
                                 unsigned long long seed, int s0, int s1, int s2, int m0, int m1, int m2, float scale,
                                 PhaseTab ph, int conj_phase) {
  int sh0 = s0, sh1 = s1, sh2 = s2;
  if (it_ptr) {
    const long long it = *it_ptr;
    sh0 = llr_shift_draw(seed, it, 0, m0);
    sh1 = llr_shift_draw(seed, it, 1, m1);
    sh2 = llr_shift_draw(seed, it, 2, m2);
  }
  const long long tot = g.V * g.nq;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < tot; i += (long long)gridDim.x * blockDim.x) {
    const int q = (int)(i / g.V);
    long long r = i - (long long)q * g.V;
    const int iy = (int)(r % g.ny);
    r /= g.ny;
    const int iz = (int)(r % g.nz);
    const int ix = (int)(r / g.nz);
    int ox = ix - sh0; ox += (ox < 0) ? g.nx : 0;
    int oy = iy - sh1; oy += (oy < 0) ? g.ny : 0;
    int oz = iz - sh2; oz += (oz < 0) ? g.nz : 0;
    if (ox >= cx || oy >= cy || oz >= cz) {
      float2 v = cscale(data[i], scale);
      if (conj_phase) v = cmul_bc(v, phase_at(ph, g, q, ix, iy, iz));
      data[i] = v;
    }
  }
}

// y = scale * x (in place, or copy); used for planar scaling passes.
__global__ void scale_kernel(float2* x, long long n, float s) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    x[i] = cscale(x[i], s);
}

inline unsigned grid_for(long long n, int bs = 256, long long cap = 148LL * 32) {
  long long b = (n + bs - 1) / bs;
  if (b < 1) b = 1;
  return (unsigned)std::min(b, cap);
}

}  // namespace

// ---------------------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------------------
int launch_ref_to_planar(const float2* ref, float2* planar, const Geom& g, float scale, PhaseTab ph, int phase_sign,
                         cudaStream_t s) {
  dim3 grid((unsigned)((g.nx + 31) / 32), (unsigned)((g.nyz + 31) / 32), (unsigned)g.nq);
  note_launch();
  transpose_kernel<<<grid, dim3(32, 8), 0, s>>>(ref, planar, g, 1, scale, ph, phase_sign);
  LLR_CUDA_TRY(cudaGetLastError());
  return LLR_OK;
}

int launch_planar_to_ref(const float2* planar, float2* ref, const Geom& g, float scale, PhaseTab ph, int phase_sign,
                         cudaStream_t s) {
  dim3 grid((unsigned)((g.nyz + 31) / 32), (unsigned)((g.nx + 31) / 32), (unsigned)g.nq);
  note_launch();
  transpose_kernel<<<grid, dim3(32, 8), 0, s>>>(planar, ref, g, 0, scale, ph, phase_sign);
  LLR_CUDA_TRY(cudaGetLastError());
  return LLR_OK;
}

int launch_scale_uncovered(float2* data, const Geom& g, const int* cover, const long long* it_ptr,
                           unsigned long long seed, const int shift[3], const int maxs[3], float scale, PhaseTab ph,
                           int conj_phase, cudaStream_t s) {
  note_launch();
  uncovered_kernel<<<grid_for(g.V * g.nq), 256, 0, s>>>(data, g, cover[0], cover[1], cover[2], it_ptr, seed,
                                                        shift ? shift[0] : 0, shift ? shift[1] : 0,
                                                        shift ? shift[2] : 0, maxs[0], maxs[1], maxs[2], scale, ph,
                                                        conj_phase);
  LLR_CUDA_TRY(cudaGetLastError());
  return LLR_OK;
}

int launch_dc_hybrid(float2* u, const float2* yhat, const int* pos, const long long* off, const Geom& g, int max_lines,
                     double* partials, int n_part_x, int replace_only, cudaStream_t s) {
  dim3 grid((unsigned)n_part_x, (unsigned)g.nq);
  (void)max_lines;
  note_launch();
  dc_hybrid_kernel<<<grid, 256, 0, s>>>(u, yhat, pos, off, g, partials, replace_only);
  LLR_CUDA_TRY(cudaGetLastError());
  return LLR_OK;
}

int launch_dc_full(float2* u, const float2* yhat, long long n, double* partials, int nblocks, int replace_only,
                   cudaStream_t s) {
  note_launch();
  dc_full_kernel<<<nblocks, 256, 0, s>>>(u, yhat, n, partials, replace_only);
  LLR_CUDA_TRY(cudaGetLastError());
  return LLR_OK;
}

int launch_finalize(const double* partials, int np, double scale, double* hist, long long cap, long long* it,
                    int advance, double* out, cudaStream_t s) {
  note_launch();
  finalize_kernel<<<1, 256, 0, s>>>(partials, np, scale, hist, cap, it, advance, out);
  LLR_CUDA_TRY(cudaGetLastError());
  return LLR_OK;
}

int launch_objective(const double* blk_nuc, long long nb, double lam, const double* hist, double* obj, long long cap,
                     const long long* it, cudaStream_t s) {
  note_launch();
  objective_kernel<<<1, 256, 0, s>>>(blk_nuc, nb, lam, hist, obj, cap, it);
  LLR_CUDA_TRY(cudaGetLastError());
  return LLR_OK;
}

int launch_line_nnz(const float2* y, long long nlines, int nx, int* cnt, cudaStream_t s) {
  long long threads = nlines * 32;
  note_launch();
  line_nnz_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(y, nlines, nx, cnt);
  LLR_CUDA_TRY(cudaGetLastError());
  return LLR_OK;
}

int launch_diff_norm(const float2* a, const float2* b, long long n, double* part_d, double* part_b, int nblocks,
                     cudaStream_t s) {
  note_launch();
  diff_norm_kernel<<<nblocks, 256, 0, s>>>(a, b, n, part_d, part_b);
  LLR_CUDA_TRY(cudaGetLastError());
  return LLR_OK;
}

int launch_energy(const float2* y, long long n, double* part_e, double* part_n, int nblocks, cudaStream_t s) {
  note_launch();
  energy_kernel<<<nblocks, 256, 0, s>>>(y, n, part_e, part_n);
  LLR_CUDA_TRY(cudaGetLastError());
  return LLR_OK;
}

int launch_gather_lines(const float2* yh, float2* yhat, const int* pos, const long long* off, const Geom& g,
                        PhaseTab ph_img, float scale, cudaStream_t s) {
  dim3 grid(256, (unsigned)g.nq);
  note_launch();
  gather_lines_kernel<<<grid, 256, 0, s>>>(yh, yhat, pos, off, g, ph_img, scale);
  LLR_CUDA_TRY(cudaGetLastError());
  return LLR_OK;
}

int launch_prep_full(float2* y, const Geom& g, PhaseTab ph_img, float scale, cudaStream_t s) {
  note_launch();
  prep_full_kernel<<<grid_for(g.V * g.nq), 256, 0, s>>>(y, g, ph_img, scale);
  LLR_CUDA_TRY(cudaGetLastError());
  return LLR_OK;
}

int launch_phase_ref(float2* x, const Geom& g, int nvol, const float2* tx, const float2* ty, const float2* tz, int sign,
                     float scale, cudaStream_t s) {
  note_launch();
  phase_ref_kernel<<<grid_for(g.V * nvol), 256, 0, s>>>(x, g, nvol, tx, ty, tz, sign, scale);
  LLR_CUDA_TRY(cudaGetLastError());
  return LLR_OK;
}

int launch_phase_x(float2* x, const Geom& g, int nvol, const float2* tx, int sign, float scale, cudaStream_t s) {
  note_launch();
  phase_x_kernel<<<grid_for(g.V * nvol), 256, 0, s>>>(x, g, nvol, tx, sign, scale);
  LLR_CUDA_TRY(cudaGetLastError());
  return LLR_OK;
}

int launch_scale(float2* x, long long n, float sc, cudaStream_t s) {
  note_launch();
  scale_kernel<<<grid_for(n), 256, 0, s>>>(x, n, sc);
  LLR_CUDA_TRY(cudaGetLastError());
  return LLR_OK;
}

int launch_hard_project(float2* x, const float2* y, long long n, double* partials, int nblocks, cudaStream_t s) {
  note_launch();
  hard_project_kernel<<<nblocks, 256, 0, s>>>(x, y, n, partials);
  LLR_CUDA_TRY(cudaGetLastError());
  return LLR_OK;
}

// ---------------------------------------------------------------------------------------
// phase tables (host, FP64): t[q*n + i] = exp(+i 2 pi s (i - n/2) / n), s = corr + n/2
// (cufft.rs:320-326, signal_model.rs:110-117).
// ---------------------------------------------------------------------------------------
void phase_table_host(int n, double corr, float2* out) {
  const double s = corr + 0.5 * n;
  for (int i = 0; i < n; ++i) {
    double turns = s * ((double)i - 0.5 * n) / (double)n;
    turns -= std::floor(turns);
    const double th = 2.0 * M_PI * turns;
    out[i] = make_float2((float)std::cos(th), (float)std::sin(th));
  }
}

// Tables for nvol volumes: layout [x: nvol*nx][y: nvol*ny][z: nvol*nz].
void phase_tables_host(const int dims[3], int nvol, const float* corr /* nvol x 3 or null */, float2* out) {
  float2* tx = out;
  float2* ty = tx + (size_t)nvol * dims[0];
  float2* tz = ty + (size_t)nvol * dims[1];
  for (int q = 0; q < nvol; ++q) {
    phase_table_host(dims[0], corr ? corr[3 * q + 0] : 0.0, tx + (size_t)q * dims[0]);
    phase_table_host(dims[1], corr ? corr[3 * q + 1] : 0.0, ty + (size_t)q * dims[1]);
    phase_table_host(dims[2], corr ? corr[3 * q + 2] : 0.0, tz + (size_t)q * dims[2]);
  }
}

// ---------------------------------------------------------------------------------------
// stand-alone signal model on a reference-layout device batch (signal_model.rs:34-79)
// ---------------------------------------------------------------------------------------
int signal_model_dev(float2* d_x, const int dims[3], int batch, const float* lin_ksp, const float* lin_img,
                     int direction, cudaStream_t s) {
  Geom g;
  g.nx = dims[0]; g.ny = dims[1]; g.nz = dims[2]; g.nq = batch;
  g.nyz = (long long)g.ny * g.nz;
  g.V = (long long)g.nx * g.nyz;
  const size_t nt = (size_t)batch * (dims[0] + dims[1] + dims[2]);
  std::vector<float2> h(2 * nt);
  phase_tables_host(dims, batch, lin_ksp, h.data());
  phase_tables_host(dims, batch, lin_img, h.data() + nt);
  float2* d_t = nullptr;
  LLR_CUDA_TRY(cudaMallocAsync((void**)&d_t, sizeof(float2) * 2 * nt, s));
  int st = LLR_OK;
  do {
    cudaError_t e = cudaMemcpyAsync(d_t, h.data(), sizeof(float2) * 2 * nt, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) { st = cuda_error(e, "cudaMemcpyAsync", __FILE__, __LINE__); break; }
    const float2* ksp_x = d_t;
    const float2* ksp_y = ksp_x + (size_t)batch * dims[0];
    const float2* ksp_z = ksp_y + (size_t)batch * dims[1];
    const float2* img_x = d_t + nt;
    const float2* img_y = img_x + (size_t)batch * dims[0];
    const float2* img_z = img_y + (size_t)batch * dims[1];
    const bool fwd = direction == LLR_FORWARD;
    // pre: Forward uses the k-space correction, Inverse the image correction; sign +1
    st = launch_phase_ref(d_x, g, batch, fwd ? ksp_x : img_x, fwd ? ksp_y : img_y, fwd ? ksp_z : img_z, +1, 1.f, s);
    if (st) break;
    cufftHandle plan;
    long long n[3] = {dims[2], dims[1], dims[0]};  // reversed: x fastest (cufft.rs:86)
    st = get_c2c_plan(3, n, batch, &plan);
    if (st) break;
    cufftResult r = cufftSetStream(plan, s);
    if (r != CUFFT_SUCCESS) { st = cufft_error(r, "cufftSetStream"); break; }
    r = cufftExecC2C(plan, (cufftComplex*)d_x, (cufftComplex*)d_x, fwd ? CUFFT_FORWARD : CUFFT_INVERSE);
    if (r != CUFFT_SUCCESS) { st = cufft_error(r, "cufftExecC2C"); break; }
    // post: sign -1 with the other correction, and the unitary 1/sqrt(N) (cufft.rs:161-163)
    const float sc = (float)(1.0 / std::sqrt((double)g.V));
    st = launch_phase_ref(d_x, g, batch, fwd ? img_x : ksp_x, fwd ? img_y : ksp_y, fwd ? img_z : ksp_z, -1, sc, s);
  } while (0);
  cudaError_t e = cudaFreeAsync(d_t, s);
  if (st == LLR_OK && e != cudaSuccess) st = cuda_error(e, "cudaFreeAsync", __FILE__, __LINE__);
  return st;
}

}  // namespace llr
