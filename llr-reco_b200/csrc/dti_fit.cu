// DTI scalar maps downstream of the recon (diffusion_models.rs:21-129, calc_scalars):
// per voxel, s0 = mean |b0|, rhs_q = ln(clamp(|s_q| / max(s0, FLT_MIN), FLT_MIN, 1)), the
// 6-parameter tensor d = argmin ||A d - rhs|| with the design matrix of build_design_matrix
// (columns -b gx^2, -b gy^2, -b gz^2, -2b gx gy, -2b gx gz, -2b gy gz), the eigenvalues of the
// 3 x 3 tensor (e1 >= e2 >= e3), and MD = mean, RD = (e2 + e3) / 2,
// FA = sqrt(3/2) sqrt(sum (e_i - MD)^2) / sqrt(sum e_i^2) (NaN for a zero tensor, as there).
//
// One thread per voxel: the least-squares solve is the same pseudo-inverse for every voxel
// (A has full column rank for six or more non-coplanar directions), formed once on the host in
// FP64 from the normal equations and applied from shared memory; the symmetric 3 x 3 eigen
// problem is a few cyclic Jacobi sweeps in registers.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <vector>

#include "llr_common.cuh"
#include "llr_internal.h"

namespace llr {

namespace {

constexpr int kDtiOut = 7;   // b0av, e1, e2, e3, md, rd, fa

__device__ __forceinline__ void jacobi_rot(float& app, float& aqq, float& apq, float& arp, float& arq) {
  // zero apq; arp / arq: the third row's entries against p and q
  if (apq == 0.f) return;
  const float th = (aqq - app) / (2.f * apq);
  const float t = copysignf(1.f, th) / (fabsf(th) + sqrtf(th * th + 1.f));
  const float c = 1.f / sqrtf(t * t + 1.f), s = t * c;
  app -= t * apq;
  aqq += t * apq;
  apq = 0.f;
  const float rp = arp, rq = arq;
  arp = c * rp - s * rq;
  arq = s * rp + c * rq;
}

// eigenvalues of the symmetric [[a, d, e], [d, b, f], [e, f, c]], descending
__device__ void sym3_eigenvalues(float a, float b, float c, float d, float e, float f, float* out) {
  for (int sweep = 0; sweep < 8; ++sweep) {
    if (fabsf(d) + fabsf(e) + fabsf(f) <= 1e-30f + 1e-9f * (fabsf(a) + fabsf(b) + fabsf(c))) break;
    jacobi_rot(a, b, d, e, f);   // (0,1); third index 2: (a02, a12) = (e, f)
    jacobi_rot(a, c, e, d, f);   // (0,2); third index 1: (a01, a21) = (d, f)
    jacobi_rot(b, c, f, d, e);   // (1,2); third index 0: (a10, a20) = (d, e)
  }
  float l[3] = {a, b, c};
  if (l[0] < l[1]) { float t = l[0]; l[0] = l[1]; l[1] = t; }
  if (l[1] < l[2]) { float t = l[1]; l[1] = l[2]; l[2] = t; }
  if (l[0] < l[1]) { float t = l[0]; l[0] = l[1]; l[1] = t; }
  out[0] = l[0]; out[1] = l[1]; out[2] = l[2];
}

__global__ void dti_fit_kernel(const float2* __restrict__ dwi, const float2* __restrict__ b0, long long V, int nq,
                               int nb0, const float* __restrict__ pinv, float* __restrict__ out) {
  extern __shared__ float s_pinv[];   // [6][nq]
  for (int i = threadIdx.x; i < 6 * nq; i += blockDim.x) s_pinv[i] = pinv[i];
  __syncthreads();
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < V; v += (long long)gridDim.x * blockDim.x) {
    float s0 = 0.f;
    for (int k = 0; k < nb0; ++k) {
      const float2 z = b0[v + V * k];
      s0 += sqrtf(z.x * z.x + z.y * z.y);
    }
    s0 = nb0 > 0 ? s0 / (float)nb0 : 0.f;
    const float s0c = fmaxf(s0, FLT_MIN);
    float dt[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    for (int q = 0; q < nq; ++q) {
      const float2 z = dwi[v + V * q];
      const float r = logf(fminf(fmaxf(sqrtf(z.x * z.x + z.y * z.y) / s0c, FLT_MIN), 1.f));
#pragma unroll
      for (int j = 0; j < 6; ++j) dt[j] = fmaf(s_pinv[j * nq + q], r, dt[j]);
    }
    float l[3];
    sym3_eigenvalues(dt[0], dt[1], dt[2], dt[3], dt[4], dt[5], l);
    const float md = (l[0] + l[1] + l[2]) / 3.f;
    const float rd = 0.5f * (l[1] + l[2]);
    const float num = sqrtf((l[0] - md) * (l[0] - md) + (l[1] - md) * (l[1] - md) + (l[2] - md) * (l[2] - md));
    const float den = sqrtf(l[0] * l[0] + l[1] * l[1] + l[2] * l[2]);
    const float fa = 1.22474487139158904910f * num / den;
    out[v] = s0;
    out[V + v] = l[0];
    out[2 * V + v] = l[1];
    out[3 * V + v] = l[2];
    out[4 * V + v] = md;
    out[5 * V + v] = rd;
    out[6 * V + v] = fa;
  }
}

// (A^T A)^{-1} A^T in FP64 (Gauss-Jordan with partial pivoting on the 6 x 6 normal matrix)
int design_pinv(const float* b, const float* g, int nq, std::vector<float>& pinv) {
  std::vector<double> A((size_t)nq * 6);
  for (int q = 0; q < nq; ++q) {
    const double bb = b[q], gx = g[3 * q], gy = g[3 * q + 1], gz = g[3 * q + 2];
    const double row[6] = {-bb * gx * gx, -bb * gy * gy, -bb * gz * gz, -2 * bb * gx * gy, -2 * bb * gx * gz,
                           -2 * bb * gy * gz};
    for (int j = 0; j < 6; ++j) A[(size_t)q * 6 + j] = row[j];
  }
  double M[6][12];
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) {
      double s = 0.0;
      for (int q = 0; q < nq; ++q) s += A[(size_t)q * 6 + i] * A[(size_t)q * 6 + j];
      M[i][j] = s;
      M[i][6 + j] = i == j ? 1.0 : 0.0;
    }
  double scale = 0.0;
  for (int i = 0; i < 6; ++i) scale = std::max(scale, std::fabs(M[i][i]));
  for (int c = 0; c < 6; ++c) {
    int p = c;
    for (int r = c + 1; r < 6; ++r)
      if (std::fabs(M[r][c]) > std::fabs(M[p][c])) p = r;
    if (!(std::fabs(M[p][c]) > 1e-12 * scale))
      return set_error(LLR_ERR_INVALID, "DTI design matrix is rank deficient (need 6 independent directions)");
    if (p != c)
      for (int j = 0; j < 12; ++j) std::swap(M[p][j], M[c][j]);
    const double inv = 1.0 / M[c][c];
    for (int j = 0; j < 12; ++j) M[c][j] *= inv;
    for (int r = 0; r < 6; ++r)
      if (r != c) {
        const double f = M[r][c];
        for (int j = 0; j < 12; ++j) M[r][j] -= f * M[c][j];
      }
  }
  pinv.assign((size_t)6 * nq, 0.f);
  for (int j = 0; j < 6; ++j)
    for (int q = 0; q < nq; ++q) {
      double s = 0.0;
      for (int i = 0; i < 6; ++i) s += M[j][6 + i] * A[(size_t)q * 6 + i];
      pinv[(size_t)j * nq + q] = (float)s;
    }
  return LLR_OK;
}

}  // namespace

}  // namespace llr

using namespace llr;

extern "C" {

int llr_dti_fit_dev(const llr_cf32* d_dwi, int32_t nq, const llr_cf32* d_b0, int32_t nb0, int64_t n_vox,
                    const float* b_vals, const float* b_vecs, float* d_out, void* stream) {
  if (!d_dwi || !b_vals || !b_vecs || !d_out || nq < 6 || nb0 < 0 || (nb0 > 0 && !d_b0) || n_vox < 0)
    return set_error(LLR_ERR_INVALID, "bad DTI fit arguments (need >= 6 diffusion volumes)");
  if (n_vox == 0) return LLR_OK;
  std::vector<float> pinv;
  LLR_TRY(design_pinv(b_vals, b_vecs, nq, pinv));
  cudaStream_t s = (cudaStream_t)stream;
  float* d_pinv = nullptr;
  LLR_CUDA_TRY(cudaMallocAsync((void**)&d_pinv, sizeof(float) * pinv.size(), s));
  cudaError_t e = cudaMemcpyAsync(d_pinv, pinv.data(), sizeof(float) * pinv.size(), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) {
    const long long blocks = std::min<long long>((n_vox + 255) / 256, 148LL * 32);
    note_launch();
    dti_fit_kernel<<<(unsigned)blocks, 256, sizeof(float) * 6 * nq, s>>>(
        (const float2*)d_dwi, (const float2*)d_b0, n_vox, nq, nb0, d_pinv, d_out);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);   // the host pinv copy must outlive the transfer
  cudaFreeAsync(d_pinv, s);
  if (e != cudaSuccess) return cuda_error(e, "dti_fit_kernel", __FILE__, __LINE__);
  return LLR_OK;
}

int llr_dti_fit(const llr_cf32* dwi, int32_t nq, const llr_cf32* b0, int32_t nb0, int64_t n_vox, const float* b_vals,
                const float* b_vecs, float* out) {
  if (!dwi || !out || (nb0 > 0 && !b0) || n_vox < 0) return set_error(LLR_ERR_INVALID, "null pointer");
  float2 *d_dwi = nullptr, *d_b0 = nullptr;
  float* d_out = nullptr;
  int st = LLR_OK;
  auto fail = [&](int code) {
    cudaFree(d_dwi);
    cudaFree(d_b0);
    cudaFree(d_out);
    return code;
  };
  cudaError_t e = cudaMalloc((void**)&d_dwi, sizeof(float2) * (size_t)n_vox * nq);
  if (e == cudaSuccess && nb0 > 0) e = cudaMalloc((void**)&d_b0, sizeof(float2) * (size_t)n_vox * nb0);
  if (e == cudaSuccess) e = cudaMalloc((void**)&d_out, sizeof(float) * (size_t)n_vox * kDtiOut);
  if (e == cudaSuccess) e = cudaMemcpy(d_dwi, dwi, sizeof(float2) * (size_t)n_vox * nq, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && nb0 > 0)
    e = cudaMemcpy(d_b0, b0, sizeof(float2) * (size_t)n_vox * nb0, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return fail(cuda_error(e, "DTI fit buffers", __FILE__, __LINE__));
  st = llr_dti_fit_dev((const llr_cf32*)d_dwi, nq, (const llr_cf32*)d_b0, nb0, n_vox, b_vals, b_vecs, d_out, nullptr);
  if (st != LLR_OK) return fail(st);
  e = cudaMemcpy(out, d_out, sizeof(float) * (size_t)n_vox * kDtiOut, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return fail(cuda_error(e, "cudaMemcpy", __FILE__, __LINE__));
  return fail(LLR_OK);
}

}  // extern "C"
