// Temporal subspace for the DTI subspace constraint, built on the GPU: simulated tensor
// signals (S0 = 1, eigenvalues uniform in [lam_lo, lam_hi], principal direction uniform on the
// sphere, frame from eigenvector_matrix / sample_unit_sphere, dti_subspace.rs:13-76), their
// q x q Gram matrix accumulated in FP64, and its leading eigenvectors (the left singular
// vectors of the q x N signal matrix) from a cyclic Jacobi solve in FP64.  The reference only
// loads a precomputed subspace (lib.rs:212-222).
//
// Draws are counter-based (SplitMix64 keyed by seed, stream, 5 i + k), so the oracle restates the
// same signals; per-CTA partial Gram matrices are added in a fixed order (deterministic).
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <vector>

#include "llr_common.cuh"
#include "llr_internal.h"

namespace llr {

namespace {

constexpr unsigned long long kSubspaceStream = 0x5342ull;   // "SB"
constexpr int kSimThreads = 256;
constexpr int kSimBatch = 64;          // signals staged per round
constexpr int kMaxQ = 64;              // q-samples supported by the solver

__device__ __forceinline__ double unit_draw(unsigned long long seed, long long i, int k) {
  const unsigned long long x = llr_rng_u64(seed, kSubspaceStream, 5ull * (unsigned long long)i + k);
  return ((double)(x >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}

// signal of draw i at every q -> out[q * stride]
__device__ void simulate(long long i, unsigned long long seed, double lo, double hi, const double* b, const double* g,
                         int nq, double* out, int stride, int q0, int dq) {
  const double u1 = unit_draw(seed, i, 0), u2 = unit_draw(seed, i, 1);
  const double lam[3] = {lo + (hi - lo) * unit_draw(seed, i, 2), lo + (hi - lo) * unit_draw(seed, i, 3),
                         lo + (hi - lo) * unit_draw(seed, i, 4)};
  const double th = 6.283185307179586476925286766559 * u1, ph = acos(2.0 * u2 - 1.0);
  double e1[3] = {sin(ph) * cos(th), sin(ph) * sin(th), cos(ph)};
  const double n1 = sqrt(e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2]);
  for (int a = 0; a < 3; ++a) e1[a] /= n1;
  const double tmp[3] = {fabs(e1[0] - 1.0) < (double)FLT_EPSILON ? 0.0 : 1.0,
                         fabs(e1[0] - 1.0) < (double)FLT_EPSILON ? 1.0 : 0.0, 0.0};
  double e2[3] = {e1[1] * tmp[2] - e1[2] * tmp[1], e1[2] * tmp[0] - e1[0] * tmp[2], e1[0] * tmp[1] - e1[1] * tmp[0]};
  const double n2 = sqrt(e2[0] * e2[0] + e2[1] * e2[1] + e2[2] * e2[2]);
  for (int a = 0; a < 3; ++a) e2[a] /= n2;
  const double e3[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
  for (int q = q0; q < nq; q += dq) {
    const double* gq = g + 3 * q;
    const double p1 = e1[0] * gq[0] + e1[1] * gq[1] + e1[2] * gq[2];
    const double p2 = e2[0] * gq[0] + e2[1] * gq[1] + e2[2] * gq[2];
    const double p3 = e3[0] * gq[0] + e3[1] * gq[1] + e3[2] * gq[2];
    out[q * stride] = exp(-b[q] * (lam[0] * p1 * p1 + lam[1] * p2 * p2 + lam[2] * p3 * p3));
  }
}

// partial Gram (upper triangle, packed row-major i <= j) of this CTA's contiguous draw range
__global__ void __launch_bounds__(kSimThreads) gram_partial_kernel(const double* __restrict__ b_g, int nq,
                                                                    long long n_sig, unsigned long long seed,
                                                                    double lo, double hi, double* __restrict__ part) {
  extern __shared__ double sm[];
  double* b = sm;                    // [nq]
  double* g = sm + nq;               // [nq][3]
  double* sig = sm + 4 * nq;         // [kSimBatch][nq + 1]
  const int ld = nq + 1;
  for (int i = threadIdx.x; i < 4 * nq; i += blockDim.x) sm[i] = b_g[i];
  const long long per = (n_sig + gridDim.x - 1) / gridDim.x;
  const long long i0 = (long long)blockIdx.x * per, i1 = min(n_sig, i0 + per);
  const int np = nq * (nq + 1) / 2;
  double acc[(kMaxQ * (kMaxQ + 1) / 2 + kSimThreads - 1) / kSimThreads];
  int ei[sizeof(acc) / sizeof(double)], ej[sizeof(acc) / sizeof(double)];
  constexpr int K = sizeof(acc) / sizeof(double);
#pragma unroll
  for (int k = 0; k < K; ++k) {
    acc[k] = 0.0;
    int e = threadIdx.x + k * kSimThreads, i = 0;
    if (e < np) {
      while (e >= nq - i) { e -= nq - i; ++i; }
      ei[k] = i;
      ej[k] = i + e;
    } else {
      ei[k] = ej[k] = -1;
    }
  }
  __syncthreads();
  for (long long s0 = i0; s0 < i1; s0 += kSimBatch) {
    const int cnt = (int)min((long long)kSimBatch, i1 - s0);
    // 4 threads per draw, each a quarter of the q-samples
    const int d = threadIdx.x & (kSimBatch - 1), part_q = threadIdx.x / kSimBatch;
    if (d < cnt) simulate(s0 + d, seed, lo, hi, b, g, nq, sig + d * ld, 1, part_q, kSimThreads / kSimBatch);
    __syncthreads();
    for (int t = 0; t < cnt; ++t) {
      const double* st = sig + t * ld;
#pragma unroll
      for (int k = 0; k < K; ++k)
        if (ei[k] >= 0) acc[k] = fma(st[ei[k]], st[ej[k]], acc[k]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int e = threadIdx.x + k * kSimThreads;
    if (e < np) part[(long long)blockIdx.x * np + e] = acc[k];
  }
}

__global__ void gram_reduce_kernel(const double* __restrict__ part, int nparts, int np, double* __restrict__ out) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < np; e += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int p = 0; p < nparts; ++p) s += part[(long long)p * np + e];
    out[e] = s;
  }
}

// Cyclic Jacobi on the symmetric n x n matrix (one CTA, FP64): round-robin pairings, n/2
// rotations per round computed in parallel, applied to rows then columns; V accumulates.
__global__ void __launch_bounds__(256) jacobi_sym_kernel(const double* __restrict__ packed, int n, double* __restrict__ evals,
                                                         double* __restrict__ evecs, int max_sweeps) {
  extern __shared__ double js[];
  const int n2 = (n + 1) & ~1;         // even order with a zero row/column when n is odd
  const int ld = n2 + 1;
  double* A = js;                      // [n2][ld]
  double* V = A + n2 * ld;             // [n2][ld]
  double* cs = V + n2 * ld;            // [n2/2][2] rotation c, s
  int* pr = reinterpret_cast<int*>(cs + n2);   // [n2/2][2] pair (p, q)
  __shared__ double off_s;
  const int tid = threadIdx.x;
  for (int e = tid; e < n2 * n2; e += blockDim.x) {
    const int i = e / n2, j = e - i * n2;
    double v = 0.0;
    if (i < n && j < n) {
      const int a = min(i, j), bcol = max(i, j);
      v = packed[a * n - a * (a - 1) / 2 + (bcol - a)];
    }
    A[i * ld + j] = v;
    V[i * ld + j] = i == j ? 1.0 : 0.0;
  }
  __syncthreads();
  const int half = n2 / 2, M = n2 - 1;
  for (int sweep = 0; sweep < max_sweeps; ++sweep) {
    if (tid == 0) off_s = 0.0;
    __syncthreads();
    double loc = 0.0, dia = 0.0;
    for (int e = tid; e < n2 * n2; e += blockDim.x) {
      const int i = e / n2, j = e - i * n2;
      const double v = A[i * ld + j];
      if (i != j) loc += v * v;
      else dia += v * v;
    }
    atomicAdd(&off_s, loc - 1e-28 * dia);   // off-diagonal mass against (1e-14)^2 of the diagonal
    __syncthreads();
    if (!(off_s > 0.0)) break;
    __syncthreads();
    for (int round = 0; round < M; ++round) {
      for (int k = tid; k < half; k += blockDim.x) {
        // circle method: fixed element M, the others rotate
        int p, q;
        if (k == 0) { p = M; q = round; }
        else { p = (round + k) % M; q = (round - k + M) % M; }
        if (p > q) { const int t = p; p = q; q = t; }
        const double apq = A[p * ld + q];
        double c = 1.0, s = 0.0;
        if (apq != 0.0) {
          const double th = (A[q * ld + q] - A[p * ld + p]) / (2.0 * apq);
          const double t = (th >= 0.0 ? 1.0 : -1.0) / (fabs(th) + sqrt(th * th + 1.0));
          c = 1.0 / sqrt(t * t + 1.0);
          s = t * c;
        }
        cs[2 * k] = c; cs[2 * k + 1] = s;
        pr[2 * k] = p; pr[2 * k + 1] = q;
      }
      __syncthreads();
      // A <- J^T A: rows p, q
      for (int e = tid; e < half * n2; e += blockDim.x) {
        const int k = e / n2, j = e - k * n2;
        const int p = pr[2 * k], q = pr[2 * k + 1];
        const double c = cs[2 * k], s = cs[2 * k + 1];
        const double ap = A[p * ld + j], aq = A[q * ld + j];
        A[p * ld + j] = c * ap - s * aq;
        A[q * ld + j] = s * ap + c * aq;
      }
      __syncthreads();
      // A <- A J and V <- V J: columns p, q
      for (int e = tid; e < half * n2; e += blockDim.x) {
        const int k = e / n2, i = e - k * n2;
        const int p = pr[2 * k], q = pr[2 * k + 1];
        const double c = cs[2 * k], s = cs[2 * k + 1];
        const double ap = A[i * ld + p], aq = A[i * ld + q];
        A[i * ld + p] = c * ap - s * aq;
        A[i * ld + q] = s * ap + c * aq;
        const double vp = V[i * ld + p], vq = V[i * ld + q];
        V[i * ld + p] = c * vp - s * vq;
        V[i * ld + q] = s * vp + c * vq;
      }
      __syncthreads();
    }
  }
  for (int i = tid; i < n; i += blockDim.x) evals[i] = A[i * ld + i];
  for (int e = tid; e < n * n; e += blockDim.x) {
    const int i = e / n, j = e - i * n;
    evecs[i + (long long)n * j] = V[i * ld + j];   // column j = eigenvector j
  }
}

}  // namespace

}  // namespace llr

using namespace llr;

extern "C" {

int llr_dti_subspace(const float* b_vals, const float* b_vecs, int32_t nq, int32_t rank, int64_t n_signals,
                     uint64_t seed, float lam_lo, float lam_hi, llr_cf32* S_out, double* sv_out) {
  if (!b_vals || !b_vecs || !S_out || nq < 1 || nq > kMaxQ || rank < 1 || rank > nq || n_signals < 1 ||
      !(lam_hi >= lam_lo))
    return set_error(LLR_ERR_INVALID, "bad subspace arguments (1 <= rank <= nq <= %d, n_signals >= 1)", kMaxQ);
  const int np = nq * (nq + 1) / 2;
  int dev = 0, nsm = 0;
  LLR_CUDA_TRY(cudaGetDevice(&dev));
  LLR_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  const int nparts = (int)std::max<long long>(1, std::min<long long>(2LL * nsm, (n_signals + kSimBatch - 1) / kSimBatch));
  std::vector<double> bg(4 * (size_t)nq);
  for (int q = 0; q < nq; ++q) {
    bg[q] = b_vals[q];
    for (int a = 0; a < 3; ++a) bg[nq + 3 * q + a] = b_vecs[3 * q + a];
  }
  double *d_bg = nullptr, *d_part = nullptr, *d_gram = nullptr, *d_ev = nullptr, *d_vec = nullptr;
  auto cleanup = [&]() {
    cudaFree(d_bg); cudaFree(d_part); cudaFree(d_gram); cudaFree(d_ev); cudaFree(d_vec);
  };
  cudaError_t e = cudaMalloc((void**)&d_bg, sizeof(double) * bg.size());
  if (e == cudaSuccess) e = cudaMalloc((void**)&d_part, sizeof(double) * (size_t)nparts * np);
  if (e == cudaSuccess) e = cudaMalloc((void**)&d_gram, sizeof(double) * np);
  if (e == cudaSuccess) e = cudaMalloc((void**)&d_ev, sizeof(double) * nq);
  if (e == cudaSuccess) e = cudaMalloc((void**)&d_vec, sizeof(double) * nq * nq);
  if (e == cudaSuccess) e = cudaMemcpy(d_bg, bg.data(), sizeof(double) * bg.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    const size_t smem = sizeof(double) * (4 * (size_t)nq + (size_t)kSimBatch * (nq + 1));
    e = cudaFuncSetAttribute(gram_partial_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) {
      note_launch();
      gram_partial_kernel<<<nparts, kSimThreads, smem>>>(d_bg, nq, n_signals, seed, (double)lam_lo, (double)lam_hi,
                                                          d_part);
      e = cudaGetLastError();
    }
  }
  if (e == cudaSuccess) {
    note_launch();
    gram_reduce_kernel<<<(np + 255) / 256, 256>>>(d_part, nparts, np, d_gram);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    const int n2 = (nq + 1) & ~1;
    const size_t smem = sizeof(double) * (2 * (size_t)n2 * (n2 + 1) + n2) + sizeof(int) * n2;
    e = cudaFuncSetAttribute(jacobi_sym_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) {
      note_launch();
      jacobi_sym_kernel<<<1, 256, smem>>>(d_gram, nq, d_ev, d_vec, 30);
      e = cudaGetLastError();
    }
  }
  std::vector<double> ev(nq), vec((size_t)nq * nq);
  if (e == cudaSuccess) e = cudaMemcpy(ev.data(), d_ev, sizeof(double) * nq, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(vec.data(), d_vec, sizeof(double) * nq * nq, cudaMemcpyDeviceToHost);
  cleanup();
  if (e != cudaSuccess) return cuda_error(e, "subspace construction", __FILE__, __LINE__);
  std::vector<int> order(nq);
  for (int i = 0; i < nq; ++i) order[i] = i;
  std::sort(order.begin(), order.end(), [&](int a, int b) { return ev[a] > ev[b]; });
  for (int r = 0; r < rank; ++r) {
    const int c = order[r];
    // sign convention: the largest-magnitude entry of each vector is positive
    int imax = 0;
    for (int q = 1; q < nq; ++q)
      if (std::fabs(vec[q + (size_t)nq * c]) > std::fabs(vec[imax + (size_t)nq * c])) imax = q;
    const double sgn = vec[imax + (size_t)nq * c] < 0.0 ? -1.0 : 1.0;
    for (int q = 0; q < nq; ++q) S_out[q + (size_t)nq * r] = llr_cf32{(float)(sgn * vec[q + (size_t)nq * c]), 0.f};
    if (sv_out) sv_out[r] = std::sqrt(std::max(ev[c], 0.0));
  }
  return LLR_OK;
}

}  // extern "C"
