// Fused locally-low-rank proximal step.
//
// One CTA owns one Casorati matrix at a time (persistent grid):
//   gather (periodic wrap, scale + phase on load)  -> shared memory C (m x n)
//   Gram G = C^H C on FP32 FMA                      -> shared memory
//   cyclic parallel Jacobi (round-robin pairs)      -> eigenpairs of G
//   singular-value map g(sigma) (hard rank / soft threshold)
//   W = V diag(g) V^H ;  C' = C W                   -> scatter (phase on store)
// This replaces, per block, lift_data_set (block.rs:147-164), cusolver gesvda
// (cusolver.rs:20-151), rhsCdgmmBatched (kernels.cu:11-67), the CGEMM (U S) V^H
// (low_rank.rs:55) and un_lift_data_set (block.rs:166-184): since U_r S_r V_r^H = C V_r V_r^H,
// every prox is C -> C W with W Hermitian n x n.
#include <cstdio>
#include <algorithm>

#include "llr_prox_common.cuh"

namespace llr {

namespace {

struct SmemLayout {
  int ldc;        // leading dimension of C in shared memory (odd)
  int np;         // padded n for Gram tiles
  int ksplit;     // Gram K-split factor
  size_t off_rot, off_pair, off_ev, off_g, off_act, off_A, off_V, off_scr, off_C, total;
};



template <int NPMAX, int TG>
SmemLayout make_layout(int m, int n) {
  SmemLayout L;
  L.ldc = (m & 1) ? m : m + 1;
  int nt = (n + TG - 1) / TG;
  L.np = nt * TG;
  int tiles = nt * nt;
  L.ksplit = std::max(1, kLlrThreads / tiles);
  size_t off = 256;  // misc
  L.off_rot = off; off = align16(off + sizeof(float4) * (NPMAX / 2));
  L.off_pair = off; off = align16(off + sizeof(int2) * (NPMAX / 2));
  L.off_ev = off; off = align16(off + sizeof(float) * NPMAX);
  L.off_g = off; off = align16(off + sizeof(float) * NPMAX);
  L.off_act = off; off = align16(off + sizeof(int) * NPMAX);
  L.off_A = off; off = align16(off + sizeof(float2) * NPMAX * (NPMAX + 1));
  L.off_V = off; off = align16(off + sizeof(float2) * NPMAX * (NPMAX + 1));
  L.off_scr = off;
  if (L.ksplit > 1) off = align16(off + sizeof(float2) * (size_t)L.ksplit * L.np * L.np);
  L.off_C = off; off = align16(off + sizeof(float2) * (size_t)n * L.ldc);
  L.total = off;
  return L;
}

template <int NPMAX, int TG>
__global__ void __launch_bounds__(kLlrThreads) llr_prox_jacobi_kernel(BlockSource src, ProxOp op, SmemLayout L) {
  extern __shared__ __align__(16) unsigned char smem[];
  Misc* misc = reinterpret_cast<Misc*>(smem);
  float4* rot = reinterpret_cast<float4*>(smem + L.off_rot);
  int2* pairs = reinterpret_cast<int2*>(smem + L.off_pair);
  float* ev = reinterpret_cast<float*>(smem + L.off_ev);
  float* g = reinterpret_cast<float*>(smem + L.off_g);
  int* act = reinterpret_cast<int*>(smem + L.off_act);
  float2* A = reinterpret_cast<float2*>(smem + L.off_A);
  float2* V = reinterpret_cast<float2*>(smem + L.off_V);
  float2* scr = reinterpret_cast<float2*>(smem + L.off_scr);
  float2* Cs = reinterpret_cast<float2*>(smem + L.off_C);
  constexpr int lda = NPMAX + 1;
  const int m = op.m, n = op.n;

  if (threadIdx.x == 0) block_shift(src, misc->shift);
  __syncthreads();
  int sh[3] = {misc->shift[0], misc->shift[1], misc->shift[2]};
  const long long count = src.blk_list ? (long long)*src.blk_count : src.nblocks;

  for (long long i = blockIdx.x; i < count; i += gridDim.x) {
    const long long blk = src.blk_list ? (long long)src.blk_list[i] : i;
    gather_block(src, blk, sh, m, n, Cs, L.ldc);
    __syncthreads();
    gram<NPMAX, TG>(Cs, L.ldc, m, n, A, scr, L.ksplit);
    jacobi<NPMAX>(A, V, n, rot, pairs, misc, 16);
    if (op.block_stat) {
      if (threadIdx.x == 0) {
        float mx = 0.f;
        for (int k = 0; k < n; ++k) mx = fmaxf(mx, A[k * lda + k].x);
        op.block_stat[blk] = mx;
      }
      __syncthreads();
      continue;
    }
    singular_map(A, lda, n, op.mode, op.rank, op.lambda, ev, g, act, misc);
    if (op.blk_nuc && op.mode != LLR_PROX_HARD_RANK && threadIdx.x == 0)
      op.blk_nuc[blk] = nuclear_from_eigs(ev, n, op.lambda);
    const int na = misc->n_active;
    if (!(na == n && op.mode == LLR_PROX_HARD_RANK)) {
      form_W(A, V, lda, n, g, act, na);
      apply_W<NPMAX, TG>(Cs, L.ldc, m, n, A);
    }
    scatter_block(src, blk, sh, m, n, Cs, L.ldc);
    __syncthreads();
  }
}

template <int NPMAX, int TG>
int launch_jacobi_instance(const BlockSource& src, const ProxOp& op, cudaStream_t stream) {
  SmemLayout L = make_layout<NPMAX, TG>(op.m, op.n);
  if (L.total > 227 * 1024)
    return set_error(LLR_ERR_UNSUPPORTED, "Casorati %dx%d needs %zu B of shared memory (max 232448)", op.m, op.n,
                     L.total);
  auto kern = llr_prox_jacobi_kernel<NPMAX, TG>;
  LLR_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.total));
    LLR_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
  int dev = 0, nsm = 0, occ = 0;
  LLR_CUDA_TRY(cudaGetDevice(&dev));
  LLR_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  LLR_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kLlrThreads, L.total));
  if (occ < 1) return set_error(LLR_ERR_UNSUPPORTED, "prox kernel cannot be resident (smem %zu B)", L.total);
  long long grid = std::min<long long>(src.nblocks, (long long)nsm * occ);
  if (grid < 1) return LLR_OK;
  note_launch();
  kern<<<(unsigned)grid, kLlrThreads, L.total, stream>>>(src, op, L);
  LLR_CUDA_TRY(cudaGetLastError());
  return LLR_OK;
}

}  // namespace

bool llr_prox_jacobi_supported(int m, int n) {
  if (m < 1 || n < 1 || n > 64) return false;
  size_t t;
  if (n <= 16) t = make_layout<16, 2>(m, n).total;
  else if (n <= 32) t = make_layout<32, 2>(m, n).total;
  else t = make_layout<64, 4>(m, n).total;
  return t <= 227 * 1024;
}

// Jacobi-path prox over all blocks of `src` (or over src.blk_list when set).
int launch_llr_prox_jacobi(const BlockSource& src, const ProxOp& op, cudaStream_t stream) {
  if (op.n < 1 || op.m < 1) return set_error(LLR_ERR_INVALID, "empty Casorati matrix %dx%d", op.m, op.n);
  if (src.nblocks == 0) return LLR_OK;
  if (op.n <= 16) return launch_jacobi_instance<16, 2>(src, op, stream);
  if (op.n <= 32) return launch_jacobi_instance<32, 2>(src, op, stream);
  if (op.n <= 64) return launch_jacobi_instance<64, 4>(src, op, stream);
  return set_error(LLR_ERR_UNSUPPORTED, "Casorati column count %d > 64 is not supported", op.n);
}



// =======================================================================================
// Subspace-constrained prox: X <- LR(X S) S^H per block (lib.rs:281-289).  The projected
// matrix Z = X S (m x srank) is formed while gathering (each voxel's nq-vector times S),
// so the full m x nq Casorati never needs to be staged; Z' = Z W (srank x srank Jacobi);
// the store streams X' = Z' S^H back volume by volume.
// =======================================================================================
namespace {

constexpr int kSubMax = 16;   // max subspace rank

template <int NPMAX, int KM>
__global__ void __launch_bounds__(kLlrThreads) llr_subspace_kernel(BlockSource src, SubspaceOp op, SmemLayout L) {
  extern __shared__ __align__(16) unsigned char smem[];
  Misc* misc = reinterpret_cast<Misc*>(smem);
  float4* rot = reinterpret_cast<float4*>(smem + L.off_rot);
  int2* pairs = reinterpret_cast<int2*>(smem + L.off_pair);
  float* ev = reinterpret_cast<float*>(smem + L.off_ev);
  float* g = reinterpret_cast<float*>(smem + L.off_g);
  int* act = reinterpret_cast<int*>(smem + L.off_act);
  float2* A = reinterpret_cast<float2*>(smem + L.off_A);
  float2* V = reinterpret_cast<float2*>(smem + L.off_V);
  float2* scr = reinterpret_cast<float2*>(smem + L.off_scr);
  float2* Z = reinterpret_cast<float2*>(smem + L.off_C);           // srank x ldc
  float2* Ss = Z + (size_t)op.srank * L.ldc;                        // nq x srank
  constexpr int lda = NPMAX + 1;
  const int m = op.m, nq = op.nq, sr = op.srank;
  // S is nq x srank column-major; keep it row-major (q, k) in shared memory.
  for (int i = threadIdx.x; i < nq * sr; i += blockDim.x) {
    const int q = i / sr, k = i - q * sr;
    Ss[i] = op.S[q + (long long)nq * k];
  }
  if (threadIdx.x == 0) block_shift(src, misc->shift);
  __syncthreads();
  int sh[3] = {misc->shift[0], misc->shift[1], misc->shift[2]};

  for (long long blk = blockIdx.x; blk < src.nblocks; blk += gridDim.x) {
    // Z[r, k] = sum_q X[r, q] S[q, k]
    for (int r = threadIdx.x; r < m; r += blockDim.x) {
      float2 z[KM];
#pragma unroll
      for (int k = 0; k < KM; ++k) z[k] = make_float2(0.f, 0.f);
      int ix = 0, iy = 0, iz = 0;
      if (src.kind == 1) block_row_coord(src, blk, sh, r, ix, iy, iz);
      for (int q = 0; q < nq; ++q) {
        float2 v;
        if (src.kind == 0) {
          v = src.data[blk * (long long)m * nq + (long long)q * m + r];
        } else {
          v = src.data[planar_index(src.g, ix, iy, iz, q)];
          v = cscale(cmul_bc(v, phase_at(src.ph, src.g, q, ix, iy, iz)), src.load_scale);
        }
#pragma unroll
        for (int k = 0; k < KM; ++k)
          if (k < sr) cfma(z[k], v, Ss[q * sr + k]);
      }
#pragma unroll
      for (int k = 0; k < KM; ++k)
        if (k < sr) Z[k * L.ldc + r] = z[k];
    }
    __syncthreads();
    gram<NPMAX, 2>(Z, L.ldc, m, sr, A, scr, L.ksplit);
    if (threadIdx.x < 32) jacobi_warp<NPMAX>(A, V, sr, rot, pairs, misc, 16);
    __syncthreads();
    singular_map(A, lda, sr, op.mode, op.rank, op.lambda, ev, g, act, misc);
    form_W(A, V, lda, sr, g, act, misc->n_active);
    apply_W<NPMAX, 2>(Z, L.ldc, m, sr, A);
    // X'[r, q] = sum_k Z'[r, k] conj(S[q, k])
    for (int r = threadIdx.x; r < m; r += blockDim.x) {
      float2 z[KM];
#pragma unroll
      for (int k = 0; k < KM; ++k) z[k] = (k < sr) ? Z[k * L.ldc + r] : make_float2(0.f, 0.f);
      int ix = 0, iy = 0, iz = 0;
      if (src.kind == 1) block_row_coord(src, blk, sh, r, ix, iy, iz);
      for (int q = 0; q < nq; ++q) {
        float2 v = make_float2(0.f, 0.f);
#pragma unroll
        for (int k = 0; k < KM; ++k)
          if (k < sr) cfma_cb(v, z[k], Ss[q * sr + k]);
        if (src.kind == 0) {
          src.data[blk * (long long)m * nq + (long long)q * m + r] = v;
        } else {
          v = cscale(v, src.store_scale);
          if (src.store_phase) v = cmul(v, phase_at(src.ph, src.g, q, ix, iy, iz));
          src.data[planar_index(src.g, ix, iy, iz, q)] = v;
        }
      }
    }
    __syncthreads();
  }
}

// Coefficient output: the same gather and low-rank step, storing Z' = LR(X S) as srank
// planar coefficient volumes (image space) for a shrink in the coefficient domain.
template <int NPMAX, int KM>
__global__ void __launch_bounds__(kLlrThreads) llr_subspace_coef_kernel(BlockSource src, SubspaceOp op, SmemLayout L) {
  extern __shared__ __align__(16) unsigned char smem[];
  Misc* misc = reinterpret_cast<Misc*>(smem);
  float4* rot = reinterpret_cast<float4*>(smem + L.off_rot);
  int2* pairs = reinterpret_cast<int2*>(smem + L.off_pair);
  float* ev = reinterpret_cast<float*>(smem + L.off_ev);
  float* g = reinterpret_cast<float*>(smem + L.off_g);
  int* act = reinterpret_cast<int*>(smem + L.off_act);
  float2* A = reinterpret_cast<float2*>(smem + L.off_A);
  float2* V = reinterpret_cast<float2*>(smem + L.off_V);
  float2* scr = reinterpret_cast<float2*>(smem + L.off_scr);
  float2* Z = reinterpret_cast<float2*>(smem + L.off_C);
  float2* Ss = Z + (size_t)op.srank * L.ldc;
  const int m = op.m, nq = op.nq, sr = op.srank;
  for (int i = threadIdx.x; i < nq * sr; i += blockDim.x) {
    const int q = i / sr, k = i - q * sr;
    Ss[i] = op.S[q + (long long)nq * k];
  }
  if (threadIdx.x == 0) block_shift(src, misc->shift);
  __syncthreads();
  int sh[3] = {misc->shift[0], misc->shift[1], misc->shift[2]};
  Geom gc = src.g;
  gc.nq = sr;
  for (long long blk = blockIdx.x; blk < src.nblocks; blk += gridDim.x) {
    for (int r = threadIdx.x; r < m; r += blockDim.x) {
      float2 z[KM];
#pragma unroll
      for (int k = 0; k < KM; ++k) z[k] = make_float2(0.f, 0.f);
      int ix = 0, iy = 0, iz = 0;
      block_row_coord(src, blk, sh, r, ix, iy, iz);
      const float2 p0 = phase_at(src.ph, src.g, 0, ix, iy, iz);   // every volume's, when uniform
#pragma unroll 4
      for (int q = 0; q < nq; ++q) {
        float2 v = src.data[planar_index(src.g, ix, iy, iz, q)];
        v = cscale(cmul_bc(v, src.ph_uniform ? p0 : phase_at(src.ph, src.g, q, ix, iy, iz)), src.load_scale);
#pragma unroll
        for (int k = 0; k < KM; ++k)
          if (k < sr) cfma(z[k], v, Ss[q * sr + k]);
      }
#pragma unroll
      for (int k = 0; k < KM; ++k)
        if (k < sr) Z[k * L.ldc + r] = z[k];
    }
    __syncthreads();
    gram<NPMAX, 2>(Z, L.ldc, m, sr, A, scr, L.ksplit);
    if (threadIdx.x < 32) jacobi_warp<NPMAX>(A, V, sr, rot, pairs, misc, 16);
    __syncthreads();
    singular_map(A, NPMAX + 1, sr, op.mode, op.rank, op.lambda, ev, g, act, misc);
    form_W(A, V, NPMAX + 1, sr, g, act, misc->n_active);
    apply_W<NPMAX, 2>(Z, L.ldc, m, sr, A);
    for (int r = threadIdx.x; r < m; r += blockDim.x) {
      int ix = 0, iy = 0, iz = 0;
      block_row_coord(src, blk, sh, r, ix, iy, iz);
      for (int k = 0; k < sr; ++k) op.coef_out[planar_index(gc, ix, iy, iz, k)] = Z[k * L.ldc + r];
    }
    __syncthreads();
  }
}

template <int KM>
__global__ void __launch_bounds__(256) subspace_expand_kernel(const float2* __restrict__ coef, float2* __restrict__ x,
                                                              const float2* __restrict__ S, int srank, Geom g,
                                                              PhaseTab ph, int store_phase, int ph_uniform,
                                                              float scale) {
  __shared__ float2 Ss[64 * kSubMax];
  for (int i = threadIdx.x; i < g.nq * srank; i += blockDim.x) Ss[i] = S[i];   // column-major (q, k)
  __syncthreads();
  for (long long v = blockIdx.x * 256LL + threadIdx.x; v < g.V; v += (long long)gridDim.x * 256) {
    float2 c[KM];
#pragma unroll
    for (int k = 0; k < KM; ++k) c[k] = k < srank ? coef[v + g.V * k] : make_float2(0.f, 0.f);
    const int iy = (int)(v % g.ny);
    const long long r = v / g.ny;
    const int iz = (int)(r % g.nz), ix = (int)(r / g.nz);
    // the stored value's factor: scale times the phase (computed once when every volume shares it)
    const float2 f0 = cscale(store_phase ? phase_at(ph, g, 0, ix, iy, iz) : make_float2(1.f, 0.f), scale);
#pragma unroll 4
    for (int q = 0; q < g.nq; ++q) {
      float2 a = make_float2(0.f, 0.f);
#pragma unroll
      for (int k = 0; k < KM; ++k)
        if (k < srank) cfma_cb(a, c[k], Ss[q + g.nq * k]);
      const float2 f = (ph_uniform || !store_phase) ? f0 : cscale(phase_at(ph, g, q, ix, iy, iz), scale);
      x[v + g.V * q] = cmul(a, f);
    }
  }
}

}  // namespace

int launch_llr_prox_subspace(const BlockSource& src, const SubspaceOp& op, cudaStream_t stream) {
  if (op.srank < 1 || op.srank > kSubMax)
    return set_error(LLR_ERR_UNSUPPORTED, "subspace rank %d outside [1, %d]", op.srank, kSubMax);
  if (src.nblocks == 0) return LLR_OK;
  SmemLayout L = make_layout<16, 2>(op.m, op.srank);
  L.total = align16(L.total + sizeof(float2) * (size_t)op.nq * op.srank);
  if (L.total > 227 * 1024) return set_error(LLR_ERR_UNSUPPORTED, "subspace prox needs %zu B smem", L.total);
  if (op.coef_out && src.kind != 1) return set_error(LLR_ERR_INVALID, "coefficient output needs volume blocks");
  // per-thread coefficient registers sized to the rank class (fewer registers, more CTAs per SM)
  auto kern = op.coef_out ? (op.srank <= 8 ? llr_subspace_coef_kernel<16, 8> : llr_subspace_coef_kernel<16, 16>)
                          : (op.srank <= 8 ? llr_subspace_kernel<16, 8> : llr_subspace_kernel<16, 16>);
  LLR_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.total));
    LLR_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
  int dev = 0, nsm = 0, occ = 0;
  LLR_CUDA_TRY(cudaGetDevice(&dev));
  LLR_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  LLR_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kLlrThreads, L.total));
  if (occ < 1) return set_error(LLR_ERR_UNSUPPORTED, "subspace kernel cannot be resident");
  long long grid = std::min<long long>(src.nblocks, (long long)nsm * occ);
  note_launch();
  kern<<<(unsigned)grid, kLlrThreads, L.total, stream>>>(src, op, L);
  LLR_CUDA_TRY(cudaGetLastError());
  return LLR_OK;
}

// =======================================================================================
// Reference-layout lift / un-lift (block.rs:147-184): row r of block i in block
// col-major order (x fastest), volume q is column q.
// =======================================================================================
namespace {

__global__ void lift_kernel(const float2* __restrict__ vol, float2* __restrict__ mat, int nx, int ny, int nz,
                            int nq, int bx, int by, int bz, int gx, int gy, int sx, int sy, int sz,
                            long long start, long long n, int dir) {
  const long long m = (long long)bx * by * bz;
  const long long per = m * nq;
  const long long tot = per * n;
  const long long V = (long long)nx * ny * nz;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < tot; i += (long long)gridDim.x * blockDim.x) {
    const long long c = i / per;
    const long long rem = i - c * per;
    const int q = (int)(rem / m);
    const int r = (int)(rem - (long long)q * m);
    const long long blk = start + c;
    const int gxi = (int)(blk % gx);
    const long long t = blk / gx;
    const int gyi = (int)(t % gy);
    const int gzi = (int)(t / gy);
    const int rx = r % bx, ry = (r / bx) % by, rz = r / (bx * by);
    const int ix = (gxi * bx + sx + rx) % nx;
    const int iy = (gyi * by + sy + ry) % ny;
    const int iz = (gzi * bz + sz + rz) % nz;
    const long long a = (long long)ix + (long long)nx * ((long long)iy + (long long)ny * iz) + V * q;
    if (dir == 0) mat[i] = vol[a];
    else const_cast<float2*>(vol)[a] = mat[i];
  }
}

}  // namespace

int launch_lift(const float2* vol, float2* mat, const int* vs, int nq, const int* bs, const int* sh, long long start,
                long long n, int dir, cudaStream_t s) {
  int g[3];
  for (int a = 0; a < 3; ++a) g[a] = vs[a] / bs[a];
  const long long tot = (long long)bs[0] * bs[1] * bs[2] * nq * n;
  if (tot == 0) return LLR_OK;
  long long blocks = std::min<long long>((tot + 255) / 256, 148LL * 16);
  note_launch();
  lift_kernel<<<(unsigned)blocks, 256, 0, s>>>(vol, mat, vs[0], vs[1], vs[2], nq, bs[0], bs[1], bs[2], g[0], g[1],
                                               sh[0], sh[1], sh[2], start, n, dir);
  LLR_CUDA_TRY(cudaGetLastError());
  return LLR_OK;
}

// =======================================================================================
// rhsCdgmmBatched (kernels.cu:11-67) and a batched complex GEMM with the semantics of
// cublas_cgemm_strided_batched_device (cublas.rs:12-105).
int launch_subspace_expand(const float2* coef, float2* x, const float2* S, int srank, const Geom& g, PhaseTab ph,
                           int store_phase, int ph_uniform, float scale, cudaStream_t s) {
  if (srank < 1 || srank > kSubMax || g.nq > 64) return set_error(LLR_ERR_UNSUPPORTED, "subspace expand shape");
  const long long blocks = std::min<long long>((g.V + 255) / 256, 148LL * 16);
  note_launch();
  if (srank <= 8)
    subspace_expand_kernel<8><<<(unsigned)blocks, 256, 0, s>>>(coef, x, S, srank, g, ph, store_phase, ph_uniform, scale);
  else
    subspace_expand_kernel<16><<<(unsigned)blocks, 256, 0, s>>>(coef, x, S, srank, g, ph, store_phase, ph_uniform,
                                                                scale);
  LLR_CUDA_TRY(cudaGetLastError());
  return LLR_OK;
}

// =======================================================================================
namespace {

__global__ void rhs_cdgmm_kernel(int m, int n, int batch, float2* a, const float* d) {
  const long long tot = (long long)m * n * batch;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < tot; i += (long long)gridDim.x * blockDim.x) {
    const long long col = i / m;  // j + n * b
    a[i] = cscale(a[i], d[col]);
  }
}

// C[i, j] = alpha * sum_l op(A)[i, l] op(B)[l, j] + beta * C[i, j], 16x16 output tiles.
__global__ void cgemm_kernel(int m, int k, int n, int broadcast_a, float2 alpha, float2 beta, int ta, int tb,
                             const float2* __restrict__ A, const float2* __restrict__ B, float2* __restrict__ C) {
  __shared__ float2 As[16][17];
  __shared__ float2 Bs[16][17];
  const int b = blockIdx.z;
  const float2* Ab = A + (broadcast_a ? 0 : (long long)b * m * k);
  const float2* Bb = B + (long long)b * k * n;
  float2* Cb = C + (long long)b * m * n;
  const int i = blockIdx.x * 16 + threadIdx.x;
  const int j = blockIdx.y * 16 + threadIdx.y;
  float2 acc = make_float2(0.f, 0.f);
  for (int l0 = 0; l0 < k; l0 += 16) {
    {  // A tile: rows blockIdx.x*16 + tx, cols l0 + ty
      const int ii = blockIdx.x * 16 + threadIdx.x, ll = l0 + threadIdx.y;
      float2 v = make_float2(0.f, 0.f);
      if (ii < m && ll < k) v = ta ? cconj(Ab[ll + (long long)k * ii]) : Ab[ii + (long long)m * ll];
      As[threadIdx.x][threadIdx.y] = v;
    }
    {  // B tile: rows l0 + tx, cols blockIdx.y*16 + ty
      const int ll = l0 + threadIdx.x, jj = blockIdx.y * 16 + threadIdx.y;
      float2 v = make_float2(0.f, 0.f);
      if (ll < k && jj < n) v = tb ? cconj(Bb[jj + (long long)n * ll]) : Bb[ll + (long long)k * jj];
      Bs[threadIdx.x][threadIdx.y] = v;
    }
    __syncthreads();
#pragma unroll
    for (int l = 0; l < 16; ++l) cfma(acc, As[threadIdx.x][l], Bs[l][threadIdx.y]);
    __syncthreads();
  }
  if (i < m && j < n) {
    float2 c = Cb[i + (long long)m * j];
    float2 out = cmul(alpha, acc);
    if (beta.x != 0.f || beta.y != 0.f) out = cadd(out, cmul(beta, c));
    Cb[i + (long long)m * j] = out;
  }
}

}  // namespace

namespace {
// out (n x m per batch) = conj(in (m x n per batch))^T, column-major (dti_subspace.rs:211-221).
__global__ void conj_transpose_kernel(const float2* __restrict__ in, float2* __restrict__ out, int m, int n) {
  __shared__ float2 tile[32][33];
  const long long off = (long long)blockIdx.z * m * n;
  const int i0 = blockIdx.x * 32, j0 = blockIdx.y * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int i = i0 + threadIdx.x, j = j0 + k;
    if (i < m && j < n) tile[k][threadIdx.x] = in[off + i + (long long)m * j];
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int j = j0 + threadIdx.x, i = i0 + k;
    if (i < m && j < n) out[off + j + (long long)n * i] = cconj(tile[threadIdx.x][k]);
  }
}
}  // namespace

int launch_conj_transpose(const float2* in, float2* out, int m, int n, int batch, cudaStream_t s) {
  if ((long long)m * n * batch == 0) return LLR_OK;
  dim3 grid((m + 31) / 32, (n + 31) / 32, batch);
  note_launch();
  conj_transpose_kernel<<<grid, dim3(32, 8), 0, s>>>(in, out, m, n);
  LLR_CUDA_TRY(cudaGetLastError());
  return LLR_OK;
}

int launch_rhs_cdgmm(int m, int n, int batch, float2* a, const float* d, cudaStream_t s) {
  const long long tot = (long long)m * n * batch;
  if (tot == 0) return LLR_OK;
  long long blocks = std::min<long long>((tot + 255) / 256, 148LL * 32);
  note_launch();
  rhs_cdgmm_kernel<<<(unsigned)blocks, 256, 0, s>>>(m, n, batch, a, d);
  LLR_CUDA_TRY(cudaGetLastError());
  return LLR_OK;
}

int launch_cgemm(int m, int k, int n, int batch, int broadcast_a, float2 alpha, float2 beta, int ta, int tb,
                 const float2* A, const float2* B, float2* C, cudaStream_t s) {
  if (m == 0 || n == 0 || batch == 0) return LLR_OK;
  dim3 grid((m + 15) / 16, (n + 15) / 16, batch);
  dim3 block(16, 16);
  note_launch();
  cgemm_kernel<<<grid, block, 0, s>>>(m, k, n, broadcast_a, alpha, beta, ta, tb, A, B, C);
  LLR_CUDA_TRY(cudaGetLastError());
  return LLR_OK;
}

}  // namespace llr
