// Device building blocks shared by the LLR prox kernels (llr_prox.cu: Jacobi and subspace
// kernels; llr_prox_trd.cu: tridiagonal-path kernel).  Everything here has internal linkage.
#pragma once

#include <algorithm>

#include "llr_internal.h"

namespace llr {
namespace {

__host__ __device__ inline size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

struct Misc {
  int flag[2];
  float normF;
  int n_active;
  int shift[3];
  int n_below;      // eigenvalues below the threshold (tridiagonal path)
  int ra;           // active eigenpairs (tridiagonal path)
  int fail;         // tridiagonal path rejected -> Jacobi fallback
  float tnorm;      // max |Gershgorin bound| of T'
  float gl, gu;     // Gershgorin interval
  float pivmin;
  float red[32];
};

// ---------------------------------------------------------------------------------------
// block geometry
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ void block_shift(const BlockSource& s, int* sh) {
  if (s.it_ptr) {
    long long it = *s.it_ptr;
    sh[0] = llr_shift_draw(s.seed, it, 0, s.mx);
    sh[1] = llr_shift_draw(s.seed, it, 1, s.my);
    sh[2] = llr_shift_draw(s.seed, it, 2, s.mz);
  } else {
    sh[0] = s.sx; sh[1] = s.sy; sh[2] = s.sz;
  }
  sh[0] += s.ox; sh[1] += s.oy; sh[2] += s.oz;
}

// Voxel coordinates of row r of block `blk`.  Rows are ordered y fastest, then z, then x, and
// so are the blocks (the planar layout's order: blocks that run at the same time share DRAM
// pages; the order of independent blocks does not change any result).  Corner = grid index *
// block + shift (block.rs:122-133); every coordinate wraps modulo the volume (block.rs:20-22).
__device__ __forceinline__ void block_row_coord(const BlockSource& s, long long blk, const int* sh, int r,
                                                int& ix, int& iy, int& iz) {
  int gyi = (int)(blk % s.gy);
  long long t = blk / s.gy;
  int gzi = (int)(t % s.gz);
  int gxi = (int)(t / s.gz);
  int ry = r % s.by;
  int t2 = r / s.by;
  int rz = t2 % s.bz;
  int rx = t2 / s.bz;
  ix = gxi * s.bx + sh[0] + rx; if (ix >= s.g.nx) ix -= s.g.nx; if (ix >= s.g.nx) ix %= s.g.nx;
  iy = gyi * s.by + sh[1] + ry; if (iy >= s.g.ny) iy -= s.g.ny; if (iy >= s.g.ny) iy %= s.g.ny;
  iz = gzi * s.bz + sh[2] + rz; if (iz >= s.g.nz) iz -= s.g.nz; if (iz >= s.g.nz) iz %= s.g.nz;
}

__device__ void gather_block(const BlockSource& s, long long blk, const int* sh, int m, int n, float2* Cs,
                             int ldc) {
  const int tot = m * n;
  if (s.kind == 0) {
    const float2* src = s.data + blk * (long long)m * n;
    for (int i = threadIdx.x; i < tot; i += blockDim.x) {
      int q = i / m, r = i - q * m;
      Cs[q * ldc + r] = src[i];
    }
    return;
  }
  for (int i = threadIdx.x; i < tot; i += blockDim.x) {
    int q = i / m, r = i - q * m;
    int ix, iy, iz;
    block_row_coord(s, blk, sh, r, ix, iy, iz);
    float2 v = s.data[planar_index(s.g, ix, iy, iz, q)];
    float2 p = phase_at(s.ph, s.g, q, ix, iy, iz);
    v = cscale(cmul_bc(v, p), s.load_scale);
    Cs[q * ldc + r] = v;
  }
}

__device__ void scatter_block(const BlockSource& s, long long blk, const int* sh, int m, int n,
                              const float2* Cs, int ldc) {
  const int tot = m * n;
  if (s.kind == 0) {
    float2* dst = s.data + blk * (long long)m * n;
    for (int i = threadIdx.x; i < tot; i += blockDim.x) {
      int q = i / m, r = i - q * m;
      dst[i] = Cs[q * ldc + r];
    }
    return;
  }
  for (int i = threadIdx.x; i < tot; i += blockDim.x) {
    int q = i / m, r = i - q * m;
    int ix, iy, iz;
    block_row_coord(s, blk, sh, r, ix, iy, iz);
    float2 v = cscale(Cs[q * ldc + r], s.store_scale);
    if (s.store_phase) v = cmul(v, phase_at(s.ph, s.g, q, ix, iy, iz));
    float2* dst = (s.out ? s.out : s.data) + planar_index(s.g, ix, iy, iz, q);
    if (s.accumulate) v = cadd(v, *dst);
    *dst = v;
  }
}

// ---------------------------------------------------------------------------------------
// Gram matrix A = C^H C  (n x n, lda = NPMAX + 1), zero padded to NPMAX.
// Thread tile TG x TG with interleaved columns (j = tj + nt * b) so that a half-warp reads
// consecutive columns of C at one row: conflict-free with an odd ldc.
// ---------------------------------------------------------------------------------------
template <int NPMAX, int TG>
__device__ void gram(const float2* Cs, int ldc, int m, int n, float2* A, float2* scr, int ksplit) {
  constexpr int lda = NPMAX + 1;
  const int tid = threadIdx.x;
  for (int i = tid; i < NPMAX * lda; i += blockDim.x) A[i] = make_float2(0.f, 0.f);
  __syncthreads();
  const int nt = (n + TG - 1) / TG;
  const int tiles = nt * nt;
  const int np = nt * TG;
  if (tid < tiles * ksplit) {
    const int tile = tid % tiles, ks = tid / tiles;
    const int ti = tile / nt, tj = tile - ti * nt;
    const int r0 = (int)(((long long)m * ks) / ksplit), r1 = (int)(((long long)m * (ks + 1)) / ksplit);
    float2 acc[TG][TG];
#pragma unroll
    for (int a = 0; a < TG; ++a)
#pragma unroll
      for (int b = 0; b < TG; ++b) acc[a][b] = make_float2(0.f, 0.f);
    int ci_col[TG], cj_col[TG];
    bool ci_ok[TG], cj_ok[TG];
#pragma unroll
    for (int a = 0; a < TG; ++a) {
      ci_col[a] = ti + nt * a; ci_ok[a] = ci_col[a] < n;
      cj_col[a] = tj + nt * a; cj_ok[a] = cj_col[a] < n;
    }
    for (int r = r0; r < r1; ++r) {
      float2 ci[TG], cj[TG];
#pragma unroll
      for (int a = 0; a < TG; ++a) {
        ci[a] = ci_ok[a] ? Cs[ci_col[a] * ldc + r] : make_float2(0.f, 0.f);
        cj[a] = cj_ok[a] ? Cs[cj_col[a] * ldc + r] : make_float2(0.f, 0.f);
      }
#pragma unroll
      for (int a = 0; a < TG; ++a)
#pragma unroll
        for (int b = 0; b < TG; ++b) cfma_ca(acc[a][b], ci[a], cj[b]);
    }
    if (ksplit == 1) {
#pragma unroll
      for (int a = 0; a < TG; ++a)
#pragma unroll
        for (int b = 0; b < TG; ++b)
          if (ci_ok[a] && cj_ok[b]) A[ci_col[a] * lda + cj_col[b]] = acc[a][b];
    } else {
      float2* P = scr + (size_t)ks * np * np;
#pragma unroll
      for (int a = 0; a < TG; ++a)
#pragma unroll
        for (int b = 0; b < TG; ++b) P[ci_col[a] * np + cj_col[b]] = acc[a][b];
    }
  }
  __syncthreads();
  if (ksplit > 1) {
    for (int idx = tid; idx < n * n; idx += blockDim.x) {
      int i = idx / n, j = idx - i * n;
      float2 s = make_float2(0.f, 0.f);
      for (int k = 0; k < ksplit; ++k) s = cadd(s, scr[(size_t)k * np * np + i * np + j]);
      A[i * lda + j] = s;
    }
    __syncthreads();
  }
}

__device__ float block_sum(float v, float* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  float s = 0.f;
  const int nw = (blockDim.x + 31) >> 5;
  for (int i = 0; i < nw; ++i) s += red[i];
  return s;
}

// ---------------------------------------------------------------------------------------
// Cyclic parallel Jacobi on the Hermitian A (n x n) -> A diagonal, V eigenvectors.
// Round-robin (circle) ordering: n2/2 disjoint pairs per step, n2-1 steps per sweep.
// Each thread applies the combined row/column rotation to whole 2x2 blocks, so one step
// is one barrier for the rotation angles plus one for the update.
// ---------------------------------------------------------------------------------------
template <int NPMAX>
__device__ void jacobi(float2* A, float2* V, int n, float4* rot, int2* pairs, Misc* misc, int max_sweeps,
                       int lda = NPMAX + 1) {
  const int tid = threadIdx.x;
  const int n2 = (n + 1) & ~1;
  const int half = n2 >> 1;
  const int M = n2 - 1;
  for (int idx = tid; idx < n2 * n2; idx += blockDim.x) {
    int i = idx / n2, j = idx - i * n2;
    V[i * lda + j] = make_float2(i == j ? 1.f : 0.f, 0.f);
  }
  float loc = 0.f;
  for (int idx = tid; idx < n * n; idx += blockDim.x) {
    int i = idx / n, j = idx - i * n;
    loc += cabs2(A[i * lda + j]);
  }
  float fro2 = block_sum(loc, misc->red);
  if (tid == 0) { misc->normF = sqrtf(fro2); misc->flag[0] = 0; misc->flag[1] = 0; }
  __syncthreads();
  const float thr = 2.4e-7f * misc->normF;
  if (n2 < 2 || !(misc->normF > 0.f)) return;

  for (int sweep = 0; sweep < max_sweeps; ++sweep) {
    const int fs = sweep & 1;
    for (int step = 0; step < M; ++step) {
      if (tid < half) {
        const int k = tid;
        int p, q;
        if (k == 0) { p = step; q = M; }
        else { p = (step + k) % M; q = (step - k + M) % M; }
        if (p > q) { int t = p; p = q; q = t; }
        float c = 1.f, s = 0.f, ex = 1.f, ey = 0.f;
        if (q < n) {
          const float app = A[p * lda + p].x, aqq = A[q * lda + q].x;
          const float2 apq = A[p * lda + q];
          const float r = hypotf(apq.x, apq.y);
          if (r > thr) {
            const float tau = (aqq - app) / (2.f * r);
            float t;
            if (fabsf(tau) > 1e15f) t = 0.5f / tau;
            else t = copysignf(1.f, tau) / (fabsf(tau) + sqrtf(1.f + tau * tau));
            c = rsqrtf(1.f + t * t);
            s = t * c;
            ex = apq.x / r; ey = apq.y / r;
            misc->flag[fs] = 1;
          }
        }
        rot[k] = make_float4(c, s, ex, ey);
        pairs[k] = make_int2(p, q);
      }
      __syncthreads();
      if (step == 0 && tid == 0) misc->flag[fs ^ 1] = 0;
      for (int b = tid; b < half * half; b += blockDim.x) {
        const int k1 = b / half, k2 = b - k1 * half;
        const int2 P1 = pairs[k1], P2 = pairs[k2];
        const float4 R1 = rot[k1], R2 = rot[k2];
        const bool id1 = (R1.y == 0.f), id2 = (R2.y == 0.f);
        if (id1 && id2) continue;
        const float2 e1 = make_float2(R1.z, R1.w);
        const float2 e2c = make_float2(R2.z, -R2.w);
        float2 a11 = A[P1.x * lda + P2.x], a12 = A[P1.x * lda + P2.y];
        float2 a21 = A[P1.y * lda + P2.x], a22 = A[P1.y * lda + P2.y];
        if (!id2) {  // columns: [x_p, x_q] J2,  J2 = [[c, s], [-s e2*, c e2*]]
          float2 t12 = cmul(a12, e2c), t22 = cmul(a22, e2c);
          float2 b11 = make_float2(R2.x * a11.x - R2.y * t12.x, R2.x * a11.y - R2.y * t12.y);
          float2 b12 = make_float2(R2.y * a11.x + R2.x * t12.x, R2.y * a11.y + R2.x * t12.y);
          float2 b21 = make_float2(R2.x * a21.x - R2.y * t22.x, R2.x * a21.y - R2.y * t22.y);
          float2 b22 = make_float2(R2.y * a21.x + R2.x * t22.x, R2.y * a21.y + R2.x * t22.y);
          a11 = b11; a12 = b12; a21 = b21; a22 = b22;
        }
        if (!id1) {  // rows: J1^H [row_p; row_q],  J1^H = [[c, -s e1], [s, c e1]]
          float2 t21 = cmul(e1, a21), t22 = cmul(e1, a22);
          float2 n11 = make_float2(R1.x * a11.x - R1.y * t21.x, R1.x * a11.y - R1.y * t21.y);
          float2 n12 = make_float2(R1.x * a12.x - R1.y * t22.x, R1.x * a12.y - R1.y * t22.y);
          float2 n21 = make_float2(R1.y * a11.x + R1.x * t21.x, R1.y * a11.y + R1.x * t21.y);
          float2 n22 = make_float2(R1.y * a12.x + R1.x * t22.x, R1.y * a12.y + R1.x * t22.y);
          a11 = n11; a12 = n12; a21 = n21; a22 = n22;
        }
        if (k1 == k2) { a12 = make_float2(0.f, 0.f); a21 = a12; a11.y = 0.f; a22.y = 0.f; }
        A[P1.x * lda + P2.x] = a11; A[P1.x * lda + P2.y] = a12;
        A[P1.y * lda + P2.x] = a21; A[P1.y * lda + P2.y] = a22;
        if (!id2) {  // V <- V J2 on rows P1 x columns P2
          float2 v11 = V[P1.x * lda + P2.x], v12 = V[P1.x * lda + P2.y];
          float2 v21 = V[P1.y * lda + P2.x], v22 = V[P1.y * lda + P2.y];
          float2 t12 = cmul(v12, e2c), t22 = cmul(v22, e2c);
          V[P1.x * lda + P2.x] = make_float2(R2.x * v11.x - R2.y * t12.x, R2.x * v11.y - R2.y * t12.y);
          V[P1.x * lda + P2.y] = make_float2(R2.y * v11.x + R2.x * t12.x, R2.y * v11.y + R2.x * t12.y);
          V[P1.y * lda + P2.x] = make_float2(R2.x * v21.x - R2.y * t22.x, R2.x * v21.y - R2.y * t22.y);
          V[P1.y * lda + P2.y] = make_float2(R2.y * v21.x + R2.x * t22.x, R2.y * v21.y + R2.x * t22.y);
        }
      }
      __syncthreads();
    }
    if (misc->flag[fs] == 0) break;
  }
}

// The same cyclic Jacobi run by one warp (the calling warp's lanes; warp barriers only), for the
// small matrices of the subspace prox (n <= 16): the rotations of a step are a handful, and the
// CTA-wide version spent most of its time in block barriers.  Call it from one whole warp with
// the CTA synchronised before and after.
template <int NPMAX>
__device__ void jacobi_warp(float2* A, float2* V, int n, float4* rot, int2* pairs, Misc* misc, int max_sweeps,
                       int lda = NPMAX + 1) {
  const int tid = threadIdx.x & 31;
  const int n2 = (n + 1) & ~1;
  const int half = n2 >> 1;
  const int M = n2 - 1;
  for (int idx = tid; idx < n2 * n2; idx += 32) {
    int i = idx / n2, j = idx - i * n2;
    V[i * lda + j] = make_float2(i == j ? 1.f : 0.f, 0.f);
  }
  float loc = 0.f;
  for (int idx = tid; idx < n * n; idx += 32) {
    int i = idx / n, j = idx - i * n;
    loc += cabs2(A[i * lda + j]);
  }
  for (int o = 16; o > 0; o >>= 1) loc += __shfl_xor_sync(0xffffffffu, loc, o);
  const float fro2 = loc;
  if (tid == 0) { misc->normF = sqrtf(fro2); misc->flag[0] = 0; misc->flag[1] = 0; }
  __syncwarp();
  const float thr = 2.4e-7f * misc->normF;
  if (n2 < 2 || !(misc->normF > 0.f)) return;

  for (int sweep = 0; sweep < max_sweeps; ++sweep) {
    const int fs = sweep & 1;
    for (int step = 0; step < M; ++step) {
      if (tid < half) {
        const int k = tid;
        int p, q;
        if (k == 0) { p = step; q = M; }
        else { p = (step + k) % M; q = (step - k + M) % M; }
        if (p > q) { int t = p; p = q; q = t; }
        float c = 1.f, s = 0.f, ex = 1.f, ey = 0.f;
        if (q < n) {
          const float app = A[p * lda + p].x, aqq = A[q * lda + q].x;
          const float2 apq = A[p * lda + q];
          const float r = hypotf(apq.x, apq.y);
          if (r > thr) {
            const float tau = (aqq - app) / (2.f * r);
            float t;
            if (fabsf(tau) > 1e15f) t = 0.5f / tau;
            else t = copysignf(1.f, tau) / (fabsf(tau) + sqrtf(1.f + tau * tau));
            c = rsqrtf(1.f + t * t);
            s = t * c;
            ex = apq.x / r; ey = apq.y / r;
            misc->flag[fs] = 1;
          }
        }
        rot[k] = make_float4(c, s, ex, ey);
        pairs[k] = make_int2(p, q);
      }
      __syncwarp();
      if (step == 0 && tid == 0) misc->flag[fs ^ 1] = 0;
      for (int b = tid; b < half * half; b += 32) {
        const int k1 = b / half, k2 = b - k1 * half;
        const int2 P1 = pairs[k1], P2 = pairs[k2];
        const float4 R1 = rot[k1], R2 = rot[k2];
        const bool id1 = (R1.y == 0.f), id2 = (R2.y == 0.f);
        if (id1 && id2) continue;
        const float2 e1 = make_float2(R1.z, R1.w);
        const float2 e2c = make_float2(R2.z, -R2.w);
        float2 a11 = A[P1.x * lda + P2.x], a12 = A[P1.x * lda + P2.y];
        float2 a21 = A[P1.y * lda + P2.x], a22 = A[P1.y * lda + P2.y];
        if (!id2) {  // columns: [x_p, x_q] J2,  J2 = [[c, s], [-s e2*, c e2*]]
          float2 t12 = cmul(a12, e2c), t22 = cmul(a22, e2c);
          float2 b11 = make_float2(R2.x * a11.x - R2.y * t12.x, R2.x * a11.y - R2.y * t12.y);
          float2 b12 = make_float2(R2.y * a11.x + R2.x * t12.x, R2.y * a11.y + R2.x * t12.y);
          float2 b21 = make_float2(R2.x * a21.x - R2.y * t22.x, R2.x * a21.y - R2.y * t22.y);
          float2 b22 = make_float2(R2.y * a21.x + R2.x * t22.x, R2.y * a21.y + R2.x * t22.y);
          a11 = b11; a12 = b12; a21 = b21; a22 = b22;
        }
        if (!id1) {  // rows: J1^H [row_p; row_q],  J1^H = [[c, -s e1], [s, c e1]]
          float2 t21 = cmul(e1, a21), t22 = cmul(e1, a22);
          float2 n11 = make_float2(R1.x * a11.x - R1.y * t21.x, R1.x * a11.y - R1.y * t21.y);
          float2 n12 = make_float2(R1.x * a12.x - R1.y * t22.x, R1.x * a12.y - R1.y * t22.y);
          float2 n21 = make_float2(R1.y * a11.x + R1.x * t21.x, R1.y * a11.y + R1.x * t21.y);
          float2 n22 = make_float2(R1.y * a12.x + R1.x * t22.x, R1.y * a12.y + R1.x * t22.y);
          a11 = n11; a12 = n12; a21 = n21; a22 = n22;
        }
        if (k1 == k2) { a12 = make_float2(0.f, 0.f); a21 = a12; a11.y = 0.f; a22.y = 0.f; }
        A[P1.x * lda + P2.x] = a11; A[P1.x * lda + P2.y] = a12;
        A[P1.y * lda + P2.x] = a21; A[P1.y * lda + P2.y] = a22;
        if (!id2) {  // V <- V J2 on rows P1 x columns P2
          float2 v11 = V[P1.x * lda + P2.x], v12 = V[P1.x * lda + P2.y];
          float2 v21 = V[P1.y * lda + P2.x], v22 = V[P1.y * lda + P2.y];
          float2 t12 = cmul(v12, e2c), t22 = cmul(v22, e2c);
          V[P1.x * lda + P2.x] = make_float2(R2.x * v11.x - R2.y * t12.x, R2.x * v11.y - R2.y * t12.y);
          V[P1.x * lda + P2.y] = make_float2(R2.y * v11.x + R2.x * t12.x, R2.y * v11.y + R2.x * t12.y);
          V[P1.y * lda + P2.x] = make_float2(R2.x * v21.x - R2.y * t22.x, R2.x * v21.y - R2.y * t22.y);
          V[P1.y * lda + P2.y] = make_float2(R2.y * v21.x + R2.x * t22.x, R2.y * v21.y + R2.x * t22.y);
        }
      }
      __syncwarp();
    }
    if (misc->flag[fs] == 0) break;
  }
}

// g(lambda) for every eigenvalue and the compacted list of active eigenvectors.
__device__ void singular_map(const float2* A, int lda, int n, int mode, int rank, float lam, float* ev, float* g,
                             int* act, Misc* misc) {
  const int tid = threadIdx.x;
  if (tid < n) ev[tid] = A[tid * lda + tid].x;
  __syncthreads();
  if (tid < n) {
    const float e = ev[tid];
    float gv;
    if (mode == LLR_PROX_HARD_RANK) {
      int pos = 0;
      for (int j = 0; j < n; ++j) {
        const float ej = ev[j];
        pos += (ej > e) || (ej == e && j < tid);
      }
      gv = pos < rank ? 1.f : 0.f;
    } else {
      const float s = sqrtf(fmaxf(e, 0.f));
      gv = (s > lam) ? (1.f - lam / s) : 0.f;
    }
    g[tid] = gv;
  }
  __syncthreads();
  if (tid == 0) {
    int c = 0;
    for (int j = 0; j < n; ++j)
      if (g[j] != 0.f) act[c++] = j;
    misc->n_active = c;
  }
  __syncthreads();
}

// Nuclear norm of a soft-thresholded block from the eigenvalues e of its Gram matrix (squared
// singular values): sum of (sqrt(e) - lambda)+ in FP64, in index order.
__device__ __forceinline__ double nuclear_from_eigs(const float* e, int k, float lam) {
  double t = 0.0;
  for (int j = 0; j < k; ++j) {
    const double sv = sqrt((double)fmaxf(e[j], 0.f));
    if (sv > (double)lam) t += sv - (double)lam;
  }
  return t;
}

// W = V diag(g) V^H written into A (lda).
__device__ void form_W(float2* A, const float2* V, int lda, int n, const float* g, const int* act, int na) {
  for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) {
    const int i = idx / n, j = idx - i * n;
    float2 s = make_float2(0.f, 0.f);
    for (int t = 0; t < na; ++t) {
      const int k = act[t];
      float2 vik = V[i * lda + k];
      float2 vjk = V[j * lda + k];
      float2 p = cmul_bc(vik, vjk);
      s.x = fmaf(g[k], p.x, s.x);
      s.y = fmaf(g[k], p.y, s.y);
    }
    A[i * lda + j] = s;
  }
  __syncthreads();
}

// C <- C W in place (row blocks processed in rounds; rows of one round depend only on
// themselves, so each round writes back after one barrier).
template <int NPMAX, int TG>
__device__ void apply_W(float2* Cs, int ldc, int m, int n, const float2* W, int lda = NPMAX + 1) {
  constexpr int RT = 4;
  const int nt = (n + TG - 1) / TG;               // column tiles (interleaved columns)
  const int row_tiles_per_round = max(1, (int)blockDim.x / nt);
  const int rows_per_round = row_tiles_per_round * RT;
  const int tid = threadIdx.x;
  const bool active = tid < row_tiles_per_round * nt;
  const int tj = tid % nt, tr = tid / nt;
  for (int r0 = 0; r0 < m; r0 += rows_per_round) {
    float2 acc[RT][TG];
#pragma unroll
    for (int a = 0; a < RT; ++a)
#pragma unroll
      for (int b = 0; b < TG; ++b) acc[a][b] = make_float2(0.f, 0.f);
    const int rb = r0 + tr * RT;
    if (active && rb < m) {
      for (int k = 0; k < n; ++k) {
        float2 c[RT], w[TG];
#pragma unroll
        for (int a = 0; a < RT; ++a) c[a] = (rb + a < m) ? Cs[k * ldc + rb + a] : make_float2(0.f, 0.f);
#pragma unroll
        for (int b = 0; b < TG; ++b) {
          const int j = tj + nt * b;
          w[b] = (j < n) ? W[k * lda + j] : make_float2(0.f, 0.f);
        }
#pragma unroll
        for (int a = 0; a < RT; ++a)
#pragma unroll
          for (int b = 0; b < TG; ++b) cfma(acc[a][b], c[a], w[b]);
      }
    }
    __syncthreads();
    if (active && rb < m) {
#pragma unroll
      for (int a = 0; a < RT; ++a)
#pragma unroll
        for (int b = 0; b < TG; ++b) {
          const int j = tj + nt * b;
          if (rb + a < m && j < n) Cs[j * ldc + rb + a] = acc[a][b];
        }
    }
  }
  __syncthreads();
}


}  // namespace
}  // namespace llr
