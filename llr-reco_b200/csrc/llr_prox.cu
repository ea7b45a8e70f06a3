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

#include "llr_internal.h"

namespace llr {

namespace {

struct SmemLayout {
  int ldc;        // leading dimension of C in shared memory (odd)
  int np;         // padded n for Gram tiles
  int ksplit;     // Gram K-split factor
  size_t off_rot, off_pair, off_ev, off_g, off_act, off_A, off_V, off_scr, off_C, off_trd, total;
};

// Tridiagonal-path scratch (NPMAX-sized vectors and the real eigenvectors of T').
template <int NPMAX>
struct TrdSmem {
  float2 u[NPMAX];      // current Householder vector
  float2 p[NPMAX];      // tau * A22 u
  float2 e[NPMAX];      // complex sub-diagonal of T
  float2 delta[NPMAX];  // unitary diagonal making T' = D^H T D real
  float d[NPMAX];       // diagonal of T
  float ae[NPMAX];      // |e|
  float e2[NPMAX];      // |e|^2
  float tau[NPMAX];     // reflector scalars
  float lam[NPMAX];     // active eigenvalues (ascending), perturbed for inverse iteration
  float Y[NPMAX * NPMAX];  // eigenvectors of T', column a at Y[a * NPMAX]
};

__host__ __device__ inline size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

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
  L.off_trd = off; off = align16(off + sizeof(TrdSmem<NPMAX>));
  L.total = off;
  return L;
}

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
}

// Voxel coordinates of row r of block `blk` (rows ordered y fastest, then z, then x:
// the contiguous axis of the planar layout).  Corner = grid index * block + shift
// (block.rs:122-133); every coordinate wraps modulo the volume (block.rs:20-22).
__device__ __forceinline__ void block_row_coord(const BlockSource& s, long long blk, const int* sh, int r,
                                                int& ix, int& iy, int& iz) {
  int gxi = (int)(blk % s.gx);
  long long t = blk / s.gx;
  int gyi = (int)(t % s.gy);
  int gzi = (int)(t / s.gy);
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
    s.data[planar_index(s.g, ix, iy, iz, q)] = v;
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
__device__ void jacobi(float2* A, float2* V, int n, float4* rot, int2* pairs, Misc* misc, int max_sweeps) {
  constexpr int lda = NPMAX + 1;
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
__device__ void apply_W(float2* Cs, int ldc, int m, int n, const float2* W) {
  constexpr int lda = NPMAX + 1;
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

// =======================================================================================
// Tridiagonal eigen path.  Householder reduction of the Hermitian Gram matrix to
// tridiagonal T (H = I - tau u u^H, tau real), a unitary diagonal D making T' = D^H T D
// real, Sturm-count multisection for only the eigenvalues that the singular-value map keeps
// (above lambda^2, or the top `rank`), inverse iteration for their eigenvectors, modified
// Gram-Schmidt plus a residual check, and back-transformation V = Q D Y.  About n^3 complex
// flops in total against sweeps * 8 n^3 for Jacobi; blocks whose eigenvectors fail the
// residual check take the Jacobi path.
// =======================================================================================
template <int NPMAX>
__device__ void hermitian_tridiag(float2* A, int n, TrdSmem<NPMAX>* T, float* red) {
  constexpr int lda = NPMAX + 1;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nwarps = blockDim.x >> 5;
  for (int k = 0; k + 2 < n; ++k) {
    const int L = n - k - 1;
    if (warp == 0) {
      const int i0 = lane, i1 = lane + 32;
      float2 x0 = make_float2(0.f, 0.f), x1 = make_float2(0.f, 0.f);
      if (i0 < L) x0 = A[(k + 1 + i0) * lda + k];
      if (i1 < L) x1 = A[(k + 1 + i1) * lda + k];
      float s2 = cabs2(x0) + cabs2(x1);
      for (int o = 16; o > 0; o >>= 1) s2 += __shfl_xor_sync(0xffffffffu, s2, o);
      const float ax = __shfl_sync(0xffffffffu, x0.x, 0), ay = __shfl_sync(0xffffffffu, x0.y, 0);
      const float xn = sqrtf(s2);
      const float aa = sqrtf(ax * ax + ay * ay);
      const float phx = aa > 0.f ? ax / aa : 1.f, phy = aa > 0.f ? ay / aa : 0.f;
      const float2 u0 = make_float2(ax + phx * xn, ay + phy * xn);
      const float un2 = s2 - aa * aa + cabs2(u0);
      const float t = (xn > 0.f && un2 > 0.f) ? 2.f / un2 : 0.f;
      if (lane == 0) {
        T->tau[k] = t;
        T->e[k] = make_float2(-phx * xn, -phy * xn);
        A[(k + 1) * lda + k] = u0;  // column k now stores u_k for the back-transformation
      }
      if (i0 < L) T->u[i0] = (i0 == 0) ? u0 : x0;
      if (i1 < L) T->u[i1] = x1;
    }
    __syncthreads();
    const float t = T->tau[k];
    if (t != 0.f) {
      // p = t * A22 u : four threads per row
      const int row = tid >> 2, part = tid & 3;
      float2 acc = make_float2(0.f, 0.f);
      if (row < L) {
        const float2* Ar = A + (k + 1 + row) * lda + (k + 1);
        for (int j = part; j < L; j += 4) cfma(acc, Ar[j], T->u[j]);
      }
      acc.x += __shfl_xor_sync(0xffffffffu, acc.x, 1);
      acc.y += __shfl_xor_sync(0xffffffffu, acc.y, 1);
      acc.x += __shfl_xor_sync(0xffffffffu, acc.x, 2);
      acc.y += __shfl_xor_sync(0xffffffffu, acc.y, 2);
      float dp = 0.f;
      if (row < L && part == 0) {
        const float2 pv = cscale(acc, t);
        T->p[row] = pv;
        const float2 uv = T->u[row];
        dp = uv.x * pv.x + uv.y * pv.y;  // Re(conj(u) p)
      }
      for (int o = 16; o > 0; o >>= 1) dp += __shfl_xor_sync(0xffffffffu, dp, o);
      if (lane == 0) red[warp] = dp;
      __syncthreads();
      float up = 0.f;
      for (int w = 0; w < nwarps; ++w) up += red[w];
      const float K = 0.5f * t * up;
      // A22 -= u w^H + w u^H,  w = p - K u
      const int tj = tid & 15, ti = tid >> 4;
      for (int i = ti; i < L; i += 16) {
        const float2 ui = T->u[i];
        const float2 wi = csub(T->p[i], cscale(ui, K));
        float2* Ar = A + (k + 1 + i) * lda + (k + 1);
        for (int j = tj; j < L; j += 16) {
          const float2 uj = T->u[j];
          const float2 wj = csub(T->p[j], cscale(uj, K));
          Ar[j] = csub(csub(Ar[j], cmul_bc(ui, wj)), cmul_bc(wi, uj));
        }
      }
    }
    __syncthreads();
  }
  if (tid < n) T->d[tid] = A[tid * lda + tid].x;
  if (tid == 0) {
    if (n >= 2) T->e[n - 2] = A[(n - 1) * lda + n - 2];
    for (int k = n - 2; k < n; ++k)
      if (k >= 0) T->tau[k] = 0.f;
  }
  __syncthreads();
}

// Sturm count: number of eigenvalues of the real tridiagonal (d, e2 = offdiag^2) below x.
__device__ __forceinline__ int sturm_count(const float* d, const float* e2, int n, float x, float pivmin) {
  float q = d[0] - x;
  if (fabsf(q) <= pivmin) q = -pivmin;
  int c = q < 0.f;
  for (int i = 1; i < n; ++i) {
    q = d[i] - x - e2[i - 1] / q;
    if (fabsf(q) <= pivmin) q = -pivmin;
    c += q < 0.f;
  }
  return c;
}

// Real form T' (D), Gershgorin interval, and the active index range (eigenvalues
// n_below .. n_below + ra - 1 in ascending order).
template <int NPMAX>
__device__ void tridiag_setup(TrdSmem<NPMAX>* T, int n, int mode, int rank, float lam, Misc* misc) {
  if (threadIdx.x == 0) {
    float2 dl = make_float2(1.f, 0.f);
    float e2max = 0.f;
    for (int k = 0; k < n; ++k) {
      T->delta[k] = dl;
      if (k + 1 < n) {
        const float2 ek = T->e[k];
        const float a = sqrtf(cabs2(ek));
        T->ae[k] = a;
        T->e2[k] = a * a;
        e2max = fmaxf(e2max, a * a);
        if (a > 0.f) dl = cmul(dl, make_float2(ek.x / a, ek.y / a));
      } else {
        T->ae[k] = 0.f;
        T->e2[k] = 0.f;
      }
    }
    float gl = 3.0e38f, gu = -3.0e38f;
    for (int k = 0; k < n; ++k) {
      const float r = (k > 0 ? T->ae[k - 1] : 0.f) + (k + 1 < n ? T->ae[k] : 0.f);
      gl = fminf(gl, T->d[k] - r);
      gu = fmaxf(gu, T->d[k] + r);
    }
    const float tn = fmaxf(fabsf(gl), fabsf(gu));
    gl -= 4.f * 1.1920929e-7f * tn * n + 1e-30f;
    gu += 4.f * 1.1920929e-7f * tn * n + 1e-30f;
    misc->gl = gl;
    misc->gu = gu;
    misc->tnorm = tn;
    misc->pivmin = 1.1754944e-38f * fmaxf(1.f, e2max);
    int nb;
    if (mode == LLR_PROX_HARD_RANK) nb = max(0, n - rank);
    else if (!(lam > 0.f)) nb = 0;
    else nb = sturm_count(T->d, T->e2, n, lam * lam, misc->pivmin);
    misc->n_below = nb;
    misc->ra = n - nb;
    misc->fail = 0;
  }
  __syncthreads();
}

// Multisection: groups of 8 lanes refine eigenvalue j by 9-way splits (warp-uniform loop).
template <int NPMAX>
__device__ void tridiag_eigenvalues(TrdSmem<NPMAX>* T, int n, int j0, int count, const Misc* misc) {
  const int lane = threadIdx.x & 31;
  const int gl8 = lane & 7;
  const int group = threadIdx.x >> 3;
  const int ngroups = blockDim.x >> 3;
  for (int base = 0; base < count; base += ngroups) {
    const int a = base + group;
    const bool act = a < count;
    const int j = j0 + (act ? a : 0);
    float lo = misc->gl, hi = misc->gu;
    for (int round = 0; round < 14; ++round) {
      const bool conv = !act || (hi - lo) <= 2.4e-7f * fmaxf(fabsf(lo), fabsf(hi)) + misc->pivmin;
      if (__all_sync(0xffffffffu, conv)) break;
      const float x = lo + (hi - lo) * (float)(gl8 + 1) * (1.f / 9.f);
      const bool le = act ? (sturm_count(T->d, T->e2, n, x, misc->pivmin) <= j) : true;
      const unsigned bal = __ballot_sync(0xffffffffu, le);
      const int nt = __popc((bal >> (lane & 24)) & 0xffu);
      const float nlo = nt > 0 ? lo + (hi - lo) * (float)nt * (1.f / 9.f) : lo;
      const float nhi = nt < 8 ? lo + (hi - lo) * (float)(nt + 1) * (1.f / 9.f) : hi;
      lo = nlo;
      hi = nhi;
    }
    if (act && gl8 == 0) T->lam[a] = 0.5f * (lo + hi);
  }
  __syncthreads();
}

// Inverse iteration (one thread per active eigenvalue) on T' - lambda I with partial
// pivoting; three solves from a deterministic start vector.
template <int NPMAX>
__device__ void tridiag_vectors(TrdSmem<NPMAX>* T, int n, int ra, Misc* misc) {
  const float eps = 1.1920929e-7f;
  const float tiny = eps * fmaxf(misc->tnorm, 1e-30f);
  if (threadIdx.x == 0) {  // separate (near-)equal eigenvalues (LAPACK stein convention)
    const float sep = 10.f * eps * fmaxf(misc->tnorm, 1e-30f);
    for (int a = 1; a < ra; ++a)
      if (T->lam[a] - T->lam[a - 1] < sep) T->lam[a] = T->lam[a - 1] + sep;
  }
  __syncthreads();
  for (int a = threadIdx.x; a < ra; a += blockDim.x) {
    const float lam = T->lam[a];
    float dd[NPMAX], du[NPMAX], du2[NPMAX], dl[NPMAX], b[NPMAX];
    unsigned long long piv = 0ull;
    for (int i = 0; i < n; ++i) {
      dd[i] = T->d[i] - lam;
      du[i] = (i + 1 < n) ? T->ae[i] : 0.f;
      dl[i] = du[i];
      du2[i] = 0.f;
    }
    for (int i = 0; i + 1 < n; ++i) {
      if (fabsf(dd[i]) >= fabsf(dl[i])) {
        if (fabsf(dd[i]) < tiny) dd[i] = copysignf(tiny, dd[i] == 0.f ? 1.f : dd[i]);
        const float f = dl[i] / dd[i];
        dl[i] = f;
        dd[i + 1] -= f * du[i];
      } else {
        const float f = dd[i] / dl[i];
        dd[i] = dl[i];
        dl[i] = f;
        const float tmp = du[i];
        du[i] = dd[i + 1];
        dd[i + 1] = tmp - f * dd[i + 1];
        if (i + 2 < n) {
          du2[i] = du[i + 1];
          du[i + 1] = -f * du[i + 1];
        }
        piv |= (1ull << i);
      }
    }
    if (fabsf(dd[n - 1]) < tiny) dd[n - 1] = copysignf(tiny, dd[n - 1] == 0.f ? 1.f : dd[n - 1]);
    uint64_t h = llr_splitmix64(0x1234567ull + (uint64_t)a);
    for (int i = 0; i < n; ++i) {
      h = llr_splitmix64(h);
      b[i] = (float)((h >> 40) & 0xffffff) * (1.f / 16777216.f) - 0.5f;
    }
    for (int it = 0; it < 3; ++it) {
      for (int i = 0; i + 1 < n; ++i) {
        if (piv & (1ull << i)) {
          const float t = b[i];
          b[i] = b[i + 1];
          b[i + 1] = t - dl[i] * b[i];
        } else {
          b[i + 1] -= dl[i] * b[i];
        }
      }
      b[n - 1] /= dd[n - 1];
      if (n >= 2) b[n - 2] = (b[n - 2] - du[n - 2] * b[n - 1]) / dd[n - 2];
      for (int i = n - 3; i >= 0; --i) b[i] = (b[i] - du[i] * b[i + 1] - du2[i] * b[i + 2]) / dd[i];
      float mx = 0.f;
      for (int i = 0; i < n; ++i) mx = fmaxf(mx, fabsf(b[i]));
      const float sc = mx > 0.f ? 1.f / mx : 1.f;
      for (int i = 0; i < n; ++i) b[i] *= sc;
    }
    for (int i = 0; i < n; ++i) T->Y[a * NPMAX + i] = b[i];
  }
  __syncthreads();
  // modified Gram-Schmidt over the active vectors + residual check (warp 0)
  if ((threadIdx.x >> 5) == 0) {
    const int lane = threadIdx.x & 31;
    const float tol = 2e-5f * fmaxf(misc->tnorm, 1e-30f);
    int bad = 0;
    for (int a = 0; a < ra; ++a) {
      float* y = T->Y + a * NPMAX;
      float y0 = lane < n ? y[lane] : 0.f, y1 = lane + 32 < n ? y[lane + 32] : 0.f;
      for (int c = 0; c < a; ++c) {
        const float* z = T->Y + c * NPMAX;
        const float z0 = lane < n ? z[lane] : 0.f, z1 = lane + 32 < n ? z[lane + 32] : 0.f;
        float dp = y0 * z0 + y1 * z1;
        for (int o = 16; o > 0; o >>= 1) dp += __shfl_xor_sync(0xffffffffu, dp, o);
        y0 -= dp * z0;
        y1 -= dp * z1;
      }
      float nn = y0 * y0 + y1 * y1;
      for (int o = 16; o > 0; o >>= 1) nn += __shfl_xor_sync(0xffffffffu, nn, o);
      const float inv = nn > 0.f ? rsqrtf(nn) : 0.f;
      y0 *= inv;
      y1 *= inv;
      if (lane < n) y[lane] = y0;
      if (lane + 32 < n) y[lane + 32] = y1;
      __syncwarp();
      // residual |T' y - lambda y|
      const float lam = T->lam[a];
      float r2 = 0.f;
      for (int h = 0; h < 2; ++h) {
        const int i = lane + 32 * h;
        if (i < n) {
          float r = (T->d[i] - lam) * y[i];
          if (i > 0) r += T->ae[i - 1] * y[i - 1];
          if (i + 1 < n) r += T->ae[i] * y[i + 1];
          r2 += r * r;
        }
      }
      for (int o = 16; o > 0; o >>= 1) r2 += __shfl_xor_sync(0xffffffffu, r2, o);
      if (!(nn > 0.f) || !(sqrtf(r2) <= tol)) bad = 1;
      __syncwarp();
    }
    if (lane == 0) misc->fail = bad;
  }
  __syncthreads();
}

// V[:, a] = Q D y_a (complex), one warp per vector.
template <int NPMAX>
__device__ void tridiag_backtransform(const float2* A, TrdSmem<NPMAX>* T, float2* V, int n, int ra) {
  constexpr int lda = NPMAX + 1;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int a = warp; a < ra; a += nw) {
    const float* y = T->Y + a * NPMAX;
    float2 v0 = make_float2(0.f, 0.f), v1 = make_float2(0.f, 0.f);
    const int i0 = lane, i1 = lane + 32;
    if (i0 < n) v0 = cscale(T->delta[i0], y[i0]);
    if (i1 < n) v1 = cscale(T->delta[i1], y[i1]);
    for (int k = n - 3; k >= 0; --k) {
      const float t = T->tau[k];
      if (t == 0.f) continue;
      // u_k lives in column k of A below the diagonal (rows k+1 .. n-1), with u_k[0] at row k+1
      // replaced by the value kept in column k during the reduction.
      const float2 u0 = (i0 > k && i0 < n) ? A[i0 * lda + k] : make_float2(0.f, 0.f);
      const float2 u1 = (i1 > k && i1 < n) ? A[i1 * lda + k] : make_float2(0.f, 0.f);
      float2 s = cadd(cmulc(u0, v0), cmulc(u1, v1));
      for (int o = 16; o > 0; o >>= 1) {
        s.x += __shfl_xor_sync(0xffffffffu, s.x, o);
        s.y += __shfl_xor_sync(0xffffffffu, s.y, o);
      }
      s = cscale(s, t);
      v0 = csub(v0, cmul(u0, s));
      v1 = csub(v1, cmul(u1, s));
    }
    if (i0 < n) V[i0 * lda + a] = v0;
    if (i1 < n) V[i1 * lda + a] = v1;
  }
  __syncthreads();
}

// C <- (C V_a) diag(g) V_a^H for ra <= RM active vectors: one thread owns whole rows, so
// rows are rewritten in place without a barrier.
template <int NPMAX, int RM>
__device__ void apply_lowrank_rows(float2* Cs, int ldc, int m, int n, const float2* V, const float* g, int ra) {
  constexpr int lda = NPMAX + 1;
  for (int r = threadIdx.x; r < m; r += blockDim.x) {
    float2 t[RM];
#pragma unroll
    for (int a = 0; a < RM; ++a) t[a] = make_float2(0.f, 0.f);
    for (int k = 0; k < n; ++k) {
      const float2 c = Cs[k * ldc + r];
#pragma unroll
      for (int a = 0; a < RM; ++a)
        if (a < ra) cfma(t[a], c, V[k * lda + a]);
    }
#pragma unroll
    for (int a = 0; a < RM; ++a)
      if (a < ra) t[a] = cscale(t[a], g[a]);
    for (int q = 0; q < n; ++q) {
      float2 c = make_float2(0.f, 0.f);
#pragma unroll
      for (int a = 0; a < RM; ++a)
        if (a < ra) cfma_cb(c, t[a], V[q * lda + a]);
      Cs[q * ldc + r] = c;
    }
  }
  __syncthreads();
}

template <int NPMAX, int TG>
__global__ void __launch_bounds__(kLlrThreads) llr_prox_kernel(BlockSource src, ProxOp op, SmemLayout L) {
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
  TrdSmem<NPMAX>* trd = reinterpret_cast<TrdSmem<NPMAX>*>(smem + L.off_trd);
  constexpr int lda = NPMAX + 1;
  const int m = op.m, n = op.n;

  if (threadIdx.x == 0) block_shift(src, misc->shift);
  __syncthreads();
  int sh[3] = {misc->shift[0], misc->shift[1], misc->shift[2]};

  for (long long blk = blockIdx.x; blk < src.nblocks; blk += gridDim.x) {
    gather_block(src, blk, sh, m, n, Cs, L.ldc);
    __syncthreads();
    gram<NPMAX, TG>(Cs, L.ldc, m, n, A, scr, L.ksplit);
    bool use_jacobi = op.eig_solver == 1;
    if (!use_jacobi) {
      hermitian_tridiag<NPMAX>(A, n, trd, misc->red);
      if (op.block_stat) {
        tridiag_setup<NPMAX>(trd, n, LLR_PROX_HARD_RANK, 1, 0.f, misc);
        tridiag_eigenvalues<NPMAX>(trd, n, n - 1, 1, misc);
        if (threadIdx.x == 0) op.block_stat[blk] = trd->lam[0];
        __syncthreads();
        continue;
      }
      tridiag_setup<NPMAX>(trd, n, op.mode, op.rank, op.lambda, misc);
      const int ra = misc->ra, nb = misc->n_below;
      if (ra == n && op.mode == LLR_PROX_HARD_RANK) {
        // rank >= n: identity
      } else if (ra == 0) {
        for (int i = threadIdx.x; i < n * L.ldc; i += blockDim.x) Cs[i] = make_float2(0.f, 0.f);
        __syncthreads();
      } else {
        tridiag_eigenvalues<NPMAX>(trd, n, nb, ra, misc);
        tridiag_vectors<NPMAX>(trd, n, ra, misc);
        if (misc->fail) {
          use_jacobi = true;
          gram<NPMAX, TG>(Cs, L.ldc, m, n, A, scr, L.ksplit);
        } else {
          tridiag_backtransform<NPMAX>(A, trd, V, n, ra);
          if (threadIdx.x < ra) {
            float gv = 1.f;
            if (op.mode != LLR_PROX_HARD_RANK) {
              const float sv = sqrtf(fmaxf(trd->lam[threadIdx.x], 0.f));
              gv = (sv > op.lambda) ? (1.f - op.lambda / sv) : 0.f;
            }
            g[threadIdx.x] = gv;
            act[threadIdx.x] = threadIdx.x;
          }
          __syncthreads();
          if (ra <= 8) {
            apply_lowrank_rows<NPMAX, 8>(Cs, L.ldc, m, n, V, g, ra);
          } else {
            form_W(A, V, lda, n, g, act, ra);
            apply_W<NPMAX, TG>(Cs, L.ldc, m, n, A);
          }
        }
      }
    }
    if (use_jacobi) {
      jacobi<NPMAX>(A, V, n, rot, pairs, misc, 16);
      if (op.block_stat) {
        if (threadIdx.x == 0) {
          float mx = 0.f;
          for (int i = 0; i < n; ++i) mx = fmaxf(mx, A[i * lda + i].x);
          op.block_stat[blk] = mx;
        }
        __syncthreads();
        continue;
      }
      singular_map(A, lda, n, op.mode, op.rank, op.lambda, ev, g, act, misc);
      const int na = misc->n_active;
      if (!(na == n && op.mode == LLR_PROX_HARD_RANK)) {
        form_W(A, V, lda, n, g, act, na);
        apply_W<NPMAX, TG>(Cs, L.ldc, m, n, A);
      }
    }
    scatter_block(src, blk, sh, m, n, Cs, L.ldc);
    __syncthreads();
  }
}

template <int NPMAX, int TG>
int launch_instance(const BlockSource& src, const ProxOp& op, cudaStream_t stream) {
  SmemLayout L = make_layout<NPMAX, TG>(op.m, op.n);
  if (L.total > 227 * 1024)
    return set_error(LLR_ERR_UNSUPPORTED, "Casorati %dx%d needs %zu B of shared memory (max 232448)", op.m, op.n,
                     L.total);
  auto kern = llr_prox_kernel<NPMAX, TG>;
  LLR_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.total));
  int dev = 0, nsm = 0, occ = 0;
  LLR_CUDA_TRY(cudaGetDevice(&dev));
  LLR_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  LLR_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kLlrThreads, L.total));
  if (occ < 1) return set_error(LLR_ERR_UNSUPPORTED, "prox kernel cannot be resident (smem %zu B)", L.total);
  long long grid = std::min<long long>(src.nblocks, (long long)nsm * occ);
  if (grid < 1) return LLR_OK;
  kern<<<(unsigned)grid, kLlrThreads, L.total, stream>>>(src, op, L);
  LLR_CUDA_TRY(cudaGetLastError());
  return LLR_OK;
}

}  // namespace

bool llr_prox_supported(int m, int n) {
  if (m < 1 || n < 1 || n > 64) return false;
  size_t t;
  if (n <= 16) t = make_layout<16, 2>(m, n).total;
  else if (n <= 32) t = make_layout<32, 2>(m, n).total;
  else t = make_layout<64, 4>(m, n).total;
  return t <= 227 * 1024;
}

int launch_llr_prox(const BlockSource& src, const ProxOp& op, cudaStream_t stream) {
  if (op.n < 1 || op.m < 1) return set_error(LLR_ERR_INVALID, "empty Casorati matrix %dx%d", op.m, op.n);
  if (src.nblocks == 0) return LLR_OK;
  if (op.n <= 16) return launch_instance<16, 2>(src, op, stream);
  if (op.n <= 32) return launch_instance<32, 2>(src, op, stream);
  if (op.n <= 64) return launch_instance<64, 4>(src, op, stream);
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

template <int NPMAX>
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
      float2 z[kSubMax];
#pragma unroll
      for (int k = 0; k < kSubMax; ++k) z[k] = make_float2(0.f, 0.f);
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
        for (int k = 0; k < kSubMax; ++k)
          if (k < sr) cfma(z[k], v, Ss[q * sr + k]);
      }
#pragma unroll
      for (int k = 0; k < kSubMax; ++k)
        if (k < sr) Z[k * L.ldc + r] = z[k];
    }
    __syncthreads();
    gram<NPMAX, 2>(Z, L.ldc, m, sr, A, scr, L.ksplit);
    jacobi<NPMAX>(A, V, sr, rot, pairs, misc, 16);
    singular_map(A, lda, sr, op.mode, op.rank, op.lambda, ev, g, act, misc);
    form_W(A, V, lda, sr, g, act, misc->n_active);
    apply_W<NPMAX, 2>(Z, L.ldc, m, sr, A);
    // X'[r, q] = sum_k Z'[r, k] conj(S[q, k])
    for (int r = threadIdx.x; r < m; r += blockDim.x) {
      float2 z[kSubMax];
#pragma unroll
      for (int k = 0; k < kSubMax; ++k) z[k] = (k < sr) ? Z[k * L.ldc + r] : make_float2(0.f, 0.f);
      int ix = 0, iy = 0, iz = 0;
      if (src.kind == 1) block_row_coord(src, blk, sh, r, ix, iy, iz);
      for (int q = 0; q < nq; ++q) {
        float2 v = make_float2(0.f, 0.f);
#pragma unroll
        for (int k = 0; k < kSubMax; ++k)
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

}  // namespace

int launch_llr_prox_subspace(const BlockSource& src, const SubspaceOp& op, cudaStream_t stream) {
  if (op.srank < 1 || op.srank > kSubMax)
    return set_error(LLR_ERR_UNSUPPORTED, "subspace rank %d outside [1, %d]", op.srank, kSubMax);
  if (src.nblocks == 0) return LLR_OK;
  SmemLayout L = make_layout<16, 2>(op.m, op.srank);
  L.total = align16(L.total + sizeof(float2) * (size_t)op.nq * op.srank);
  if (L.total > 227 * 1024) return set_error(LLR_ERR_UNSUPPORTED, "subspace prox needs %zu B smem", L.total);
  auto kern = llr_subspace_kernel<16>;
  LLR_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.total));
  int dev = 0, nsm = 0, occ = 0;
  LLR_CUDA_TRY(cudaGetDevice(&dev));
  LLR_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  LLR_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kLlrThreads, L.total));
  if (occ < 1) return set_error(LLR_ERR_UNSUPPORTED, "subspace kernel cannot be resident");
  long long grid = std::min<long long>(src.nblocks, (long long)nsm * occ);
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
  lift_kernel<<<(unsigned)blocks, 256, 0, s>>>(vol, mat, vs[0], vs[1], vs[2], nq, bs[0], bs[1], bs[2], g[0], g[1],
                                               sh[0], sh[1], sh[2], start, n, dir);
  LLR_CUDA_TRY(cudaGetLastError());
  return LLR_OK;
}

// =======================================================================================
// rhsCdgmmBatched (kernels.cu:11-67) and a batched complex GEMM with the semantics of
// cublas_cgemm_strided_batched_device (cublas.rs:12-105).
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
  conj_transpose_kernel<<<grid, dim3(32, 8), 0, s>>>(in, out, m, n);
  LLR_CUDA_TRY(cudaGetLastError());
  return LLR_OK;
}

int launch_rhs_cdgmm(int m, int n, int batch, float2* a, const float* d, cudaStream_t s) {
  const long long tot = (long long)m * n * batch;
  if (tot == 0) return LLR_OK;
  long long blocks = std::min<long long>((tot + 255) / 256, 148LL * 32);
  rhs_cdgmm_kernel<<<(unsigned)blocks, 256, 0, s>>>(m, n, batch, a, d);
  LLR_CUDA_TRY(cudaGetLastError());
  return LLR_OK;
}

int launch_cgemm(int m, int k, int n, int batch, int broadcast_a, float2 alpha, float2 beta, int ta, int tb,
                 const float2* A, const float2* B, float2* C, cudaStream_t s) {
  if (m == 0 || n == 0 || batch == 0) return LLR_OK;
  dim3 grid((m + 15) / 16, (n + 15) / 16, batch);
  dim3 block(16, 16);
  cgemm_kernel<<<grid, block, 0, s>>>(m, k, n, broadcast_a, alpha, beta, ta, tb, A, B, C);
  LLR_CUDA_TRY(cudaGetLastError());
  return LLR_OK;
}

}  // namespace llr
