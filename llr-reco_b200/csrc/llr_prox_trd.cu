// Fused locally-low-rank proximal step, tridiagonal eigen path (the default solver).
//
// One CTA owns one Casorati matrix at a time (persistent grid, two CTAs per SM):
//   row tables (periodic wrap, block.rs:122-133 and :20-22; per-row phase)
//   Gram G = C^H C over row chunks staged in shared memory, tiles accumulated in registers
//   Householder tridiagonalisation, Sturm multisection for the kept eigenvalues only,
//   inverse iteration, modified Gram-Schmidt + residual check, back-transformation
//   C' = (C V_a) g V_a^H, one thread per row, read from and written to global memory
// This replaces, per block, lift_data_set (block.rs:147-164), cusolver gesvda
// (cusolver.rs:20-151), rhsCdgmmBatched (kernels.cu:11-67), the CGEMM (U S) V^H
// (low_rank.rs:55) and un_lift_data_set (block.rs:166-184), since U_r S_r V_r^H = C V_r V_r^H.
// Blocks keeping more than kRaMax components, or whose eigenvectors fail the residual check,
// are appended to a device list and finished by the Jacobi kernel (llr_prox.cu).
#include <cstdio>
#include <algorithm>

#include "llr_prox_common.cuh"

namespace llr {

int launch_llr_prox_jacobi(const BlockSource& src, const ProxOp& op, cudaStream_t stream);
bool llr_prox_jacobi_supported(int m, int n);

namespace {

constexpr int kRaMax = 16;   // kept components handled by the tridiagonal path

// Tridiagonal-path scratch (NPMAX-sized vectors and the real eigenvectors of T').
template <int NPMAX>
struct TrdSmem {
  float2 u[2][NPMAX];   // Householder vector of the current step and x of the next one
  float2 p[NPMAX];      // tau * A22 u
  float2 e[NPMAX];      // complex sub-diagonal of T
  float2 delta[NPMAX];  // unitary diagonal making T' = D^H T D real
  float d[NPMAX];       // diagonal of T
  float ae[NPMAX];      // |e|
  float e2[NPMAX];      // |e|^2
  float tau[NPMAX];     // reflector scalars
  float nrm[16];        // partial squared norms of the next column
  float lam[kRaMax];    // kept eigenvalues (ascending), separated for the vector solve
  float Y[NPMAX * kRaMax];  // eigenvectors of T', column a at Y[a * NPMAX]
};

// Element (i, j), j <= i, of the Gram matrix in shared memory: full row-major storage with
// leading dimension NPMAX + 1, or packed lower triangle i(i+1)/2 + j.
template <int NPMAX, bool PACKED>
struct AIdx {
  __device__ __forceinline__ static int at(int i, int j) {
    return PACKED ? (i * (i + 1)) / 2 + j : i * (NPMAX + 1) + j;
  }
};

__device__ __forceinline__ float warp_sum(float v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// =======================================================================================
// Tridiagonal eigen path.  Householder reduction of the Hermitian Gram matrix to
// tridiagonal T (H = I - tau u u^H, tau real) working on the lower triangle only, a
// unitary diagonal D making T' = D^H T D real, Sturm-count multisection for only the
// eigenvalues that the singular-value map keeps (above lambda^2, or the top `rank`),
// eigenvectors of T' from a twisted factorisation (stationary and progressive qd
// recurrences, twist index at the smallest |gamma|), modified Gram-Schmidt plus a residual
// check, and back-transformation V = Q D Y.  About n^3 complex flops in total against
// sweeps * 8 n^3 for Jacobi; blocks whose eigenvectors fail the residual check go to the
// Jacobi kernel.
// =======================================================================================
template <int NPMAX, bool PACKED>
__device__ void hermitian_tridiag(float2* A, int n, TrdSmem<NPMAX>* T, float* red) {
  typedef AIdx<NPMAX, PACKED> I;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nwarps = blockDim.x >> 5;
  const int tj = tid & 15, ti = tid >> 4, TI = blockDim.x >> 4;   // 16-wide update grid
  const int tpr = blockDim.x >> 6;                                  // matvec threads per row
  if (n >= 3) {  // vector and norm of column 0; later columns come from the previous update
    if (warp == 0) {
      float s2 = 0.f;
      for (int i = lane; i < n - 1; i += 32) {
        const float2 x = A[I::at(1 + i, 0)];
        s2 += cabs2(x);
        T->u[0][i] = x;
      }
      s2 = warp_sum(s2);
      if (lane < 16) T->nrm[lane] = lane == 0 ? s2 : 0.f;
    }
    __syncthreads();
  }
  for (int k = 0; k + 2 < n; ++k) {
    const int L = n - k - 1;
    const int cur = k & 1, nxt = cur ^ 1;
    float2* U = T->u[cur];
    const int o = k + 1;   // A22 starts at (o, o)
    if (tid == 0) {
      float s2 = 0.f;
      for (int i = 0; i < 16; ++i) { s2 += T->nrm[i]; T->nrm[i] = 0.f; }
      const float2 x0 = A[I::at(o, k)];
      const float xn = sqrtf(s2);
      const float aa = sqrtf(cabs2(x0));
      const float phx = aa > 0.f ? x0.x / aa : 1.f, phy = aa > 0.f ? x0.y / aa : 0.f;
      const float2 u0 = make_float2(x0.x + phx * xn, x0.y + phy * xn);
      const float un2 = s2 - aa * aa + cabs2(u0);
      const float t = (xn > 0.f && un2 > 0.f) ? 2.f / un2 : 0.f;
      T->tau[k] = t;
      T->e[k] = make_float2(-phx * xn, -phy * xn);
      A[I::at(o, k)] = u0;  // column k keeps u_k for the back-transformation
      U[0] = u0;
    }
    __syncthreads();
    const float t = T->tau[k];
    if (t != 0.f) {
      // p = t * A22 u from the lower triangle (A22[i][j] = conj(A22[j][i]) for j > i)
      const int row = tid / tpr, part = tid - row * tpr;
      float2 acc = make_float2(0.f, 0.f);
      if (row < L) {
        for (int j = part; j < L; j += tpr) {
          const float2 a = (j <= row) ? A[I::at(o + row, o + j)] : cconj(A[I::at(o + j, o + row)]);
          cfma(acc, a, U[j]);
        }
      }
      for (int sft = 1; sft < tpr; sft <<= 1) {
        acc.x += __shfl_xor_sync(0xffffffffu, acc.x, sft);
        acc.y += __shfl_xor_sync(0xffffffffu, acc.y, sft);
      }
      float dp = 0.f;
      if (row < L && part == 0) {
        const float2 pv = cscale(acc, t);
        T->p[row] = pv;
        const float2 uv = U[row];
        dp = uv.x * pv.x + uv.y * pv.y;  // Re(conj(u) p)
      }
      dp = warp_sum(dp);
      if (lane == 0) red[warp] = dp;
      __syncthreads();
      float up = 0.f;
      for (int w = 0; w < nwarps; ++w) up += red[w];
      const float K = 0.5f * t * up;
      // lower-triangle update A22 -= u w^H + w u^H,  w = p - K u; the threads of column 0
      // also hand the next step its x vector and the partial norms.
      float nacc = 0.f;
      for (int i = ti; i < L; i += TI) {
        const float2 ui = U[i];
        const float2 wi = csub(T->p[i], cscale(ui, K));
        const int rb = I::at(o + i, o);
        for (int j = tj; j <= i; j += 16) {
          const float2 uj = U[j];
          const float2 wj = csub(T->p[j], cscale(uj, K));
          const float2 a = csub(csub(A[rb + j], cmul_bc(ui, wj)), cmul_bc(wi, uj));
          A[rb + j] = a;
          if (j == 0 && i >= 1) {
            T->u[nxt][i - 1] = a;
            nacc += cabs2(a);
          }
        }
      }
      if (tj == 0) T->nrm[ti] = nacc;
    } else {
      if (warp == 0) {  // no reflection: column k+1 is unchanged
        float s2 = 0.f;
        for (int i = lane; i < L - 1; i += 32) {
          const float2 x = A[I::at(o + 1 + i, o)];
          s2 += cabs2(x);
          T->u[nxt][i] = x;
        }
        s2 = warp_sum(s2);
        if (lane == 0) T->nrm[0] = s2;
      }
    }
    __syncthreads();
  }
  if (tid < n) T->d[tid] = A[I::at(tid, tid)].x;
  if (tid == 0) {
    if (n >= 2) T->e[n - 2] = A[I::at(n - 1, n - 2)];
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
    q = d[i] - x - e2[i - 1] * __frcp_rn(q);
    if (fabsf(q) <= pivmin) q = -pivmin;
    c += q < 0.f;
  }
  return c;
}

// Real form T' (D as a prefix product of unit phases), Gershgorin interval and the kept
// index range (eigenvalues n_below .. n - 1 in ascending order); warp 0 only.
template <int NPMAX>
__device__ void tridiag_setup(TrdSmem<NPMAX>* T, int n, int mode, int rank, float lam, Misc* misc) {
  if ((threadIdx.x >> 5) == 0) {
    const int lane = threadIdx.x & 31;
    float2 ph[2];
    float e2m = 0.f;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int k = 2 * lane + h;
      ph[h] = make_float2(1.f, 0.f);
      if (k + 1 < n) {
        const float2 ek = T->e[k];
        const float a = sqrtf(cabs2(ek));
        T->ae[k] = a;
        T->e2[k] = a * a;
        e2m = fmaxf(e2m, a * a);
        if (a > 0.f) ph[h] = make_float2(ek.x / a, ek.y / a);
      } else if (k < n) {
        T->ae[k] = 0.f;
        T->e2[k] = 0.f;
      }
    }
    // exclusive prefix product: delta_k = prod_{i<k} ph_i (complex products commute)
    float2 pr = cmul(ph[0], ph[1]);
    for (int o = 1; o < 32; o <<= 1) {
      const float ox = __shfl_up_sync(0xffffffffu, pr.x, o), oy = __shfl_up_sync(0xffffffffu, pr.y, o);
      if (lane >= o) pr = cmul(make_float2(ox, oy), pr);
    }
    float ex = __shfl_up_sync(0xffffffffu, pr.x, 1), ey = __shfl_up_sync(0xffffffffu, pr.y, 1);
    if (lane == 0) { ex = 1.f; ey = 0.f; }
    const float2 excl = make_float2(ex, ey);
    if (2 * lane < n) T->delta[2 * lane] = excl;
    if (2 * lane + 1 < n) T->delta[2 * lane + 1] = cmul(excl, ph[0]);
    __syncwarp();
    float gl = 3.0e38f, gu = -3.0e38f;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int k = 2 * lane + h;
      if (k < n) {
        const float r = (k > 0 ? T->ae[k - 1] : 0.f) + (k + 1 < n ? T->ae[k] : 0.f);
        gl = fminf(gl, T->d[k] - r);
        gu = fmaxf(gu, T->d[k] + r);
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      gl = fminf(gl, __shfl_xor_sync(0xffffffffu, gl, o));
      gu = fmaxf(gu, __shfl_xor_sync(0xffffffffu, gu, o));
      e2m = fmaxf(e2m, __shfl_xor_sync(0xffffffffu, e2m, o));
    }
    if (lane == 0) {
      const float tn = fmaxf(fabsf(gl), fabsf(gu));
      gl -= 4.f * 1.1920929e-7f * tn * n + 1e-30f;
      gu += 4.f * 1.1920929e-7f * tn * n + 1e-30f;
      misc->gl = gl;
      misc->gu = gu;
      misc->tnorm = tn;
      misc->pivmin = 1.1754944e-38f * fmaxf(1.f, e2m);
      int nb;
      if (mode == LLR_PROX_HARD_RANK) nb = max(0, n - rank);
      else if (!(lam > 0.f)) nb = 0;
      else nb = sturm_count(T->d, T->e2, n, lam * lam, misc->pivmin);
      misc->n_below = nb;
      misc->ra = n - nb;
      misc->fail = 0;
    }
  }
  __syncthreads();
}

// Multisection: a group of G lanes (G = 32, 16 or 8 by the number of eigenvalues) refines
// eigenvalue j by (G+1)-way splits of its Gershgorin interval; warp-uniform loop.
template <int NPMAX>
__device__ void tridiag_eigenvalues(TrdSmem<NPMAX>* T, int n, int j0, int count, const Misc* misc) {
  const int lane = threadIdx.x & 31;
  const int G = count <= (int)(blockDim.x >> 5) ? 32 : (count <= (int)(blockDim.x >> 4) ? 16 : 8);
  const int gl = lane & (G - 1);
  const int group = threadIdx.x / G;
  const int ngroups = blockDim.x / G;
  const unsigned gmask = G == 32 ? 0xffffffffu : ((1u << G) - 1u);
  const float inv = 1.f / (float)(G + 1);
  for (int base = 0; base < count; base += ngroups) {
    const int a = base + group;
    const bool act = a < count;
    const int j = j0 + (act ? a : 0);
    float lo = misc->gl, hi = misc->gu;
    for (int round = 0; round < 24; ++round) {
      const bool conv = !act || (hi - lo) <= 2.4e-7f * fmaxf(fabsf(lo), fabsf(hi)) + misc->pivmin;
      if (__all_sync(0xffffffffu, conv)) break;
      const float x = lo + (hi - lo) * (float)(gl + 1) * inv;
      const bool le = act ? (sturm_count(T->d, T->e2, n, x, misc->pivmin) <= j) : true;
      const unsigned bal = __ballot_sync(0xffffffffu, le);
      const int nt = __popc((bal >> (lane & ~(G - 1) & 31)) & gmask);
      const float nlo = nt > 0 ? lo + (hi - lo) * (float)nt * inv : lo;
      const float nhi = nt < G ? lo + (hi - lo) * (float)(nt + 1) * inv : hi;
      lo = nlo;
      hi = nhi;
    }
    if (act && gl == 0) T->lam[a] = 0.5f * (lo + hi);
  }
  __syncthreads();
}

// Eigenvectors of T' (one thread per kept eigenvalue) from the twisted factorisation
// T' - lam I = L+ D+ L+^T = U- D- U-^T; the twist r minimises |gamma_r|, z_r = 1 and the
// two bidiagonal recurrences fill the rest.  `work` holds 2 * NPMAX * kRaMax floats.
template <int NPMAX>
__device__ void tridiag_vectors(TrdSmem<NPMAX>* T, int n, int ra, Misc* misc, float* work) {
  const float eps = 1.1920929e-7f;
  const float tiny = eps * fmaxf(misc->tnorm, 1e-30f);
  if (threadIdx.x == 0) {  // separate (near-)equal eigenvalues
    const float sep = 10.f * eps * fmaxf(misc->tnorm, 1e-30f);
    for (int a = 1; a < ra; ++a)
      if (T->lam[a] - T->lam[a - 1] < sep) T->lam[a] = T->lam[a - 1] + sep;
  }
  __syncthreads();
  for (int a = threadIdx.x; a < ra; a += blockDim.x) {
    const float lam = T->lam[a];
    float* Lp = work + a;                    // stride kRaMax
    float* Dp = work + NPMAX * kRaMax + a;   // D+ then reused for U-
    float dp = T->d[0] - lam;
    for (int i = 0; i + 1 < n; ++i) {
      if (fabsf(dp) < tiny) dp = copysignf(tiny, dp);
      Dp[i * kRaMax] = dp;
      const float l = T->ae[i] * __frcp_rn(dp);
      Lp[i * kRaMax] = l;
      dp = T->d[i + 1] - lam - l * T->ae[i];
    }
    if (fabsf(dp) < tiny) dp = copysignf(tiny, dp);
    float dm = T->d[n - 1] - lam;
    float best = fabsf(dp);  // gamma_{n-1} = D+_{n-1}
    int r = n - 1;
    for (int i = n - 2; i >= 0; --i) {
      if (fabsf(dm) < tiny) dm = copysignf(tiny, dm);
      const float um = T->ae[i] * __frcp_rn(dm);
      const float dpi = Dp[i * kRaMax];
      Dp[i * kRaMax] = um;                   // U-_i overwrites D+_i (no longer needed)
      dm = T->d[i] - lam - um * T->ae[i];
      const float gamma = dpi + dm - (T->d[i] - lam);
      if (fabsf(gamma) < best) { best = fabsf(gamma); r = i; }
    }
    float* y = T->Y + a * NPMAX;
    float z = 1.f;
    y[r] = 1.f;
    for (int i = r - 1; i >= 0; --i) { z = -Lp[i * kRaMax] * z; y[i] = z; }
    z = 1.f;
    for (int i = r; i + 1 < n; ++i) { z = -Dp[i * kRaMax] * z; y[i + 1] = z; }
    float mx = 0.f;
    for (int i = 0; i < n; ++i) mx = fmaxf(mx, fabsf(y[i]));
    const float sc = (mx > 0.f && mx < 3.0e38f) ? 1.f / mx : 0.f;
    for (int i = 0; i < n; ++i) y[i] *= sc;
  }
  __syncthreads();
  // modified Gram-Schmidt over the kept vectors + residual check (warp 0)
  if ((threadIdx.x >> 5) == 0) {
    const int lane = threadIdx.x & 31;
    const float tol = 2e-5f * fmaxf(misc->tnorm, 1e-30f);
    int bad = 0;
    for (int a = 0; a < ra; ++a) {
      float* y = T->Y + a * NPMAX;
      float y0 = lane < n ? y[lane] : 0.f, y1 = lane + 32 < n ? y[lane + 32] : 0.f;
      for (int c = 0; c < a; ++c) {
        const float* zc = T->Y + c * NPMAX;
        const float z0 = lane < n ? zc[lane] : 0.f, z1 = lane + 32 < n ? zc[lane + 32] : 0.f;
        const float dpr = warp_sum(y0 * z0 + y1 * z1);
        y0 -= dpr * z0;
        y1 -= dpr * z1;
      }
      const float nn = warp_sum(y0 * y0 + y1 * y1);
      const float inv = nn > 0.f ? rsqrtf(nn) : 0.f;
      y0 *= inv;
      y1 *= inv;
      if (lane < n) y[lane] = y0;
      if (lane + 32 < n) y[lane + 32] = y1;
      __syncwarp();
      const float lam = T->lam[a];
      float r2 = 0.f;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int i = lane + 32 * h;
        if (i < n) {
          float rr = (T->d[i] - lam) * y[i];
          if (i > 0) rr += T->ae[i - 1] * y[i - 1];
          if (i + 1 < n) rr += T->ae[i] * y[i + 1];
          r2 += rr * rr;
        }
      }
      r2 = warp_sum(r2);
      if (!(nn > 0.f) || !(sqrtf(r2) <= tol)) bad = 1;
      __syncwarp();
    }
    if (lane == 0) misc->fail = bad;
  }
  __syncthreads();
}

// Va[i * kRaMax + a] = (Q D y_a)_i (complex), one warp per vector.
template <int NPMAX, bool PACKED>
__device__ void tridiag_backtransform(const float2* A, TrdSmem<NPMAX>* T, float2* V, int n, int ra) {
  typedef AIdx<NPMAX, PACKED> I;
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
      const float2 u0 = (i0 > k && i0 < n) ? A[I::at(i0, k)] : make_float2(0.f, 0.f);
      const float2 u1 = (i1 > k && i1 < n) ? A[I::at(i1, k)] : make_float2(0.f, 0.f);
      float2 sv = cadd(cmulc(u0, v0), cmulc(u1, v1));
      sv.x = warp_sum(sv.x);
      sv.y = warp_sum(sv.y);
      sv = cscale(sv, t);
      v0 = csub(v0, cmul(u0, sv));
      v1 = csub(v1, cmul(u1, sv));
    }
    if (i0 < n) V[i0 * kRaMax + a] = v0;
    if (i1 < n) V[i1 * kRaMax + a] = v1;
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------------------
// Per-block row tables: element (r, q) of the Casorati matrix lives at off[r] + q * qstride,
// and (for per-row uniform phase) carries phase ph[r].
// ---------------------------------------------------------------------------------------
struct RowTab {
  int off;   // planar offset of the voxel (volume 0) or row index (matrix batches)
  int cx;    // x coordinate
  int cyz;   // y | z << 16
  int pad;
};

// KB raw loads of row r (volumes k0 .. k0 + KB - 1) with nothing between them, then the phase
// correction: the loads are all in flight before the first use (a per-element branch between
// them would serialise the round trips).
template <int KB>
__device__ __forceinline__ void load_row_batch(const BlockSource& s, long long base, const RowTab& rt,
                                               const float2* rowph, int r, int k0, int n, long long qstride,
                                               float2 (&c)[KB]) {
  const float2* rowp = s.data + base + (long long)rt.off;
#pragma unroll
  for (int u = 0; u < KB; ++u)
    c[u] = (k0 + u < n) ? rowp[(long long)(k0 + u) * qstride] : make_float2(0.f, 0.f);
  if (s.kind == 1) {
    if (s.ph_uniform) {
      const float2 p = rowph[r];
#pragma unroll
      for (int u = 0; u < KB; ++u) c[u] = cscale(cmul_bc(c[u], p), s.load_scale);
    } else {
#pragma unroll
      for (int u = 0; u < KB; ++u)
        if (k0 + u < n)
          c[u] = cscale(cmul_bc(c[u], phase_at(s.ph, s.g, k0 + u, rt.cx, rt.cyz & 0xffff, rt.cyz >> 16)),
                        s.load_scale);
    }
  }
}

__device__ __forceinline__ void store_elem(const BlockSource& s, long long base, const RowTab& rt, const float2* rowph,
                                           int r, int q, long long qstride, float2 v) {
  if (s.kind == 1) {
    v = cscale(v, s.store_scale);
    if (s.store_phase) {
      float2 p;
      if (s.ph_uniform) p = rowph[r];
      else p = phase_at(s.ph, s.g, q, rt.cx, rt.cyz & 0xffff, rt.cyz >> 16);
      v = cmul(v, p);
    }
  }
  float2* dst = (s.out ? s.out : s.data) + base + (long long)rt.off + (long long)q * qstride;
  if (s.accumulate) v = cadd(v, *dst);
  *dst = v;
}

// Identity result of a block written to a separate output: every element loaded (with the
// load transform) and stored (with the store transform).
__device__ void copy_rows(const BlockSource& s, long long base, const RowTab* rows, const float2* rowph, int m, int n,
                          long long qstride) {
  for (int r = threadIdx.x; r < m; r += blockDim.x) {
    const RowTab rt = rows[r];
    for (int k0 = 0; k0 < n; k0 += 8) {
      float2 c[8];
      load_row_batch<8>(s, base, rt, rowph, r, k0, n, qstride, c);
#pragma unroll
      for (int u = 0; u < 8; ++u)
        if (k0 + u < n) store_elem(s, base, rt, rowph, r, k0 + u, qstride, c[u]);
    }
  }
}

struct TrdLayout {
  int rc;        // rows per staged chunk
  int ldch;      // leading dimension of a staged chunk (odd)
  int np, ksplit;
  size_t off_row, off_rowph, off_A, off_C, off_trd, off_V, off_g, total;
};

template <int NPMAX, int TG>
TrdLayout make_trd_layout(int m, int n) {
  TrdLayout L;
  const int nt = (n + TG - 1) / TG;
  L.np = nt * TG;
  L.ksplit = std::max(1, kLlrThreads / (nt * nt));
  int rc = (40 * 1024) / (8 * n);
  rc = std::max(32, std::min(rc, 256));
  L.rc = std::min(rc, m);
  L.ldch = (L.rc & 1) ? L.rc : L.rc + 1;
  size_t off = 256;
  L.off_row = off; off = align16(off + sizeof(RowTab) * (size_t)m);
  L.off_rowph = off; off = align16(off + sizeof(float2) * (size_t)m);
  L.off_A = off; off = align16(off + sizeof(float2) * NPMAX * (NPMAX + 1));
  L.off_C = off;
  const size_t chunk = sizeof(float2) * (size_t)n * L.ldch;
  const size_t scr = L.ksplit > 1 ? sizeof(float2) * (size_t)L.ksplit * L.np * L.np : 0;
  const size_t vec = sizeof(float) * 2 * NPMAX * kRaMax;   // twisted-factorisation work
  off = align16(off + std::max(std::max(chunk, scr), vec));
  L.off_trd = off; off = align16(off + sizeof(TrdSmem<NPMAX>));
  L.off_V = off; off = align16(off + sizeof(float2) * NPMAX * kRaMax);
  L.off_g = off; off = align16(off + sizeof(float) * kRaMax);
  L.total = off;
  return L;
}

template <int RM, int LDV = kRaMax>
__device__ void apply_rows(const BlockSource& s, long long base, const RowTab* rows, const float2* rowph, int m, int n,
                           long long qstride, const float2* Va, const float* g, int ra) {
  constexpr int KB = 8;   // loads in flight per thread
  for (int r = threadIdx.x; r < m; r += blockDim.x) {
    const RowTab rt = rows[r];
    float2 t[RM];
#pragma unroll
    for (int a = 0; a < RM; ++a) t[a] = make_float2(0.f, 0.f);
    for (int k0 = 0; k0 < n; k0 += KB) {
      float2 c[KB];
      load_row_batch<KB>(s, base, rt, rowph, r, k0, n, qstride, c);
#pragma unroll
      for (int u = 0; u < KB; ++u) {
        if (k0 + u < n) {
#pragma unroll
          for (int a = 0; a < RM; ++a)
            if (a < ra) cfma(t[a], c[u], Va[(k0 + u) * LDV + a]);
        }
      }
    }
#pragma unroll
    for (int a = 0; a < RM; ++a)
      if (a < ra) t[a] = cscale(t[a], g[a]);
    for (int q = 0; q < n; ++q) {
      float2 c = make_float2(0.f, 0.f);
#pragma unroll
      for (int a = 0; a < RM; ++a)
        if (a < ra) cfma_cb(c, t[a], Va[q * LDV + a]);
      store_elem(s, base, rt, rowph, r, q, qstride, c);
    }
  }
}

// Row tables of block `blk`, then its Gram matrix over staged row chunks (tile accumulators
// in registers); every lower-or-upper element (i, j) < n is handed to sink(i, j, value).
template <int NPMAX, int TG, class Sink>
__device__ void gram_block(const BlockSource& src, const TrdLayout& L, int m, int n, long long blk,
                           long long base, long long qstride, const int* sh, RowTab* rows, float2* rowph,
                           float2* Cch, Sink sink) {
  const int tid = threadIdx.x;
    // row tables
    for (int r = tid; r < m; r += blockDim.x) {
      RowTab rt;
      if (src.kind == 1) {
        int ix, iy, iz;
        block_row_coord(src, blk, sh, r, ix, iy, iz);
        rt.off = (int)planar_index(src.g, ix, iy, iz, 0);
        rt.cx = ix;
        rt.cyz = iy | (iz << 16);
        if (src.ph_uniform) rowph[r] = phase_at(src.ph, src.g, 0, ix, iy, iz);
      } else {
        rt.off = r;
        rt.cx = 0;
        rt.cyz = 0;
      }
      rt.pad = 0;
      rows[r] = rt;
    }
    // Gram over staged row chunks; tile accumulators stay in registers
    const int nt = (n + TG - 1) / TG;
    const int tiles = nt * nt;
    const bool gram_thread = tid < tiles * L.ksplit;
    const int tile = tid % tiles, ks = tid / tiles;
    const int ti = tile / nt, tj = tile - ti * nt;
    float2 acc[TG][TG];
#pragma unroll
    for (int a = 0; a < TG; ++a)
#pragma unroll
      for (int b = 0; b < TG; ++b) acc[a][b] = make_float2(0.f, 0.f);
    __syncthreads();
    for (int c0 = 0; c0 < m; c0 += L.rc) {
      const int rc = min(L.rc, m - c0);
      {
        constexpr int GB = 8;   // loads in flight per thread
        const int tot = rc * n;
        int q = tid / rc, rr = tid - (tid / rc) * rc;
        const int sq = blockDim.x / rc, sr = blockDim.x - sq * rc;
        for (int i0 = tid; i0 < tot; i0 += GB * blockDim.x) {
          float2 v[GB];
          int dq[GB], dr[GB];
#pragma unroll
          for (int u = 0; u < GB; ++u) {
            dq[u] = q;
            dr[u] = rr;
            if (i0 + u * (int)blockDim.x < tot) {
              const RowTab rt = rows[c0 + rr];
              v[u] = src.data[base + (long long)rt.off + (long long)q * qstride];
            }
            rr += sr;
            q += sq;
            if (rr >= rc) { rr -= rc; ++q; }
          }
#pragma unroll
          for (int u = 0; u < GB; ++u) {
            if (i0 + u * (int)blockDim.x < tot) {
              const int r = c0 + dr[u];
              float2 x = v[u];
              if (src.kind == 1) {
                float2 p;
                if (src.ph_uniform) p = rowph[r];
                else {
                  const RowTab rt = rows[r];
                  p = phase_at(src.ph, src.g, dq[u], rt.cx, rt.cyz & 0xffff, rt.cyz >> 16);
                }
                x = cscale(cmul_bc(x, p), src.load_scale);
              }
              Cch[dq[u] * L.ldch + dr[u]] = x;
            }
          }
        }
      }
      __syncthreads();
      if (gram_thread) {
        const int r0 = (int)(((long long)rc * ks) / L.ksplit), r1 = (int)(((long long)rc * (ks + 1)) / L.ksplit);
        for (int r = r0; r < r1; ++r) {
          float2 ci[TG], cj[TG];
#pragma unroll
          for (int a = 0; a < TG; ++a) {
            const int cI = ti + nt * a, cJ = tj + nt * a;
            ci[a] = cI < n ? Cch[cI * L.ldch + r] : make_float2(0.f, 0.f);
            cj[a] = cJ < n ? Cch[cJ * L.ldch + r] : make_float2(0.f, 0.f);
          }
#pragma unroll
          for (int a = 0; a < TG; ++a)
#pragma unroll
            for (int b = 0; b < TG; ++b) cfma_ca(acc[a][b], ci[a], cj[b]);
        }
      }
      __syncthreads();
    }
    if (L.ksplit == 1) {
      if (gram_thread) {
#pragma unroll
        for (int a = 0; a < TG; ++a)
#pragma unroll
          for (int b = 0; b < TG; ++b) {
            const int cI = ti + nt * a, cJ = tj + nt * b;
            if (cI < n && cJ < n) sink(cI, cJ, acc[a][b]);
          }
      }
    } else {
      float2* P = Cch;  // chunk buffer is free now
      if (gram_thread) {
#pragma unroll
        for (int a = 0; a < TG; ++a)
#pragma unroll
          for (int b = 0; b < TG; ++b)
            P[(size_t)ks * L.np * L.np + (ti + nt * a) * L.np + (tj + nt * b)] = acc[a][b];
      }
      __syncthreads();
      for (int idx = tid; idx < n * n; idx += blockDim.x) {
        const int i = idx / n, j = idx - i * n;
        float2 sacc = make_float2(0.f, 0.f);
        for (int k = 0; k < L.ksplit; ++k) sacc = cadd(sacc, P[(size_t)k * L.np * L.np + i * L.np + j]);
        sink(i, j, sacc);
      }
    }
    __syncthreads();
}

template <int NPMAX, int TG>
__global__ void __launch_bounds__(kLlrThreads, 2) llr_prox_trd_kernel(BlockSource src, ProxOp op, TrdLayout L) {
  extern __shared__ __align__(16) unsigned char smem[];
  Misc* misc = reinterpret_cast<Misc*>(smem);
  RowTab* rows = reinterpret_cast<RowTab*>(smem + L.off_row);
  float2* rowph = reinterpret_cast<float2*>(smem + L.off_rowph);
  float2* A = reinterpret_cast<float2*>(smem + L.off_A);
  float2* Cch = reinterpret_cast<float2*>(smem + L.off_C);
  TrdSmem<NPMAX>* trd = reinterpret_cast<TrdSmem<NPMAX>*>(smem + L.off_trd);
  float2* Va = reinterpret_cast<float2*>(smem + L.off_V);
  float* g = reinterpret_cast<float*>(smem + L.off_g);
  constexpr int lda = NPMAX + 1;
  const int m = op.m, n = op.n, tid = threadIdx.x;
  const long long qstride = src.kind == 1 ? src.g.V : (long long)m;

  if (tid == 0) block_shift(src, misc->shift);
  __syncthreads();
  const int sh[3] = {misc->shift[0], misc->shift[1], misc->shift[2]};

  for (long long blk = blockIdx.x; blk < src.nblocks; blk += gridDim.x) {
    const long long base = src.kind == 1 ? 0 : blk * (long long)m * n;
    gram_block<NPMAX, TG>(src, L, m, n, blk, base, qstride, sh, rows, rowph, Cch,
                          [&](int i, int j, float2 v) { A[i * lda + j] = v; });

    hermitian_tridiag<NPMAX, false>(A, n, trd, misc->red);
    if (op.block_stat) {
      tridiag_setup<NPMAX>(trd, n, LLR_PROX_HARD_RANK, 1, 0.f, misc);
      tridiag_eigenvalues<NPMAX>(trd, n, n - 1, 1, misc);
      if (tid == 0) op.block_stat[blk] = trd->lam[0];
      __syncthreads();
      continue;
    }
    tridiag_setup<NPMAX>(trd, n, op.mode, op.rank, op.lambda, misc);
    const int ra = misc->ra, nb = misc->n_below;
    if (ra == n && op.mode == LLR_PROX_HARD_RANK) {   // rank >= n: identity
      if (src.out) copy_rows(src, base, rows, rowph, m, n, qstride);
      __syncthreads();
      continue;
    }
    if (ra == 0) {
      if (!src.accumulate)
        for (int idx = tid; idx < m * n; idx += blockDim.x) {
          const int q = idx / m, r = idx - q * m;
          store_elem(src, base, rows[r], rowph, r, q, qstride, make_float2(0.f, 0.f));
        }
      __syncthreads();
      continue;
    }
    bool fallback = ra > kRaMax;
    if (!fallback) {
      tridiag_eigenvalues<NPMAX>(trd, n, nb, ra, misc);
      tridiag_vectors<NPMAX>(trd, n, ra, misc, reinterpret_cast<float*>(Cch));
      fallback = misc->fail != 0;
    }
    if (fallback) {
      if (tid == 0 && op.fb_list) {
        const int pos = atomicAdd(op.fb_count, 1);
        op.fb_list[pos] = (int)blk;
      }
      __syncthreads();
      continue;
    }
    tridiag_backtransform<NPMAX, false>(A, trd, Va, n, ra);
    if (tid < ra) {
      float gv = 1.f;
      if (op.mode != LLR_PROX_HARD_RANK) {
        const float sv = sqrtf(fmaxf(trd->lam[tid], 0.f));
        gv = (sv > op.lambda) ? (1.f - op.lambda / sv) : 0.f;
      }
      g[tid] = gv;
    }
    if (op.blk_nuc && op.mode != LLR_PROX_HARD_RANK && tid == 0)
      op.blk_nuc[blk] = nuclear_from_eigs(trd->lam, ra, op.lambda);
    __syncthreads();
    if (ra <= 4) apply_rows<4>(src, base, rows, rowph, m, n, qstride, Va, g, ra);
    else if (ra <= 8) apply_rows<8>(src, base, rows, rowph, m, n, qstride, Va, g, ra);
    else apply_rows<kRaMax>(src, base, rows, rowph, m, n, qstride, Va, g, ra);
    __syncthreads();
  }
}

template <int NPMAX, int TG>
int launch_trd_instance(const BlockSource& src, const ProxOp& op, cudaStream_t stream) {
  TrdLayout L = make_trd_layout<NPMAX, TG>(op.m, op.n);
  if (L.total > 227 * 1024)
    return set_error(LLR_ERR_UNSUPPORTED, "Casorati %dx%d needs %zu B of shared memory", op.m, op.n, L.total);
  auto kern = llr_prox_trd_kernel<NPMAX, TG>;
  LLR_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.total));
    LLR_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
  int dev = 0, nsm = 0, occ = 0;
  LLR_CUDA_TRY(cudaGetDevice(&dev));
  LLR_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  LLR_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kLlrThreads, L.total));
  if (occ < 1) return set_error(LLR_ERR_UNSUPPORTED, "prox kernel cannot be resident (smem %zu B)", L.total);
  const long long grid = std::min<long long>(src.nblocks, (long long)nsm * occ);
  if (grid < 1) return LLR_OK;
  note_launch();
  kern<<<(unsigned)grid, kLlrThreads, L.total, stream>>>(src, op, L);
  LLR_CUDA_TRY(cudaGetLastError());
  return LLR_OK;
}

// =======================================================================================
// Split path.  A Gram kernel (llr_gram_tc_kernel on the tensor cores, or llr_gram_kernel in
// FP32 FMA) writes every block's Gram matrix (packed lower triangle, n(n+1)/2 complex) to a
// scratch buffer; the warp eigen kernel turns it into the kept eigenvectors and the apply
// kernel forms C' = (C V_a) g V_a^H from global to global.
// =======================================================================================
template <int NPMAX, int TG>
__global__ void __launch_bounds__(kLlrThreads, 2) llr_gram_kernel(BlockSource src, ProxOp op, TrdLayout L) {
  extern __shared__ __align__(16) unsigned char smem[];
  Misc* misc = reinterpret_cast<Misc*>(smem);
  RowTab* rows = reinterpret_cast<RowTab*>(smem + L.off_row);
  float2* rowph = reinterpret_cast<float2*>(smem + L.off_rowph);
  float2* Cch = reinterpret_cast<float2*>(smem + L.off_C);
  const int m = op.m, n = op.n;
  const long long qstride = src.kind == 1 ? src.g.V : (long long)m;
  if (threadIdx.x == 0) block_shift(src, misc->shift);
  __syncthreads();
  const int sh[3] = {misc->shift[0], misc->shift[1], misc->shift[2]};
  for (long long blk = blockIdx.x; blk < src.nblocks; blk += gridDim.x) {
    const long long base = src.kind == 1 ? 0 : blk * (long long)m * n;
    float2* G = op.gram + blk * op.gram_stride;
    gram_block<NPMAX, TG>(src, L, m, n, blk, base, qstride, sh, rows, rowph, Cch, [&](int i, int j, float2 v) {
      if (j <= i) G[(i * (i + 1)) / 2 + j] = v;
    });
  }
}

// Soft-threshold apply with the refinement sweep: t_a = C v_a for the thread's (at most two)
// rows, sigma_a^2 = ||C v_a||^2 / ||v_a||^2 summed over the block in FP64 (no Gram: the
// conditioning is not squared), g_a = max(1 - lambda / sigma_a, 0), then C' = sum_a t_a g_a v_a^H.
template <int RM>
__device__ void apply_rows_refined(const BlockSource& s, long long base, const RowTab* rows, const float2* rowph,
                                   int m, int n, long long qstride, const float2* Va, float* g, int ra, float lam,
                                   double* red, double* nucs, double* nuc_out) {
  constexpr int KB = 8;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
  float2 t[2][RM];
  double mu[RM];
#pragma unroll
  for (int a = 0; a < RM; ++a) mu[a] = 0.0;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int r = tid + h * blockDim.x;
#pragma unroll
    for (int a = 0; a < RM; ++a) t[h][a] = make_float2(0.f, 0.f);
    if (r < m) {
      const RowTab rt = rows[r];
      for (int k0 = 0; k0 < n; k0 += KB) {
        float2 c[KB];
        load_row_batch<KB>(s, base, rt, rowph, r, k0, n, qstride, c);
#pragma unroll
        for (int u = 0; u < KB; ++u) {
          if (k0 + u < n) {
#pragma unroll
            for (int a = 0; a < RM; ++a)
              if (a < ra) cfma(t[h][a], c[u], Va[(k0 + u) * kFacCols + a]);
          }
        }
      }
#pragma unroll
      for (int a = 0; a < RM; ++a) mu[a] += (double)t[h][a].x * t[h][a].x + (double)t[h][a].y * t[h][a].y;
    }
  }
#pragma unroll
  for (int a = 0; a < RM; ++a) {
    for (int o = 16; o > 0; o >>= 1) mu[a] += __shfl_xor_sync(0xffffffffu, mu[a], o);
    if (lane == 0) red[warp * RM + a] = mu[a];
  }
  __syncthreads();
  if (tid < ra) {
    double sum = 0.0, vn = 0.0;
    for (int w = 0; w < nw; ++w) sum += red[w * RM + tid];
    for (int q = 0; q < n; ++q) {
      const float2 v = Va[q * kFacCols + tid];
      vn += (double)v.x * v.x + (double)v.y * v.y;
    }
    const double sig = vn > 0.0 ? sqrt(sum / vn) : 0.0;
    g[tid] = sig > (double)lam ? (float)(1.0 - (double)lam / sig) : 0.f;
    nucs[tid] = sig > (double)lam ? sig - (double)lam : 0.0;
  }
  __syncthreads();
  if (nuc_out && tid == 0) {   // the block's nuclear norm after the threshold, columns in order
    double t = 0.0;
    for (int a = 0; a < ra; ++a) t += nucs[a];
    *nuc_out = t;
  }
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int r = tid + h * blockDim.x;
    if (r >= m) continue;
    const RowTab rt = rows[r];
#pragma unroll
    for (int a = 0; a < RM; ++a) t[h][a] = cscale(t[h][a], a < ra ? g[a] : 0.f);
    for (int q = 0; q < n; ++q) {
      float2 c = make_float2(0.f, 0.f);
#pragma unroll
      for (int a = 0; a < RM; ++a)
        if (a < ra) cfma_cb(c, t[h][a], Va[q * kFacCols + a]);
      store_elem(s, base, rt, rowph, r, q, qstride, c);
    }
  }
}

// C' = (C V_a) diag(g) V_a^H for the blocks whose eigen factor the warp eigen kernel wrote
// (r_a > 0), zero for r_a = 0; r_a = -1 (Jacobi fallback) and -2 (identity) are left alone.
// One CTA per block, one thread per row with eight loads in flight.
constexpr int kApplyThreads = 256;

struct ApplyLayout {
  size_t off_row, off_rowph, off_V, off_g, off_red, off_nuc, total;
};

inline ApplyLayout make_apply_layout(int m, int n) {
  ApplyLayout L;
  size_t off = 64;
  L.off_row = off; off = align16(off + sizeof(RowTab) * (size_t)m);
  L.off_rowph = off; off = align16(off + sizeof(float2) * (size_t)m);
  L.off_V = off; off = align16(off + sizeof(float2) * (size_t)n * kFacCols);
  L.off_g = off; off = align16(off + sizeof(float) * kFacCols);
  L.off_red = off; off = align16(off + sizeof(double) * (kApplyThreads / 32) * kFacCols);
  L.off_nuc = off; off = align16(off + sizeof(double) * kFacCols);
  L.total = off;
  return L;
}

__global__ void __launch_bounds__(kApplyThreads, 3) llr_apply_kernel(BlockSource src, ProxOp op, ApplyLayout L) {
  extern __shared__ __align__(16) unsigned char smem[];
  int* sh_s = reinterpret_cast<int*>(smem);
  RowTab* rows = reinterpret_cast<RowTab*>(smem + L.off_row);
  float2* rowph = reinterpret_cast<float2*>(smem + L.off_rowph);
  float2* Va = reinterpret_cast<float2*>(smem + L.off_V);
  float* g = reinterpret_cast<float*>(smem + L.off_g);
  double* red = reinterpret_cast<double*>(smem + L.off_red);
  double* nucs = reinterpret_cast<double*>(smem + L.off_nuc);
  const int m = op.m, n = op.n, tid = threadIdx.x;
  const long long qstride = src.kind == 1 ? src.g.V : (long long)m;
  // soft threshold: gains from ||C v||^2 (FP64 sum) when the block's rows fit two per thread
  const bool refine = op.mode != LLR_PROX_HARD_RANK && m <= 2 * (int)blockDim.x;
  if (tid == 0) block_shift(src, sh_s);
  __syncthreads();
  const int sh[3] = {sh_s[0], sh_s[1], sh_s[2]};
  for (long long blk = blockIdx.x; blk < src.nblocks; blk += gridDim.x) {
    const int ra = op.blk_ra[blk];
    // uniform over the CTA: fallback blocks (-1) belong to the Jacobi kernel; identity blocks (-2)
    // stay in place unless the result goes to a separate output; zero blocks need no store when
    // deferred to the fused FFT or accumulated
    if (ra == -1 || (ra == -2 && !src.out) || (ra == 0 && (op.defer_zero || src.accumulate))) continue;
    const long long base = src.kind == 1 ? 0 : blk * (long long)m * n;
    for (int r = tid; r < m; r += blockDim.x) {
      RowTab rt;
      if (src.kind == 1) {
        int ix, iy, iz;
        block_row_coord(src, blk, sh, r, ix, iy, iz);
        rt.off = (int)planar_index(src.g, ix, iy, iz, 0);
        rt.cx = ix;
        rt.cyz = iy | (iz << 16);
        if (src.ph_uniform) rowph[r] = phase_at(src.ph, src.g, 0, ix, iy, iz);
      } else {
        rt.off = r;
        rt.cx = 0;
        rt.cyz = 0;
      }
      rt.pad = 0;
      rows[r] = rt;
    }
    if (ra > 0) {
      const float2* F = op.gram + blk * op.gram_stride;
      for (int i = tid; i < n * kFacCols; i += blockDim.x) Va[i] = F[i];
      if (tid < kFacCols) g[tid] = F[n * kFacCols + tid].x;
    }
    __syncthreads();
    if (ra > 0 && !refine && op.blk_nuc && op.mode != LLR_PROX_HARD_RANK && tid == 0) {
      // unrefined gains g = 1 - lambda / s: s - lambda = lambda g / (1 - g)
      double t = 0.0;
      for (int a = 0; a < ra; ++a)
        if (g[a] > 0.f) t += (double)op.lambda * g[a] / (1.0 - (double)g[a]);
      op.blk_nuc[blk] = t;
    }
    if (ra == -2) {
      copy_rows(src, base, rows, rowph, m, n, qstride);
    } else if (ra == 0) {   // every singular value below the threshold: the block becomes zero
      for (int r = tid; r < m; r += blockDim.x) {
        float2* rowp = (src.out ? src.out : src.data) + base + (long long)rows[r].off;
        for (int q = 0; q < n; ++q) rowp[(long long)q * qstride] = make_float2(0.f, 0.f);
      }
    } else if (refine) {
      double* nuc = op.blk_nuc ? op.blk_nuc + blk : nullptr;
      if (ra <= 2) apply_rows_refined<2>(src, base, rows, rowph, m, n, qstride, Va, g, ra, op.lambda, red, nucs, nuc);
      else if (ra <= 4)
        apply_rows_refined<4>(src, base, rows, rowph, m, n, qstride, Va, g, ra, op.lambda, red, nucs, nuc);
      else apply_rows_refined<kFacCols>(src, base, rows, rowph, m, n, qstride, Va, g, ra, op.lambda, red, nucs, nuc);
    } else if (ra <= 2) {
      apply_rows<2, kFacCols>(src, base, rows, rowph, m, n, qstride, Va, g, ra);
    } else if (ra <= 4) {
      apply_rows<4, kFacCols>(src, base, rows, rowph, m, n, qstride, Va, g, ra);
    } else {
      apply_rows<kFacCols, kFacCols>(src, base, rows, rowph, m, n, qstride, Va, g, ra);
    }
    __syncthreads();
  }
}

// =======================================================================================
// Casorati matrices with 64 < n <= 128 columns that the split path cannot finish (more kept
// components than the warp eigen kernel holds, or a failed residual check), and every block
// at that width for the Jacobi solver and the block statistics: Gram matrix over staged row
// chunks into shared memory, cyclic Jacobi with the eigenvectors in a per-CTA global scratch
// (L2-resident), W = V diag(g) V^H, C' = C W streamed over row chunks.  One CTA per SM.
// =======================================================================================
constexpr int kWideTG = 8;
constexpr int kWideRows = 32;

struct WideLayout {
  TrdLayout t;     // rc / ldch / ksplit / np and the row-table offsets for gram_block
  int lda;         // leading dimension of A (and V) = n + 1
  int v_smem;      // 1: eigenvectors in shared memory (off_V); 0: in the per-CTA global scratch
  size_t off_rot, off_pair, off_ev, off_g, off_act, off_A, off_V, total;
};

// The eigenvectors stay in shared memory when A and V both fit beside the row tables and the
// row chunk (n <= 108 for 512-row blocks); wider matrices keep them in the global scratch.
inline WideLayout make_wide_layout(int m, int n) {
  WideLayout W;
  TrdLayout& L = W.t;
  const int nt = (n + kWideTG - 1) / kWideTG;
  L.np = nt * kWideTG;
  L.ksplit = 1;
  L.rc = std::min(kWideRows, m);
  L.ldch = (L.rc & 1) ? L.rc : L.rc + 1;
  const int np2 = (n + 1) & ~1;   // Jacobi pairs up an even count: an odd n gets one zero row / column
  W.lda = np2 + 1;
  size_t off = 256;   // Misc
  W.off_rot = off; off = align16(off + sizeof(float4) * (kProxMaxN / 2));
  W.off_pair = off; off = align16(off + sizeof(int2) * (kProxMaxN / 2));
  W.off_ev = off; off = align16(off + sizeof(float) * kProxMaxN);
  W.off_g = off; off = align16(off + sizeof(float) * kProxMaxN);
  W.off_act = off; off = align16(off + sizeof(int) * kProxMaxN);
  L.off_row = off; off = align16(off + sizeof(RowTab) * (size_t)m);
  L.off_rowph = off; off = align16(off + sizeof(float2) * (size_t)m);
  W.off_A = off; off = align16(off + sizeof(float2) * (size_t)np2 * W.lda);
  L.off_C = off; off = align16(off + sizeof(float2) * (size_t)n * L.ldch);
  const size_t vbytes = sizeof(float2) * (size_t)np2 * W.lda;
  W.v_smem = off + vbytes <= 227 * 1024 ? 1 : 0;
  W.off_V = off;
  if (W.v_smem) off = align16(off + vbytes);
  L.total = W.total = off;
  return W;
}

__global__ void __launch_bounds__(kLlrThreads, 1) llr_prox_wide_kernel(BlockSource src, ProxOp op, WideLayout W) {
  constexpr int NP = kProxMaxN;
  const int lda = W.lda;
  extern __shared__ __align__(16) unsigned char smem[];
  Misc* misc = reinterpret_cast<Misc*>(smem);
  float4* rot = reinterpret_cast<float4*>(smem + W.off_rot);
  int2* pairs = reinterpret_cast<int2*>(smem + W.off_pair);
  float* ev = reinterpret_cast<float*>(smem + W.off_ev);
  float* g = reinterpret_cast<float*>(smem + W.off_g);
  int* act = reinterpret_cast<int*>(smem + W.off_act);
  RowTab* rows = reinterpret_cast<RowTab*>(smem + W.t.off_row);
  float2* rowph = reinterpret_cast<float2*>(smem + W.t.off_rowph);
  float2* A = reinterpret_cast<float2*>(smem + W.off_A);
  float2* Cch = reinterpret_cast<float2*>(smem + W.t.off_C);
  float2* V = W.v_smem ? reinterpret_cast<float2*>(smem + W.off_V) : op.vwide + (long long)blockIdx.x * wide_v_stride();
  const int m = op.m, n = op.n, tid = threadIdx.x;
  const long long qstride = src.kind == 1 ? src.g.V : (long long)m;
  if (tid == 0) block_shift(src, misc->shift);
  __syncthreads();
  const int sh[3] = {misc->shift[0], misc->shift[1], misc->shift[2]};
  const long long count = src.blk_list ? (long long)*src.blk_count : src.nblocks;
  for (long long i = blockIdx.x; i < count; i += gridDim.x) {
    const long long blk = src.blk_list ? (long long)src.blk_list[i] : i;
    const long long base = src.kind == 1 ? 0 : blk * (long long)m * n;
    for (int k = tid; k < ((n + 1) & ~1) * lda; k += blockDim.x) A[k] = make_float2(0.f, 0.f);
    gram_block<NP, kWideTG>(src, W.t, m, n, blk, base, qstride, sh, rows, rowph, Cch,
                            [&](int a, int b, float2 v) { A[a * lda + b] = v; });
    if (!op.block_stat && op.mode != LLR_PROX_HARD_RANK && op.lambda > 0.f) {
      // ||G||_F <= lambda^2, or the trace bound lambda_max <= m + s sqrt(n - 1) (m = tr G / n,
      // s^2 = ||G||_F^2 / n - m^2; Wolkowicz & Styan 1980) <= lambda^2, puts every eigenvalue of
      // G = C^H C below the threshold: the output is zero, as the Jacobi path would make it (no kept
      // component, W = 0), without the sweeps
      __syncthreads();
      float loc = 0.f, tr = 0.f;
      for (int k = tid; k < n * n; k += blockDim.x) {
        const int a = k / n, b = k - a * n;
        loc += cabs2(A[a * lda + b]);
        if (a == b) tr += A[a * lda + b].x;
      }
      const float fro2 = block_sum(loc, misc->red);
      const float trace = block_sum(tr, misc->red);
      const float thr = op.lambda * op.lambda;
      const double mu = (double)trace / n;
      const double ub = mu + sqrt(fmax((double)fro2 / n - mu * mu, 0.0)) * sqrt((double)(n > 1 ? n - 1 : 1));
      if (fro2 <= thr * thr || ub <= (double)thr) {
        if (!src.accumulate)
          for (int e = tid; e < m * n; e += blockDim.x) {
            const int q = e / m, r = e - q * m;
            store_elem(src, base, rows[r], rowph, r, q, qstride, make_float2(0.f, 0.f));
          }
        __syncthreads();
        continue;
      }
    }
    jacobi<NP>(A, V, n, rot, pairs, misc, 20, lda);
    if (op.block_stat) {
      if (tid == 0) {
        float mx = 0.f;
        for (int k = 0; k < n; ++k) mx = fmaxf(mx, A[k * lda + k].x);
        op.block_stat[blk] = mx;
      }
      __syncthreads();
      continue;
    }
    singular_map(A, lda, n, op.mode, op.rank, op.lambda, ev, g, act, misc);
    if (op.blk_nuc && op.mode != LLR_PROX_HARD_RANK && tid == 0) op.blk_nuc[blk] = nuclear_from_eigs(ev, n, op.lambda);
    const int na = misc->n_active;
    const bool identity = na == n && op.mode == LLR_PROX_HARD_RANK;
    if (identity && !src.out) {
      __syncthreads();
      continue;
    }
    if (na == 0 && src.accumulate) {
      __syncthreads();
      continue;
    }
    if (!identity) form_W(A, V, lda, n, g, act, na);
    for (int c0 = 0; c0 < m; c0 += W.t.rc) {
      const int rc = min(W.t.rc, m - c0);
      for (int e = tid; e < rc * n; e += blockDim.x) {
        const int q = e / rc, rr = e - q * rc, r = c0 + rr;
        const RowTab rt = rows[r];
        float2 x = src.data[base + (long long)rt.off + (long long)q * qstride];
        if (src.kind == 1) {
          const float2 p = src.ph_uniform ? rowph[r] : phase_at(src.ph, src.g, q, rt.cx, rt.cyz & 0xffff, rt.cyz >> 16);
          x = cscale(cmul_bc(x, p), src.load_scale);
        }
        Cch[q * W.t.ldch + rr] = x;
      }
      __syncthreads();
      if (!identity) apply_W<NP, kWideTG>(Cch, W.t.ldch, rc, n, A, lda);
      for (int e = tid; e < rc * n; e += blockDim.x) {
        const int q = e / rc, rr = e - q * rc, r = c0 + rr;
        store_elem(src, base, rows[r], rowph, r, q, qstride, Cch[q * W.t.ldch + rr]);
      }
      __syncthreads();
    }
  }
}

int launch_prox_wide(const BlockSource& src, const ProxOp& op, cudaStream_t stream) {
  if (!op.vwide || op.vwide_ctas < 1) return set_error(LLR_ERR_INVALID, "wide prox needs its eigenvector scratch");
  const WideLayout W = make_wide_layout(op.m, op.n);
  if (W.total > 227 * 1024)
    return set_error(LLR_ERR_UNSUPPORTED, "Casorati %dx%d needs %zu B of shared memory", op.m, op.n, W.total);
  LLR_CUDA_TRY(cudaFuncSetAttribute(llr_prox_wide_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)W.total));
  const long long grid = std::min<long long>(src.blk_list ? op.vwide_ctas : src.nblocks, op.vwide_ctas);
  if (grid < 1) return LLR_OK;
  note_launch();
  llr_prox_wide_kernel<<<(unsigned)grid, kLlrThreads, W.total, stream>>>(src, op, W);
  LLR_CUDA_TRY(cudaGetLastError());
  return LLR_OK;
}

int launch_apply(const BlockSource& src, const ProxOp& op, cudaStream_t stream) {
  const ApplyLayout L = make_apply_layout(op.m, op.n);
  if (L.total > 227 * 1024) return set_error(LLR_ERR_UNSUPPORTED, "apply kernel needs %zu B smem", L.total);
  LLR_CUDA_TRY(cudaFuncSetAttribute(llr_apply_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.total));
  // shared memory for up to eight resident CTAs (the thread limit; registers allow three); the
  // rest of the SM's memory stays L1
  const int carve = (int)std::min<size_t>(100, (8 * (L.total + 1024) * 100) / (228 * 1024) + 1);
  LLR_CUDA_TRY(cudaFuncSetAttribute(llr_apply_kernel, cudaFuncAttributePreferredSharedMemoryCarveout, carve));
  const long long grid = std::min<long long>(src.nblocks, 1ll << 30);
  note_launch();
  llr_apply_kernel<<<(unsigned)grid, kApplyThreads, L.total, stream>>>(src, op, L);
  LLR_CUDA_TRY(cudaGetLastError());
  return LLR_OK;
}

template <int NPMAX, int TG>
int launch_split_instance(const BlockSource& src, const ProxOp& op, cudaStream_t stream) {
  int dev = 0, nsm = 0, occ = 0;
  LLR_CUDA_TRY(cudaGetDevice(&dev));
  LLR_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  if (op.gram_mode == 0 && llr_gram_tc_supported(op.m, op.n)) {
    LLR_TRY(launch_llr_gram_tc(src, op, stream));
  } else {
    // the Gram kernel uses the row tables and the chunk buffer only
    TrdLayout L = make_trd_layout<NPMAX, TG>(op.m, op.n);
    const size_t chunk = sizeof(float2) * (size_t)op.n * L.ldch;
    const size_t scr = L.ksplit > 1 ? sizeof(float2) * (size_t)L.ksplit * L.np * L.np : 0;
    L.off_C = L.off_A;
    L.total = align16(L.off_C + std::max(chunk, scr));
    auto kern = llr_gram_kernel<NPMAX, TG>;
    LLR_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.total));
    LLR_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    LLR_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kLlrThreads, L.total));
    if (occ < 1) return set_error(LLR_ERR_UNSUPPORTED, "Gram kernel cannot be resident (smem %zu B)", L.total);
    const long long grid = std::min<long long>(src.nblocks, (long long)nsm * occ);
    note_launch();
    kern<<<(unsigned)grid, kLlrThreads, L.total, stream>>>(src, op, L);
    LLR_CUDA_TRY(cudaGetLastError());
  }
  LLR_TRY(launch_llr_eig_warp(op, src.nblocks, stream));
  return launch_apply(src, op, stream);
}

}  // namespace

int wide_jacobi_ctas() {
  int dev = 0, nsm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return 148;
  return nsm;
}

bool prox_needs_wide_fallback(int m, int n) { return n >= 1 && n <= 64 && !llr_prox_jacobi_supported(m, n); }

bool llr_prox_supported(int m, int n) {
  if (n > 64 && n <= kProxMaxN && m >= 1 && m <= 65535) return make_wide_layout(m, n).total <= 227 * 1024;
  if (m < 1 || n < 1 || n > 64 || m > 65535) return false;
  size_t t;
  if (n <= 16) t = make_trd_layout<16, 2>(m, n).total;
  else if (n <= 32) t = make_trd_layout<32, 2>(m, n).total;
  else t = make_trd_layout<64, 4>(m, n).total;
  // the blocks the tridiagonal path hands back go to the Jacobi kernel when a whole block fits in
  // shared memory, else to the wide kernel, which streams row chunks
  return t <= 227 * 1024 && (llr_prox_jacobi_supported(m, n) || make_wide_layout(m, n).total <= 227 * 1024);
}

// Tridiagonal-path prox over every block, then the Jacobi kernel over the blocks it handed
// back (more than kRaMax kept components, or eigenvectors failing the residual check).
int launch_llr_prox(const BlockSource& src, const ProxOp& op, cudaStream_t stream) {
  if (op.n < 1 || op.m < 1) return set_error(LLR_ERR_INVALID, "empty Casorati matrix %dx%d", op.m, op.n);
  if (src.nblocks == 0) return LLR_OK;
  if (op.n > 64) {   // wide matrices (64 < n <= 128): the wide Jacobi kernel over every block
    if (op.n > kProxMaxN)
      return set_error(LLR_ERR_UNSUPPORTED, "Casorati column count %d > %d is not supported", op.n, kProxMaxN);
    if (!op.vwide)
      return set_error(LLR_ERR_UNSUPPORTED, "Casorati column count %d > 64 needs the wide-kernel scratch of a "
                                            "context or of an allocating entry point", op.n);
    return launch_prox_wide(src, op, stream);
  }
  if (op.eig_solver == 1) return launch_llr_prox_jacobi(src, op, stream);   // every block by Jacobi
  if (op.block_stat) {   // largest Gram eigenvalue per block (sigma_max): fused kernel, chunked Gram, any m
    if (op.n <= 16) return launch_trd_instance<16, 2>(src, op, stream);
    if (op.n <= 32) return launch_trd_instance<32, 2>(src, op, stream);
    return launch_trd_instance<64, 4>(src, op, stream);
  }
  if (op.gram && !op.blk_ra) return set_error(LLR_ERR_INVALID, "split prox path needs the kept-count buffer");
  if (!op.block_stat && !op.fb_list)
    return set_error(LLR_ERR_INVALID, "tridiagonal prox needs a fallback block list");
  if (op.fb_count) LLR_CUDA_TRY(cudaMemsetAsync(op.fb_count, 0, sizeof(int), stream));
  int st;
  if (op.gram) {  // split path: Gram kernel + eigen/apply kernel through the scratch buffer
    if (op.n <= 16) st = launch_split_instance<16, 2>(src, op, stream);
    else if (op.n <= 32) st = launch_split_instance<32, 2>(src, op, stream);
    else st = launch_split_instance<64, 4>(src, op, stream);
  } else {        // fused path (no scratch beyond the fallback list)
    if (op.n <= 16) st = launch_trd_instance<16, 2>(src, op, stream);
    else if (op.n <= 32) st = launch_trd_instance<32, 2>(src, op, stream);
    else st = launch_trd_instance<64, 4>(src, op, stream);
  }
  if (st != LLR_OK || op.block_stat) return st;
  BlockSource fb = src;
  fb.blk_list = op.fb_list;
  fb.blk_count = op.fb_count;
  if (prox_needs_wide_fallback(op.m, op.n)) {   // a whole block does not fit the Jacobi kernel
    if (!op.vwide)
      return set_error(LLR_ERR_UNSUPPORTED, "Casorati %d x %d needs the wide-kernel scratch of a context or of an "
                                            "allocating entry point for its fallback blocks", op.m, op.n);
    return launch_prox_wide(fb, op, stream);
  }
  return launch_llr_prox_jacobi(fb, op, stream);
}

}  // namespace llr
