// Eigen stage of the split LLR prox path, one warp per Casorati block.
//
// Input: the packed lower Gram matrix G = C^H C of every block (written by the Gram kernel).
// Output, in place of G: the block's kept eigenvectors V_a (n x r_a, q-major, r_a <= kFacCols)
// and gains g_a, and the kept count r_a in op.blk_ra.  The apply kernel then forms
// C' = (C V_a) diag(g) V_a^H, which equals U_r S_r V_r^H of the reference's truncated SVD
// (low_rank.rs:10-69, cusolver.rs:20-151) for hard rank and the singular-value soft
// threshold for the soft mode.
//
// A warp owns one block at a time and synchronises only with __syncwarp, so blocks of very
// different cost (all-zero, certified-zero, full eigen path) never wait on each other:
//   (tau = (1 - margin) lambda^2 below; eigenvalues between tau and lambda^2 are near threshold)
//   * soft threshold, ||G||_F <= tau: every eigenvalue is clear below the threshold -> r_a = 0;
//   * soft threshold, max_i G_ii > tau: the top eigenvalue is kept or near -> eigen path;
//   * otherwise a Cholesky factorisation of tau I - G certifies r_a = 0 when it succeeds
//     (every pivot positive) and sends the block to the eigen path when it fails;
//   * eigen path: Householder tridiagonalisation, unitary diagonal to a real tridiagonal T',
//     Sturm counts for the kept and the near-threshold eigenvalues, multisection for them,
//     twisted-factorisation eigenvectors with Gram-Schmidt and a residual check,
//     back-transformation V = Q D Y.  The apply kernel recomputes every column's gain from
//     ||C v||^2 accumulated in FP64 (the refinement sweep: no squared conditioning).
// Blocks keeping more than kFacCols components, or whose eigenvectors fail the residual
// check, get r_a = -1 and go to the Jacobi kernel; hard rank >= n leaves the block as is
// (r_a = -2).
#include <cstdio>
#include <algorithm>

#include "llr_prox_common.cuh"

namespace llr {

namespace {

constexpr int kEigWarps = 2;   // warps (independent blocks) per CTA
// Eigenvalues within this relative margin below lambda^2 are kept as factor columns too (gain
// 0 in FP32): the apply kernel refines every column's singular value from ||C v||^2 with FP64
// accumulation, where FP32 Gram eigenvalues carry an absolute error ~ eps * sigma_1^2.
constexpr float kRefineMargin = 0.1f;

template <int NPMAX>
struct WarpEig {
  float2 A[NPMAX * (NPMAX + 1) / 2];   // packed lower triangle; later Householder vectors
  union {
    struct {
      float2 u[NPMAX];                 // Householder vector / Cholesky column
      float2 w[NPMAX];                 // p - K u
      float2 e[NPMAX];                 // complex sub-diagonal of T
      float e2[NPMAX];                 // |e|^2 for the Sturm counts
      float spare[NPMAX];
    };
    float um[kFacCols * NPMAX];        // eigenvector stage: D+ / U- of each lane's factorisation
  };
  float2 delta[NPMAX];                 // unitary diagonal: T' = D^H T D real
  float d[NPMAX];
  float ae[NPMAX];
  float tau[NPMAX];
  float lam[kFacCols];
  float Y[kFacCols * NPMAX];           // eigenvectors of T', column a at Y[a * NPMAX]
};

__device__ __forceinline__ int pk(int i, int j) { return (i * (i + 1)) / 2 + j; }

__device__ __forceinline__ float wsum(float v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ float wmax(float v) {
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Rows of the trailing L x L matrix owned by a lane: i1 = lane and i2 = L - 1 - lane, so
// that every lane holds L + 1 lower-triangle elements (the middle row of an odd L once).
struct RowPair {
  int i1, i2, n1, tot;
  __device__ __forceinline__ RowPair(int L, int lane) {
    i1 = lane < (L + 1) / 2 ? lane : -1;
    i2 = lane < L / 2 ? L - 1 - lane : -1;
    n1 = i1 + 1;
    tot = n1 + (i2 >= 0 ? i2 + 1 : 0);
  }
};

// True when thr I - G is positive definite, i.e. every eigenvalue of G is below thr:
// unpivoted Cholesky stopping at the first non-positive pivot.  Overwrites A.
template <int NPMAX>
__device__ bool warp_below(WarpEig<NPMAX>* W, int n, float thr) {
  const int lane = threadIdx.x & 31;
  float2* A = W->A;
  const int P = n * (n + 1) / 2;
  for (int i = lane; i < P; i += 32) A[i] = make_float2(-A[i].x, -A[i].y);
  __syncwarp();
  for (int i = lane; i < n; i += 32) A[pk(i, i)].x += thr;
  __syncwarp();
  for (int k = 0; k < n; ++k) {
    const float dk = A[pk(k, k)].x;
    if (!(dk > 0.f)) return false;   // warp-uniform
    const float s = 1.f / sqrtf(dk);
    const int o = k + 1, L = n - o;
    if (L == 0) break;
    const RowPair rp(L, lane);
    float2 l1 = make_float2(0.f, 0.f), l2 = l1;
    if (rp.i1 >= 0) { l1 = cscale(A[pk(o + rp.i1, k)], s); W->u[rp.i1] = l1; }
    if (rp.i2 >= 0) { l2 = cscale(A[pk(o + rp.i2, k)], s); W->u[rp.i2] = l2; }
    __syncwarp();
    const int rb1 = rp.i1 >= 0 ? pk(o + rp.i1, o) : 0, rb2 = rp.i2 >= 0 ? pk(o + rp.i2, o) : 0;
    const float2 nl1 = make_float2(-l1.x, -l1.y), nl2 = make_float2(-l2.x, -l2.y);
    float2 cl = nl1;
    int jo = 0, ib = rb1;
    for (int t = 0; t < rp.tot; ++t) {
      if (t == rp.n1) { cl = nl2; jo = rp.n1; ib = rb2 - rp.n1; }
      float2 a = A[ib + t];
      cfma_cb(a, cl, W->u[t - jo]);
      A[ib + t] = a;
    }
    __syncwarp();
  }
  return true;
}

// Householder reduction of the packed Hermitian A to tridiagonal T (H = I - tau u u^H):
// column k keeps u_k below the diagonal for the back-transformation.
template <int NPMAX>
__device__ void warp_tridiag(WarpEig<NPMAX>* W, int n) {
  const int lane = threadIdx.x & 31;
  float2* A = W->A;
  const float2 z = make_float2(0.f, 0.f);
  for (int k = 0; k + 2 < n; ++k) {
    const int o = k + 1, L = n - o;
    const RowPair rp(L, lane);
    float2 x1 = rp.i1 >= 0 ? A[pk(o + rp.i1, k)] : z;
    float2 x2 = rp.i2 >= 0 ? A[pk(o + rp.i2, k)] : z;
    const float s2 = wsum(cabs2(x1) + cabs2(x2));
    const float2 x0 = make_float2(__shfl_sync(0xffffffffu, x1.x, 0), __shfl_sync(0xffffffffu, x1.y, 0));
    const float xn = sqrtf(s2), aa = sqrtf(cabs2(x0));
    const float phx = aa > 0.f ? x0.x / aa : 1.f, phy = aa > 0.f ? x0.y / aa : 0.f;
    const float2 u0 = make_float2(x0.x + phx * xn, x0.y + phy * xn);
    const float un2 = s2 - aa * aa + cabs2(u0);
    const float t = (xn > 0.f && un2 > 0.f) ? 2.f / un2 : 0.f;
    if (lane == 0) {
      W->tau[k] = t;
      W->e[k] = make_float2(-phx * xn, -phy * xn);
      A[pk(o, k)] = u0;
    }
    if (rp.i1 == 0) x1 = u0;
    if (t == 0.f) {   // warp-uniform: no reflection at this step
      __syncwarp();
      continue;
    }
    if (rp.i1 >= 0) W->u[rp.i1] = x1;
    if (rp.i2 >= 0) W->u[rp.i2] = x2;
    __syncwarp();
    // p = t A22 u, reading A22[i][j] = conj(A22[j][i]) above the diagonal.  Lanes without a
    // row read row 0 (a valid element) and drop the result; four columns are in flight at once.
    const int r1 = max(rp.i1, 0), r2 = max(rp.i2, 0);
    const int rb1 = pk(o + r1, o), rb2 = pk(o + r2, o);
    float2 p1 = z, p2 = z, q1 = z, q2 = z;
    for (int j0 = 0; j0 < L; j0 += 4) {
      float2 a1[4], a2[4], uj[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int j = min(j0 + e, L - 1);
        const int cb = pk(o + j, o);              // trailing row j
        uj[e] = W->u[j];
        a1[e] = A[j <= r1 ? rb1 + j : cb + r1];
        a2[e] = A[j <= r2 ? rb2 + j : cb + r2];
      }
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int j = j0 + e;
        if (j < L) {                              // warp-uniform
          float2 b1 = a1[e], b2 = a2[e];
          if (j > r1) b1.y = -b1.y;
          if (j > r2) b2.y = -b2.y;
          if (e & 1) { cfma(q1, b1, uj[e]); cfma(q2, b2, uj[e]); }
          else { cfma(p1, b1, uj[e]); cfma(p2, b2, uj[e]); }
        }
      }
    }
    p1 = rp.i1 >= 0 ? cscale(cadd(p1, q1), t) : z;
    p2 = rp.i2 >= 0 ? cscale(cadd(p2, q2), t) : z;
    const float dp = wsum(x1.x * p1.x + x1.y * p1.y + x2.x * p2.x + x2.y * p2.y);
    const float K = 0.5f * t * dp;
    const float2 w1 = csub(p1, cscale(x1, K)), w2 = csub(p2, cscale(x2, K));
    if (rp.i1 >= 0) W->w[rp.i1] = w1;
    if (rp.i2 >= 0) W->w[rp.i2] = w2;
    __syncwarp();
    // A22 -= u w^H + w u^H on the lower triangle of the lane's rows: element s of the lane is
    // row i1 column s for s < n1, else row i2 column s - n1; every element has one owner lane,
    // so the four loads of a group can all go out before its stores.
    const float2 nu1 = make_float2(-x1.x, -x1.y), nu2 = make_float2(-x2.x, -x2.y);
    const float2 nw1 = make_float2(-w1.x, -w1.y), nw2 = make_float2(-w2.x, -w2.y);
    const int smax = max(rp.tot - 1, 0);
    for (int s0 = 0; s0 <= L; s0 += 4) {
      float2 a[4], wj[4], uj[4];
      int id[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int sc = min(s0 + e, smax);
        const bool f = sc < rp.n1;
        const int j = f ? sc : sc - rp.n1;
        id[e] = f ? rb1 + sc : rb2 + j;
        a[e] = A[id[e]];
        wj[e] = W->w[j];
        uj[e] = W->u[j];
      }
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const bool f = s0 + e < rp.n1;
        float2 r = a[e];
        cfma_cb(r, f ? nu1 : nu2, wj[e]);
        cfma_cb(r, f ? nw1 : nw2, uj[e]);
        if (s0 + e < rp.tot) A[id[e]] = r;
      }
    }
    __syncwarp();
  }
  for (int i = lane; i < n; i += 32) W->d[i] = A[pk(i, i)].x;
  if (lane == 0) {
    if (n >= 2) W->e[n - 2] = A[pk(n - 1, n - 2)];
    for (int k = std::max(0, n - 2); k < n; ++k) W->tau[k] = 0.f;
  }
  __syncwarp();
}

struct TriInfo {
  float gl, gu, tnorm, pivmin;
};

__device__ __forceinline__ int sturm_below(const float* d, const float* e2, int n, float x, float pivmin) {
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

// Real form T' = D^H T D (D a prefix product of unit phases), |e|, e^2, Gershgorin bounds.
template <int NPMAX>
__device__ TriInfo warp_setup(WarpEig<NPMAX>* W, int n) {
  const int lane = threadIdx.x & 31;
  float2 ph[2];
  float e2m = 0.f;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int k = 2 * lane + h;
    ph[h] = make_float2(1.f, 0.f);
    if (k + 1 < n) {
      const float2 ek = W->e[k];
      const float a = sqrtf(cabs2(ek));
      W->ae[k] = a;
      W->e2[k] = a * a;
      e2m = fmaxf(e2m, a * a);
      if (a > 0.f) ph[h] = make_float2(ek.x / a, ek.y / a);
    } else if (k < n) {
      W->ae[k] = 0.f;
      W->e2[k] = 0.f;
    }
  }
  float2 pr = cmul(ph[0], ph[1]);
  for (int o = 1; o < 32; o <<= 1) {
    const float ox = __shfl_up_sync(0xffffffffu, pr.x, o), oy = __shfl_up_sync(0xffffffffu, pr.y, o);
    if (lane >= o) pr = cmul(make_float2(ox, oy), pr);
  }
  float ex = __shfl_up_sync(0xffffffffu, pr.x, 1), ey = __shfl_up_sync(0xffffffffu, pr.y, 1);
  if (lane == 0) { ex = 1.f; ey = 0.f; }
  const float2 excl = make_float2(ex, ey);
  if (2 * lane < n) W->delta[2 * lane] = excl;
  if (2 * lane + 1 < n) W->delta[2 * lane + 1] = cmul(excl, ph[0]);
  __syncwarp();
  float gl = 3.0e38f, gu = -3.0e38f;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int k = 2 * lane + h;
    if (k < n) {
      const float r = (k > 0 ? W->ae[k - 1] : 0.f) + (k + 1 < n ? W->ae[k] : 0.f);
      gl = fminf(gl, W->d[k] - r);
      gu = fmaxf(gu, W->d[k] + r);
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    gl = fminf(gl, __shfl_xor_sync(0xffffffffu, gl, o));
    gu = fmaxf(gu, __shfl_xor_sync(0xffffffffu, gu, o));
    e2m = fmaxf(e2m, __shfl_xor_sync(0xffffffffu, e2m, o));
  }
  TriInfo ti;
  ti.tnorm = fmaxf(fabsf(gl), fabsf(gu));
  ti.gl = gl - (4.f * 1.1920929e-7f * ti.tnorm * n + 1e-30f);
  ti.gu = gu + (4.f * 1.1920929e-7f * ti.tnorm * n + 1e-30f);
  ti.pivmin = 1.1754944e-38f * fmaxf(1.f, e2m);
  return ti;
}

// Eigenvalues j0 .. j0 + count - 1 (ascending order, count <= kFacCols) by multisection:
// a group of G lanes splits its interval G + 1 ways per round.
template <int NPMAX>
__device__ void warp_eigenvalues(WarpEig<NPMAX>* W, int n, int j0, int count, const TriInfo& ti) {
  const int lane = threadIdx.x & 31;
  const int G = count == 1 ? 32 : (count == 2 ? 16 : (count <= 4 ? 8 : 4));
  const int gl = lane & (G - 1), group = lane / G;
  const unsigned gmask = G == 32 ? 0xffffffffu : ((1u << G) - 1u);
  const float inv = 1.f / (float)(G + 1);
  const bool act = group < count;
  const int j = j0 + (act ? group : 0);
  float lo = ti.gl, hi = ti.gu;
  for (int round = 0; round < 40; ++round) {
    const bool conv = !act || (hi - lo) <= 2.4e-7f * fmaxf(fabsf(lo), fabsf(hi)) + ti.pivmin;
    if (__all_sync(0xffffffffu, conv)) break;
    const float x = lo + (hi - lo) * (float)(gl + 1) * inv;
    const bool le = act ? (sturm_below(W->d, W->e2, n, x, ti.pivmin) <= j) : true;
    const unsigned bal = __ballot_sync(0xffffffffu, le);
    const int nt = __popc((bal >> (lane & ~(G - 1) & 31)) & gmask);
    const float nlo = nt > 0 ? lo + (hi - lo) * (float)nt * inv : lo;
    const float nhi = nt < G ? lo + (hi - lo) * (float)(nt + 1) * inv : hi;
    lo = nlo;
    hi = nhi;
  }
  if (act && gl == 0) W->lam[group] = 0.5f * (lo + hi);
  __syncwarp();
}

// Eigenvectors of T' for the ra kept eigenvalues: lane a solves the twisted factorisation
// T' - lam_a I = L+ D+ L+^T = U- D- U-^T (twist at the smallest |gamma|), then the warp
// orthonormalises them (modified Gram-Schmidt) and checks ||T' y - lam y||.  Returns false
// when a vector fails the check.
template <int NPMAX>
__device__ bool warp_vectors(WarpEig<NPMAX>* W, int n, int ra, const TriInfo& ti) {
  const int lane = threadIdx.x & 31;
  const float eps = 1.1920929e-7f;
  const float tiny = eps * fmaxf(ti.tnorm, 1e-30f);
  if (lane == 0) {
    const float sep = 10.f * eps * fmaxf(ti.tnorm, 1e-30f);
    for (int a = 1; a < ra; ++a)
      if (W->lam[a] - W->lam[a - 1] < sep) W->lam[a] = W->lam[a - 1] + sep;
  }
  __syncwarp();
  if (lane < ra) {
    // Lp lives in the lane's own row of Y (overwritten in place by the vector), D+ / U- in the
    // lane's row of um (the tridiagonalisation and Sturm scratch, dead by now).
    float* y = W->Y + lane * NPMAX;
    float* Um = W->um + lane * NPMAX;
    const float lam = W->lam[lane];
    float dp = W->d[0] - lam;
#pragma unroll 4
    for (int i = 0; i + 1 < n; ++i) {
      if (fabsf(dp) < tiny) dp = copysignf(tiny, dp);
      Um[i] = dp;   // D+_i, replaced by U-_i on the way back
      const float l = W->ae[i] * __frcp_rn(dp);
      y[i] = l;
      dp = W->d[i + 1] - lam - l * W->ae[i];
    }
    if (fabsf(dp) < tiny) dp = copysignf(tiny, dp);
    float dm = W->d[n - 1] - lam;
    float best = fabsf(dp);
    int r = n - 1;
#pragma unroll 4
    for (int i = n - 2; i >= 0; --i) {
      if (fabsf(dm) < tiny) dm = copysignf(tiny, dm);
      const float um = W->ae[i] * __frcp_rn(dm);
      const float dpi = Um[i];
      Um[i] = um;
      dm = W->d[i] - lam - um * W->ae[i];
      const float gamma = dpi + dm - (W->d[i] - lam);
      if (fabsf(gamma) < best) { best = fabsf(gamma); r = i; }
    }
    float zz = 1.f;
    for (int i = r - 1; i >= 0; --i) { zz = -y[i] * zz; y[i] = zz; }
    y[r] = 1.f;
    zz = 1.f;
    for (int i = r; i + 1 < n; ++i) { zz = -Um[i] * zz; y[i + 1] = zz; }
    float mx = 0.f;
    for (int i = 0; i < n; ++i) mx = fmaxf(mx, fabsf(y[i]));
    const float sc = (mx > 0.f && mx < 3.0e38f) ? 1.f / mx : 0.f;
    for (int i = 0; i < n; ++i) y[i] *= sc;
  }
  __syncwarp();
  const float tol = 2e-5f * fmaxf(ti.tnorm, 1e-30f);
  bool bad = false;
  for (int a = 0; a < ra; ++a) {
    float* y = W->Y + a * NPMAX;
    float y0 = lane < n ? y[lane] : 0.f, y1 = lane + 32 < n ? y[lane + 32] : 0.f;
    for (int c = 0; c < a; ++c) {
      const float* zc = W->Y + c * NPMAX;
      const float z0 = lane < n ? zc[lane] : 0.f, z1 = lane + 32 < n ? zc[lane + 32] : 0.f;
      const float dpr = wsum(y0 * z0 + y1 * z1);
      y0 -= dpr * z0;
      y1 -= dpr * z1;
    }
    const float nn = wsum(y0 * y0 + y1 * y1);
    const float inv = nn > 0.f ? rsqrtf(nn) : 0.f;
    y0 *= inv;
    y1 *= inv;
    if (lane < n) y[lane] = y0;
    if (lane + 32 < n) y[lane + 32] = y1;
    __syncwarp();
    const float lam = W->lam[a];
    float r2 = 0.f;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int i = lane + 32 * h;
      if (i < n) {
        float rr = (W->d[i] - lam) * y[i];
        if (i > 0) rr += W->ae[i - 1] * y[i - 1];
        if (i + 1 < n) rr += W->ae[i] * y[i + 1];
        r2 += rr * rr;
      }
    }
    r2 = wsum(r2);
    if (!(nn > 0.f) || !(sqrtf(r2) <= tol)) bad = true;
    __syncwarp();
  }
  return !bad;
}

// V = Q D Y, Q = H_0 H_1 ... H_{n-3}: a group of Gv = 32 / R lanes per kept vector (R = ra
// rounded up to a power of two), each lane holding the rows g, g + Gv, ... of its vector in
// registers; per reflector a serial partial u^H v and log2(Gv) shuffle levels.  Written
// q-major to fac[q * kFacCols + a].
template <int NPMAX>
__device__ void warp_backtransform(WarpEig<NPMAX>* W, int n, int ra, float2* fac) {
  constexpr int kPer = NPMAX / 4;                 // rows per lane at Gv = 4 (ra > 4)
  const int lane = threadIdx.x & 31;
  const int R = ra <= 1 ? 1 : (ra <= 2 ? 2 : (ra <= 4 ? 4 : 8));
  const int Gv = 32 / R;
  const int a = lane / Gv, g = lane - a * Gv;
  const bool act = a < ra;
  const int tmax = (n + Gv - 1) / Gv;             // warp-uniform
  const float2 z = make_float2(0.f, 0.f);
  float2 v[kPer];
#pragma unroll
  for (int t = 0; t < kPer; ++t) {
    const int i = g + Gv * t;
    v[t] = (act && i < n) ? cscale(W->delta[i], W->Y[a * NPMAX + i]) : z;
  }
  for (int k = n - 3; k >= 0; --k) {
    const float tk = W->tau[k];
    if (tk == 0.f) continue;                      // warp-uniform
    float2 s = z;
#pragma unroll
    for (int t = 0; t < kPer; ++t) {
      if (t >= tmax) break;
      const int i = g + Gv * t;
      if (i > k && i < n) s = cadd(s, cmulc(W->A[pk(i, k)], v[t]));
    }
    for (int o = Gv >> 1; o > 0; o >>= 1) {
      s.x += __shfl_xor_sync(0xffffffffu, s.x, o);
      s.y += __shfl_xor_sync(0xffffffffu, s.y, o);
    }
    s = cscale(s, tk);
#pragma unroll
    for (int t = 0; t < kPer; ++t) {
      if (t >= tmax) break;
      const int i = g + Gv * t;
      if (i > k && i < n) v[t] = csub(v[t], cmul(W->A[pk(i, k)], s));
    }
  }
#pragma unroll
  for (int t = 0; t < kPer; ++t) {
    const int i = g + Gv * t;
    if (act && i < n) fac[i * kFacCols + a] = v[t];
  }
}

template <int NPMAX>
__global__ void __launch_bounds__(32 * kEigWarps, 5) llr_eig_warp_kernel(ProxOp op, long long nblocks) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  WarpEig<NPMAX>* W = reinterpret_cast<WarpEig<NPMAX>*>(smem) + wib;
  const int n = op.n;
  const int P = n * (n + 1) / 2;
  const bool soft = op.mode != LLR_PROX_HARD_RANK;
  const float thr = op.lambda * op.lambda;
  const float thr_lo = thr * (1.f - kRefineMargin);
  int* counter = op.blk_ra + nblocks;   // dynamic block queue, zeroed before the launch
  for (;;) {
    int bi = 0;
    if (lane == 0) bi = atomicAdd(counter, 1);
    const long long blk = __shfl_sync(0xffffffffu, bi, 0);
    if (blk >= nblocks) break;
    float2* G = op.gram + blk * op.gram_stride;
    float s_all = 0.f;
    for (int i = lane; i < P; i += 32) {
      const float2 v = G[i];
      W->A[i] = v;
      s_all += cabs2(v);
    }
    __syncwarp();
    float s_diag = 0.f, dmax = 0.f;
    for (int i = lane; i < n; i += 32) {
      const float2 v = W->A[pk(i, i)];
      s_diag += v.x * v.x;
      dmax = fmaxf(dmax, v.x);
    }
    const float fro2 = 2.f * wsum(s_all) - wsum(s_diag);   // ||G||_F^2 from the lower triangle
    dmax = wmax(dmax);
    int ra;
    if (!soft && op.rank >= n) {
      ra = -2;                                            // identity: leave the block as is
    } else if (soft && !(op.lambda > 0.f)) {
      ra = -2;                                            // no threshold: identity
    } else if (soft && fro2 <= thr_lo * thr_lo) {
      ra = 0;                                             // lambda_max <= ||G||_F, clear of the margin
    } else {
      bool eig = !soft || dmax > thr_lo;                  // lambda_max >= max_i G_ii
      if (!eig) {
        eig = !warp_below(W, n, thr_lo);
        if (eig) {                                        // the test overwrote A: reload
          for (int i = lane; i < P; i += 32) W->A[i] = G[i];
          __syncwarp();
        }
      }
      if (!eig) {
        ra = 0;
      } else {
        warp_tridiag(W, n);
        const TriInfo ti = warp_setup(W, n);
        int nb, nb_lo;
        if (!soft) {
          nb = nb_lo = n - op.rank;
        } else {                                          // every lane runs the count: same answer
          nb = sturm_below(W->d, W->e2, n, thr, ti.pivmin);
          nb_lo = sturm_below(W->d, W->e2, n, thr_lo, ti.pivmin);
        }
        ra = n - nb;                                      // kept in FP32
        if (ra > kFacCols) {
          ra = -1;
        } else {
          ra = min(n - nb_lo, kFacCols);                  // plus the near-threshold ones
        }
        if (ra > 0) {
          warp_eigenvalues(W, n, n - ra, ra, ti);
          if (!warp_vectors(W, n, ra, ti)) {
            ra = -1;
          } else {
            warp_backtransform(W, n, ra, G);
            if (lane < ra) {
              float gv = 1.f;
              if (soft) {
                const float sv = sqrtf(fmaxf(W->lam[lane], 0.f));
                gv = sv > op.lambda ? 1.f - op.lambda / sv : 0.f;
              }
              G[n * kFacCols + lane] = make_float2(gv, 0.f);
            }
          }
        }
      }
    }
    if (lane == 0) {
      op.blk_ra[blk] = ra;
      if (ra == -1) op.fb_list[atomicAdd(op.fb_count, 1)] = (int)blk;
    }
    __syncwarp();
  }
}

template <int NPMAX>
int launch_eig_warp_instance(const ProxOp& op, long long nblocks, cudaStream_t stream) {
  const size_t smem = sizeof(WarpEig<NPMAX>) * kEigWarps;
  auto kern = llr_eig_warp_kernel<NPMAX>;
  LLR_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  LLR_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
  int dev = 0, nsm = 0, occ = 0;
  LLR_CUDA_TRY(cudaGetDevice(&dev));
  LLR_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  LLR_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, 32 * kEigWarps, smem));
  if (occ < 1) return set_error(LLR_ERR_UNSUPPORTED, "warp eigen kernel cannot be resident (smem %zu B)", smem);
  const long long want = (nblocks + kEigWarps - 1) / kEigWarps;
  const long long grid = std::min<long long>(want, (long long)nsm * occ);
  LLR_CUDA_TRY(cudaMemsetAsync(op.blk_ra + nblocks, 0, sizeof(int), stream));
  note_launch();
  kern<<<(unsigned)grid, 32 * kEigWarps, smem, stream>>>(op, nblocks);
  LLR_CUDA_TRY(cudaGetLastError());
  return LLR_OK;
}

}  // namespace

int launch_llr_eig_warp(const ProxOp& op, long long nblocks, cudaStream_t stream) {
  if (!op.gram || !op.blk_ra || !op.fb_list || !op.fb_count)
    return set_error(LLR_ERR_INVALID, "warp eigen kernel needs the Gram scratch, block codes and fallback list");
  if (op.gram_stride < prox_gram_stride(op.n)) return set_error(LLR_ERR_INVALID, "Gram scratch stride too small");
  if (nblocks == 0) return LLR_OK;
  if (op.n <= 16) return launch_eig_warp_instance<16>(op, nblocks, stream);
  if (op.n <= 32) return launch_eig_warp_instance<32>(op, nblocks, stream);
  if (op.n <= 64) return launch_eig_warp_instance<64>(op, nblocks, stream);
  return set_error(LLR_ERR_UNSUPPORTED, "Casorati column count %d > 64 is not supported", op.n);
}

}  // namespace llr
