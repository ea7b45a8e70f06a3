// Fused hybrid-space data consistency: forward 2-D DFT over (y, z), hard DC on the sampled
// lines, inverse 2-D DFT, for one (x, volume) plane at a time with the plane held in shared
// memory.  One HBM read and one write of the iterate per iteration, against two of each per
// cuFFT pass plus the DC pass (signal_model.rs:34-79 with the x-transform cancelled, see the
// hybrid-space identity; hard_project lib.rs:392-406 on the sampled lines).
//
// Each axis of length N = N1 * N2 is a four-step transform in place: N2 register DFTs of
// length N1 (stride N2) with twiddles W_N^{n2 k1}, then N1 register DFTs of length N2; the
// spectrum is left in the permuted order p = N2 (k mod N1) + k / N1, which the DC indexes
// directly and the inverse (the same steps mirrored) consumes.  Register DFTs of length
// 2, 3, 4, 6, 8, 12, 16 are nested Cooley-Tukey with FP64-computed twiddle tables.
// Forward and inverse are unnormalised like cuFFT's; the residual sum |F x - yhat|^2 is
// accumulated in FP64 per CTA (fixed plane order) for the deterministic finalize kernel.
#include <cmath>
#include <cstdio>
#include <vector>
#include <algorithm>

#include "llr_common.cuh"
#include "llr_internal.h"
#include "llr_prox_common.cuh"

namespace llr {

namespace {

constexpr int kFftThreads = 512;

__host__ __device__ inline size_t align16b(size_t x) { return (x + 15) & ~size_t(15); }

// Twiddle-table layout in shared memory (float2 entries): W_ny^j, W_nz^j, then W_R^j for the
// register sizes 16, 12, 8, 6 (W_4, W_3, W_2 are exact constants).
struct FftTab {
  int off_y, off_z, off_16, off_12, off_8, off_6, total;
};

__host__ __device__ inline FftTab fft_tab(int ny, int nz) {
  FftTab t;
  t.off_y = 0;
  t.off_z = ny;
  t.off_16 = ny + nz;
  t.off_12 = t.off_16 + 16;
  t.off_8 = t.off_12 + 12;
  t.off_6 = t.off_8 + 8;
  t.total = t.off_6 + 6;
  return t;
}

// x * W where W = tw (forward) or conj(tw) (inverse)
template <int DIR>
__device__ __forceinline__ float2 twmul(float2 x, float2 tw) {
  return DIR > 0 ? cmul(x, tw) : cmul_bc(x, tw);
}

// -i * x (forward) / +i * x (inverse)
template <int DIR>
__device__ __forceinline__ float2 rot(float2 x) {
  return DIR > 0 ? make_float2(x.y, -x.x) : make_float2(-x.y, x.x);
}

template <int R, int DIR>
struct Dft;

template <int DIR>
struct Dft<1, DIR> {
  __device__ __forceinline__ static void run(float2* v, const float2*) {}
};

template <int DIR>
struct Dft<2, DIR> {
  __device__ __forceinline__ static void run(float2* v, const float2*) {
    const float2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};

template <int DIR>
struct Dft<3, DIR> {
  __device__ __forceinline__ static void run(float2* v, const float2*) {
    const float s = 0.86602540378443864676f;   // sin(2 pi / 3)
    const float2 a = v[0], b = v[1], c = v[2];
    const float2 t1 = cadd(b, c);
    const float2 t2 = make_float2(a.x - 0.5f * t1.x, a.y - 0.5f * t1.y);
    const float2 t3 = cscale(csub(b, c), s);
    const float2 r = rot<DIR>(t3);   // -i s (b - c) forward
    v[0] = cadd(a, t1);
    v[1] = cadd(t2, r);
    v[2] = csub(t2, r);
  }
};

template <int DIR>
struct Dft<4, DIR> {
  __device__ __forceinline__ static void run(float2* v, const float2*) {
    const float2 a = v[0], b = v[1], c = v[2], d = v[3];
    const float2 s0 = cadd(a, c), s1 = csub(a, c), s2 = cadd(b, d), s3 = rot<DIR>(csub(b, d));
    v[0] = cadd(s0, s2);
    v[2] = csub(s0, s2);
    v[1] = cadd(s1, s3);
    v[3] = csub(s1, s3);
  }
};

// W_R^m = e^{-2 pi i m / R} for the register DFTs, evaluated at compile time from the Taylor
// series of cos and sin in double precision (|x| <= 2 pi, 30 terms).
constexpr double kTwoPi = 6.283185307179586476925286766559;
constexpr double taylor_cos(double x) {
  double t = 1.0, s = 1.0;
  for (int k = 1; k < 30; ++k) { t *= -x * x / ((2.0 * k - 1.0) * (2.0 * k)); s += t; }
  return s;
}
constexpr double taylor_sin(double x) {
  double t = x, s = x;
  for (int k = 1; k < 30; ++k) { t *= -x * x / ((2.0 * k) * (2.0 * k + 1.0)); s += t; }
  return s;
}
template <int R>
struct TwTab {
  float re[R], im[R];
  constexpr TwTab() : re(), im() {
    for (int m = 0; m < R; ++m) {
      re[m] = (float)taylor_cos(kTwoPi * m / R);
      im[m] = (float)-taylor_sin(kTwoPi * m / R);
    }
  }
};
template <int R>
__device__ constexpr TwTab<R> kTw = TwTab<R>();

// R = R1 * R2 Cooley-Tukey in registers: input natural order n = R2 n1 + n2, output natural
// order k = k1 + R1 k2; twiddles W_R^{n2 k1} are compile-time constants.
template <int R1, int R2, int DIR>
__device__ __forceinline__ void dft_ct(float2* v, const float2*, const float2* w1, const float2* w2) {
  constexpr int R = R1 * R2;
  float2 a[R];
#pragma unroll
  for (int n2 = 0; n2 < R2; ++n2) {
    float2 t[R1];
#pragma unroll
    for (int n1 = 0; n1 < R1; ++n1) t[n1] = v[R2 * n1 + n2];
    Dft<R1, DIR>::run(t, w1);
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) {
      const int m = (n2 * k1) % R;
      a[k1 * R2 + n2] = m == 0 ? t[k1] : twmul<DIR>(t[k1], make_float2(kTw<R>.re[m], kTw<R>.im[m]));
    }
  }
#pragma unroll
  for (int k1 = 0; k1 < R1; ++k1) {
    float2 t[R2];
#pragma unroll
    for (int n2 = 0; n2 < R2; ++n2) t[n2] = a[k1 * R2 + n2];
    Dft<R2, DIR>::run(t, w2);
#pragma unroll
    for (int k2 = 0; k2 < R2; ++k2) v[k1 + R1 * k2] = t[k2];
  }
}

template <int DIR>
struct Dft<6, DIR> {
  __device__ __forceinline__ static void run(float2* v, const float2* w) { dft_ct<3, 2, DIR>(v, w, nullptr, nullptr); }
};
template <int DIR>
struct Dft<8, DIR> {
  __device__ __forceinline__ static void run(float2* v, const float2* w) { dft_ct<4, 2, DIR>(v, w, nullptr, nullptr); }
};
template <int DIR>
struct Dft<12, DIR> {
  __device__ __forceinline__ static void run(float2* v, const float2* w) { dft_ct<4, 3, DIR>(v, w, nullptr, nullptr); }
};
template <int DIR>
struct Dft<16, DIR> {
  __device__ __forceinline__ static void run(float2* v, const float2* w) { dft_ct<4, 4, DIR>(v, w, nullptr, nullptr); }
};

__device__ __forceinline__ const float2* small_tab(const float2* tw, const FftTab& T, int R) {
  switch (R) {
    case 16: return tw + T.off_16;
    case 12: return tw + T.off_12;
    case 8: return tw + T.off_8;
    case 6: return tw + T.off_6;
    default: return tw;
  }
}

// One pass over every transform of an axis: B transforms (batch stride bs), each of length
// N = N1 N2 with element stride es.  STEP 0: DFTs of length R = N1 over n1 (stride N2), then
// twiddles; STEP 1: DFTs of length R = N2 over contiguous positions.  Forward order: 0 then 1;
// inverse: 1 then 0 (twiddles before the DFT).
template <int R, int DIR, int STEP>
__device__ __forceinline__ void axis_pass(float2* s, int B, int bs, int es, int N1, int N2, const float2* wN, int N,
                                          const float2* wR) {
  const int J = STEP == 0 ? N2 : N1;   // transforms of length R per batch entry
  const int tasks = B * J;
  for (int t = threadIdx.x; t < tasks; t += blockDim.x) {
    const int b = t % B, j = t / B;
    float2* base = s + (long long)b * bs;
    float2 v[R];
    if (STEP == 0) {   // j = n2; elements at N2 n1 + n2
#pragma unroll
      for (int i = 0; i < R; ++i) v[i] = base[(N2 * i + j) * es];
      // twiddle W_N^{n2 k1}, n2 k1 < N (before the inverse DFT, after the forward one)
      if (DIR < 0) {
#pragma unroll
        for (int i = 1; i < R; ++i) v[i] = twmul<DIR>(v[i], wN[j * i]);
      }
      Dft<R, DIR>::run(v, wR);
      if (DIR > 0) {
#pragma unroll
        for (int i = 1; i < R; ++i) v[i] = twmul<DIR>(v[i], wN[j * i]);
      }
#pragma unroll
      for (int i = 0; i < R; ++i) base[(N2 * i + j) * es] = v[i];
    } else {           // j = k1; elements at N2 k1 + n2
#pragma unroll
      for (int i = 0; i < R; ++i) v[i] = base[(N2 * j + i) * es];
      Dft<R, DIR>::run(v, wR);
#pragma unroll
      for (int i = 0; i < R; ++i) base[(N2 * j + i) * es] = v[i];
    }
  }
}

template <int DIR, int STEP>
__device__ void axis_dispatch(float2* s, int B, int bs, int es, int N1, int N2, const float2* wN, int N,
                              const float2* tw, const FftTab& T) {
  const int R = STEP == 0 ? N1 : N2;
  const float2* wR = small_tab(tw, T, R);
  switch (R) {
    case 2: axis_pass<2, DIR, STEP>(s, B, bs, es, N1, N2, wN, N, wR); break;
    case 3: axis_pass<3, DIR, STEP>(s, B, bs, es, N1, N2, wN, N, wR); break;
    case 4: axis_pass<4, DIR, STEP>(s, B, bs, es, N1, N2, wN, N, wR); break;
    case 6: axis_pass<6, DIR, STEP>(s, B, bs, es, N1, N2, wN, N, wR); break;
    case 8: axis_pass<8, DIR, STEP>(s, B, bs, es, N1, N2, wN, N, wR); break;
    case 12: axis_pass<12, DIR, STEP>(s, B, bs, es, N1, N2, wN, N, wR); break;
    case 16: axis_pass<16, DIR, STEP>(s, B, bs, es, N1, N2, wN, N, wR); break;
    default: break;
  }
}

__device__ __forceinline__ int perm_pos(int k, int N1, int N2) { return N2 * (k % N1) + k / N1; }

struct FftDcArgs {
  float2* u;                 // planar iterate: plane (ix, q) at ny * nz * (ix + nx * q)
  const float2* yhat;        // per volume q: nx x L_q, x-major (line index fastest)
  const int* pos;            // sampled (ky + ny kz) per line
  const long long* off;      // line offsets per volume (nq + 1)
  const float2* twiddle;     // FftTab entries
  double* partials;          // one FP64 residual per CTA
  int nx, ny, nz, nq;
  int y1, y2, z1, z2;        // ny = y1 y2, nz = z1 z2
  int pitch;                 // odd row pitch of the shared plane
  const int* zero_ra;        // optional: per-block kept counts of this iteration's prox; blocks
                             // with 0 were left unwritten and are zero-filled on load
  BlockSource zsrc;          // block grid and shift of that prox (when zero_ra is set)
};

constexpr int kZeroFlagMax = 4096;   // blocks per (x) block slab covered by the zero-fill table

// Passes of one axis with every size a compile-time constant (hot plane shapes).
template <int DIR, int STEP, int B, int BS, int ES, int N1, int N2, int NT>
__device__ __forceinline__ void axis_pass_fixed(float2* s, const float2* wN) {
  constexpr int R = STEP == 0 ? N1 : N2;
  constexpr int J = STEP == 0 ? N2 : N1;
  constexpr int TASKS = B * J;
#pragma unroll 1
  for (int t = threadIdx.x; t < TASKS; t += NT) {
    const int b = t % B, j = t / B;
    float2* base = s + b * BS + (STEP == 0 ? j : N2 * j) * ES;
    float2 v[R];
#pragma unroll
    for (int i = 0; i < R; ++i) v[i] = base[(STEP == 0 ? N2 * i : i) * ES];
    if (STEP == 0 && DIR < 0) {
#pragma unroll
      for (int i = 1; i < R; ++i) v[i] = twmul<DIR>(v[i], wN[j * i]);
    }
    Dft<R, DIR>::run(v, nullptr);
    if (STEP == 0 && DIR > 0) {
#pragma unroll
      for (int i = 1; i < R; ++i) v[i] = twmul<DIR>(v[i], wN[j * i]);
    }
#pragma unroll
    for (int i = 0; i < R; ++i) base[(STEP == 0 ? N2 * i : i) * ES] = v[i];
  }
}

// First forward / last inverse pass of the z axis (step 0: DFTs of length Z1 at stride Z2 down z)
// on the plane in HBM (element (y, z) at g[y + ny z], lanes along y: 256-byte warp accesses) and
// the shared plane (row pitch PP) on the other side: the forward pass loads its elements straight
// into registers, zero-filling those of zero blocks (zero(y, z)), and stores the twiddled result
// in shared memory; the inverse pass reads shared memory and stores its result to HBM.
template <int DIR, int NY, int PP, int Z1, int Z2, int NT, class ZeroFn>
__device__ __forceinline__ void z_pass_hbm(float2* s, float2* g, const float2* wN, ZeroFn zero) {
  constexpr int TASKS = NY * Z2;
#pragma unroll 1
  for (int t = threadIdx.x; t < TASKS; t += NT) {
    const int y = t % NY, j = t / NY;
    float2* sb = s + y + PP * j;
    float2* gb = g + y + NY * j;
    float2 v[Z1];
    if (DIR > 0) {
#pragma unroll
      for (int i = 0; i < Z1; ++i) v[i] = zero(y, Z2 * i + j) ? make_float2(0.f, 0.f) : gb[NY * Z2 * i];
      Dft<Z1, DIR>::run(v, nullptr);
#pragma unroll
      for (int i = 1; i < Z1; ++i) v[i] = twmul<DIR>(v[i], wN[j * i]);
#pragma unroll
      for (int i = 0; i < Z1; ++i) sb[PP * Z2 * i] = v[i];
    } else {
#pragma unroll
      for (int i = 0; i < Z1; ++i) v[i] = sb[PP * Z2 * i];
#pragma unroll
      for (int i = 1; i < Z1; ++i) v[i] = twmul<DIR>(v[i], wN[j * i]);
      Dft<Z1, DIR>::run(v, nullptr);
#pragma unroll
      for (int i = 0; i < Z1; ++i) gb[NY * Z2 * i] = v[i];
    }
  }
}

// Plane geometry with run-time sizes (any shape split_len accepts).
struct GeoRt {
  static constexpr bool kHbmPasses = false;
  int ny, nz, y1, y2, z1, z2, P;
  __device__ void forward(float2* s, const float2* tw, const FftTab& T) const {
    axis_dispatch<1, 0>(s, nz, P, 1, y1, y2, tw + T.off_y, ny, tw, T);
    __syncthreads();
    axis_dispatch<1, 1>(s, nz, P, 1, y1, y2, tw + T.off_y, ny, tw, T);
    __syncthreads();
    axis_dispatch<1, 0>(s, ny, 1, P, z1, z2, tw + T.off_z, nz, tw, T);
    __syncthreads();
    axis_dispatch<1, 1>(s, ny, 1, P, z1, z2, tw + T.off_z, nz, tw, T);
  }
  __device__ void inverse(float2* s, const float2* tw, const FftTab& T) const {
    axis_dispatch<-1, 1>(s, ny, 1, P, z1, z2, tw + T.off_z, nz, tw, T);
    __syncthreads();
    axis_dispatch<-1, 0>(s, ny, 1, P, z1, z2, tw + T.off_z, nz, tw, T);
    __syncthreads();
    axis_dispatch<-1, 1>(s, nz, P, 1, y1, y2, tw + T.off_y, ny, tw, T);
    __syncthreads();
    axis_dispatch<-1, 0>(s, nz, P, 1, y1, y2, tw + T.off_y, ny, tw, T);
  }
};

// Plane geometry with compile-time sizes: ny = Y1 Y2, nz = Z1 Z2, NT threads.  The forward
// transform runs the z axis first and the inverse the z axis last, so that the z axis's step-0
// pass reads (forward) and writes (inverse) the plane in HBM directly; the y-axis passes and the
// z axis's step 1 run in shared memory.  Each axis leaves its spectrum in the same permuted order
// whichever axis runs first.
template <int Y1, int Y2, int Z1, int Z2, int NT>
struct GeoFixed {
  static constexpr bool kHbmPasses = true;
  static constexpr int NY = Y1 * Y2, NZ = Z1 * Z2, PP = NY | 1;
  int ny = NY, nz = NZ, y1 = Y1, y2 = Y2, z1 = Z1, z2 = Z2, P = PP;
  template <class ZeroFn>
  __device__ void forward_hbm(float2* s, float2* g, const float2* tw, const FftTab& T, ZeroFn zero) const {
    z_pass_hbm<1, NY, PP, Z1, Z2, NT>(s, g, tw + T.off_z, zero);
    __syncthreads();
    axis_pass_fixed<1, 1, NY, 1, PP, Z1, Z2, NT>(s, tw + T.off_z);
    __syncthreads();
    axis_pass_fixed<1, 0, NZ, PP, 1, Y1, Y2, NT>(s, tw + T.off_y);
    __syncthreads();
    axis_pass_fixed<1, 1, NZ, PP, 1, Y1, Y2, NT>(s, tw + T.off_y);
  }
  __device__ void inverse_hbm(float2* s, float2* g, const float2* tw, const FftTab& T) const {
    axis_pass_fixed<-1, 1, NZ, PP, 1, Y1, Y2, NT>(s, tw + T.off_y);
    __syncthreads();
    axis_pass_fixed<-1, 0, NZ, PP, 1, Y1, Y2, NT>(s, tw + T.off_y);
    __syncthreads();
    axis_pass_fixed<-1, 1, NY, 1, PP, Z1, Z2, NT>(s, tw + T.off_z);
    __syncthreads();
    z_pass_hbm<-1, NY, PP, Z1, Z2, NT>(s, g, tw + T.off_z, [](int, int) { return false; });
  }
};

template <class Geo>
__device__ __forceinline__ void fft_dc_body(const FftDcArgs& a, const Geo& geo) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int ny = geo.ny, nz = geo.nz, P = geo.P;
  const FftTab T = fft_tab(ny, nz);
  float2* tw = reinterpret_cast<float2*>(smem);
  double* red = reinterpret_cast<double*>(smem + align16b(sizeof(float2) * T.total));
  float2* s = reinterpret_cast<float2*>(smem + align16b(sizeof(float2) * T.total) + 32 * sizeof(double));
  // zero-fill tables: block column of every y, block row of every z (-1: no block), the shift,
  // and one flag per block of the current x slab
  int* zgy = reinterpret_cast<int*>(s + (size_t)P * nz);
  int* zgz = zgy + ny;
  int* zsh = zgz + nz;
  unsigned char* zfl = reinterpret_cast<unsigned char*>(smem + align16b(sizeof(float2) * T.total) +
                                                        32 * sizeof(double) + sizeof(float2) * (size_t)P * nz +
                                                        align16b(sizeof(int) * (size_t)(ny + nz + 4)));
  const bool zf = a.zero_ra != nullptr;
  const int tid = threadIdx.x;
  for (int i = tid; i < T.total; i += blockDim.x) tw[i] = a.twiddle[i];
  if (zf) {
    if (tid == 0) block_shift(a.zsrc, zsh);
    __syncthreads();
    const BlockSource& zs = a.zsrc;
    for (int y = tid; y < ny; y += blockDim.x) {
      int r = (y - zsh[1]) % ny;
      if (r < 0) r += ny;
      zgy[y] = r < zs.gy * zs.by ? r / zs.by : -1;
    }
    for (int z = tid; z < nz; z += blockDim.x) {
      int r = (z - zsh[2]) % nz;
      if (r < 0) r += nz;
      zgz[z] = r < zs.gz * zs.bz ? r / zs.bz : -1;
    }
  }
  // element (y, z) of the current plane lies in a block whose prox output was left unwritten
  // (the block column of the thread's y is cached: with a thread count that is a multiple of ny,
  // y never changes along a thread's elements)
  int zy = -1, zby = -1;
  auto zero_at = [&](int y, int z) {
    if (!zf) return false;
    if (y != zy) { zy = y; zby = zgy[y]; }
    const int bz = zgz[z];
    return zby >= 0 && bz >= 0 && zfl[zby + a.zsrc.gy * bz] != 0;
  };
  const long long nyz = (long long)ny * nz;
  const long long planes = (long long)a.nx * a.nq;
  const int dz = (int)blockDim.x / ny, dy = (int)blockDim.x - dz * ny;   // per-stride (z, y) step
  double err = 0.0;
  for (long long pl = blockIdx.x; pl < planes; pl += gridDim.x) {
    const int q = (int)(pl / a.nx), ix = (int)(pl - (long long)q * a.nx);
    float2* g = a.u + pl * nyz;
    __syncthreads();   // previous plane stored, twiddles visible
    if (zf) {          // flags of the blocks of this plane's x slab
      const BlockSource& zs = a.zsrc;
      int r = (ix - zsh[0]) % a.nx;
      if (r < 0) r += a.nx;
      const int gxi = r < zs.gx * zs.bx ? r / zs.bx : -1;
      const int nslab = zs.gy * zs.gz;
      for (int t = tid; t < nslab; t += blockDim.x)
        zfl[t] = gxi >= 0 && a.zero_ra[t + (long long)nslab * gxi] == 0;
      __syncthreads();
    }
    if constexpr (Geo::kHbmPasses) {
      // forward: z axis (its first pass loads the plane from HBM), then y axis
      geo.forward_hbm(s, g, tw, T, zero_at);
    } else {
      {   // asynchronous 8-byte copies: every element in flight at once, no register staging
        int z = tid / ny, y = tid - (tid / ny) * ny;
        for (int e = tid; e < ny * nz; e += blockDim.x) {
          const unsigned dst = (unsigned)__cvta_generic_to_shared(s + z * P + y);
          if (zero_at(y, z))
            s[z * P + y] = make_float2(0.f, 0.f);
          else
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst), "l"(g + e) : "memory");
          y += dy;
          z += dz;
          if (y >= ny) { y -= ny; ++z; }
        }
        asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;" ::: "memory");
      }
      __syncthreads();
      // forward: y axis (rows, element stride 1, batch stride P), then z axis (columns)
      geo.forward(s, tw, T);
    }
    __syncthreads();
    // hard DC on the sampled lines of this plane
    {
      const long long o0 = a.off[q], L = a.off[q + 1] - o0;
      const float2* yq = a.yhat + o0 * a.nx + (long long)ix * L;
      const int* pq = a.pos + o0;
      for (long long l = tid; l < L; l += blockDim.x) {
        const int p = pq[l];
        const int ky = p % ny, kz = p / ny;
        const int at = perm_pos(kz, geo.z1, geo.z2) * P + perm_pos(ky, geo.y1, geo.y2);
        const float2 yv = yq[l];
        const float2 uv = s[at];
        const double dx = (double)uv.x - (double)yv.x, dy2 = (double)uv.y - (double)yv.y;
        err += dx * dx + dy2 * dy2;
        s[at] = yv;
      }
    }
    __syncthreads();
    if constexpr (Geo::kHbmPasses) {
      // inverse: y axis, then z axis (its last pass stores the plane to HBM)
      geo.inverse_hbm(s, g, tw, T);
    } else {
      // inverse: z axis then y axis, each mirrored (step 1 then step 0)
      geo.inverse(s, tw, T);
      __syncthreads();
      int z = tid / ny, y = tid - (tid / ny) * ny;
      for (int e = tid; e < ny * nz; e += blockDim.x) {
        g[e] = s[z * P + y];
        y += dy;
        z += dz;
        if (y >= ny) { y -= ny; ++z; }
      }
    }
  }
  // deterministic CTA reduction of the residual
  for (int o = 16; o > 0; o >>= 1) err += __shfl_xor_sync(0xffffffffu, err, o);
  __syncthreads();
  if ((tid & 31) == 0) red[tid >> 5] = err;
  __syncthreads();
  if (tid == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    a.partials[blockIdx.x] = t;
  }
}

__global__ void __launch_bounds__(kFftThreads, 1) fft_dc_kernel(FftDcArgs a) {
  GeoRt geo;
  geo.ny = a.ny; geo.nz = a.nz; geo.y1 = a.y1; geo.y2 = a.y2; geo.z1 = a.z1; geo.z2 = a.z2; geo.P = a.pitch;
  fft_dc_body(a, geo);
}

template <int Y1, int Y2, int Z1, int Z2, int NT>
__global__ void __launch_bounds__(NT, 1) fft_dc_fixed_kernel(FftDcArgs a) {
  fft_dc_body(a, GeoFixed<Y1, Y2, Z1, Z2, NT>());
}

bool split_len(int n, int& n1, int& n2) {
  static const int R[] = {16, 12, 8, 6, 4, 3, 2};
  int best = -1;
  for (int a : R)
    for (int b : R)
      if (a * b == n) {
        const int bal = std::abs(a - b);
        if (best < 0 || bal < best) { best = bal; n1 = a; n2 = b; }
      }
  return best >= 0;
}

size_t fft_dc_smem(int ny, int nz, int pitch) {
  const FftTab T = fft_tab(ny, nz);
  return align16b(sizeof(float2) * T.total) + 32 * sizeof(double) + sizeof(float2) * (size_t)pitch * nz +
         align16b(sizeof(int) * (size_t)(ny + nz + 4)) + kZeroFlagMax;
}

}  // namespace

bool fft_dc_supported(int ny, int nz) {
  int a, b, c, d;
  if (!split_len(ny, a, b) || !split_len(nz, c, d)) return false;
  return fft_dc_smem(ny, nz, ny | 1) <= 227 * 1024;
}

// FP64 twiddle table for fft_dc_kernel (FftTab layout), uploaded once per context.
std::vector<float2> fft_dc_twiddles(int ny, int nz) {
  const FftTab T = fft_tab(ny, nz);
  std::vector<float2> h((size_t)T.total);
  auto fill = [&](int off, int N) {
    for (int j = 0; j < N; ++j) {
      const double ang = -2.0 * M_PI * (double)j / (double)N;
      h[(size_t)off + j] = make_float2((float)std::cos(ang), (float)std::sin(ang));
    }
  };
  fill(T.off_y, ny);
  fill(T.off_z, nz);
  fill(T.off_16, 16);
  fill(T.off_12, 12);
  fill(T.off_8, 8);
  fill(T.off_6, 6);
  return h;
}

namespace {

// Compile-time instances for the hot plane shapes; every other factorable shape uses the
// run-time kernel.  The pass loops stride by the thread count, so any count is correct.
struct FftKernelChoice {
  void (*kern)(FftDcArgs);
  int nt, y1, y2, z1, z2;
};

FftKernelChoice choose_fft(int ny, int nz) {
  FftKernelChoice c;
  // 192 x 96 fills a CTA's shared memory (one CTA per SM): 24 warps (the pass loops take the
  // 1152-task first pass in two rounds); the smaller planes run several CTAs per SM.
  if (ny == 192 && nz == 96) c = {fft_dc_fixed_kernel<16, 12, 12, 8, 768>, 768, 16, 12, 12, 8};
  else if (ny == 96 && nz == 48) c = {fft_dc_fixed_kernel<12, 8, 8, 6, 192>, 192, 12, 8, 8, 6};
  else if (ny == 64 && nz == 64) c = {fft_dc_fixed_kernel<8, 8, 8, 8, 256>, 256, 8, 8, 8, 8};
  else {
    c.kern = fft_dc_kernel;
    c.nt = kFftThreads;
    split_len(ny, c.y1, c.y2);
    split_len(nz, c.z1, c.z2);
  }
  return c;
}

}  // namespace

int fft_dc_grid(int ny, int nz) {
  int dev = 0, nsm = 0, smem_sm = 0, regs_sm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev) != cudaSuccess) return 0;
  const FftKernelChoice c = choose_fft(ny, nz);
  cudaFuncAttributes fa{};
  if (cudaFuncGetAttributes(&fa, c.kern) != cudaSuccess) return 0;
  const int by_smem = smem_sm / (int)(fft_dc_smem(ny, nz, ny | 1) + 1024);
  const int regs_warp = ((fa.numRegs * 32 + 255) / 256) * 256;
  const int by_regs = regs_sm / std::max(1, regs_warp * (c.nt / 32));
  const int per = std::max(1, std::min(4, std::min(by_smem, by_regs)));
  return nsm * per;
}

int launch_fft_dc(float2* u, const float2* yhat, const int* pos, const long long* off, const float2* twiddle,
                  const Geom& g, double* partials, int grid, const int* zero_ra, const BlockSource* zsrc,
                  cudaStream_t s) {
  FftDcArgs a;
  a.zero_ra = nullptr;
  a.zsrc = BlockSource{};
  if (zero_ra && zsrc && zsrc->kind == 1 && (long long)zsrc->gy * zsrc->gz <= kZeroFlagMax) {
    a.zero_ra = zero_ra;
    a.zsrc = *zsrc;
  }
  a.u = u; a.yhat = yhat; a.pos = pos; a.off = off; a.twiddle = twiddle; a.partials = partials;
  a.nx = g.nx; a.ny = g.ny; a.nz = g.nz; a.nq = g.nq;
  if (!fft_dc_supported(g.ny, g.nz))
    return set_error(LLR_ERR_UNSUPPORTED, "fused FFT: %d x %d plane is not supported", g.ny, g.nz);
  const FftKernelChoice c = choose_fft(g.ny, g.nz);
  a.y1 = c.y1; a.y2 = c.y2; a.z1 = c.z1; a.z2 = c.z2;
  a.pitch = g.ny | 1;
  const size_t smem = fft_dc_smem(g.ny, g.nz, a.pitch);
  LLR_CUDA_TRY(cudaFuncSetAttribute(c.kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  LLR_CUDA_TRY(cudaFuncSetAttribute(c.kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
  if (grid < 1) return set_error(LLR_ERR_INVALID, "fused FFT: empty grid");
  note_launch();
  c.kern<<<grid, c.nt, smem, s>>>(a);
  LLR_CUDA_TRY(cudaGetLastError());
  return LLR_OK;
}

}  // namespace llr
