// Multi-level 3-D orthogonal Daubechies wavelet shrink (lib.rs:430-465) on the device.
//
// One level = three separable analysis passes (x, y, z) with the half-sample symmetric
// extension and sub-band length floor((n + F - 1) / 2) of kernels.cu:97-212; after the
// last level every sub-band is soft-shrunk (fused into each level's z pass, except the
// approximation corner of non-final levels, which the next level consumes and the
// synthesis overwrites); synthesis runs z, y, x per level (kernels.cu:215-268,
// cudwt3.rs:185-219), writing each level's reconstruction straight into the parent's
// approximation corner.  Storage keeps y fastest so warps read contiguous runs.
#include <cstring>
#include <cstdlib>
#include <cmath>
#include <algorithm>

#include "llr_internal.h"

namespace llr {

namespace {

struct Taps {
  float lo[20];
  float hi[20];
  int F;
};

struct View {
  float2* p;
  long long s[3];   // strides of x, y, z
  long long sv;     // stride between volumes
  int e[3];         // extents
};

struct StoreXf {
  int on;           // multiply by phase on store
  PhaseTab ph;
  Geom g;
  int q0;           // volume offset of this batch
  float scale;      // store scale
};

__device__ __forceinline__ int sym_index(int i, int n) {
  if (i < 0) i = -i - 1;
  if (i >= n) i = 2 * n - i - 1;
  return i;
}

// Half-sample symmetric extension (kernels.cu:97-105), folded with period 2n so that any index
// maps into [0, n) (one reflection, the reference's, whenever n >= F - 1).
__device__ __forceinline__ int msym(int i, int n) {
  const int p = 2 * n;
  i %= p;
  if (i < 0) i += p;
  return i < n ? i : p - 1 - i;
}

// ---------------------------------------------------------------------------------------
// Fused one-level analysis: the three separable filter passes of a level in one kernel.
// A CTA owns a kWT x kWT tile of (y, z) coefficient positions of one volume and a chunk of x
// coefficients.  It walks the input planes along x: each (y, z) input tile (with the filter
// halo) is staged in shared memory, filtered along y then z, and the four yz sub-band values
// of each position go to a per-thread ring of the last F planes; an x coefficient is formed
// from the ring when its last plane has arrived, shrunk, and its eight sub-bands are stored.
// The next plane's tile is loaded into registers while the current one is filtered.
// Input is read once (plus the halo of the tile, mostly from L2), output written once.
// ---------------------------------------------------------------------------------------
constexpr int kWT = 16;                 // analysis coefficient tile (y, z)
constexpr int kWS = 32;                 // synthesis sample tile (y, z)
constexpr int kWaveThreads = 256;

template <int F>
struct AnaShape {
  static constexpr int IY = 2 * kWT + F - 2;                         // staged input tile edge
  static constexpr int NIN = IY * IY;
  static constexpr int PER = (NIN + kWaveThreads - 1) / kWaveThreads;
  static constexpr size_t smem = sizeof(float2) * ((size_t)NIN + (size_t)IY * 2 * kWT + (size_t)F * 4 * kWaveThreads);
};

template <int F>
__global__ void __launch_bounds__(kWaveThreads) wave_analysis_kernel(View in, View out, Taps t, int kchunk, int nchunk,
                                                                     float alpha, int keep_corner) {
  constexpr int IY = AnaShape<F>::IY, NIN = AnaShape<F>::NIN, PER = AnaShape<F>::PER;
  extern __shared__ float2 wsm[];
  float2* tile = wsm;                       // [IY z][IY y]
  float2* yp = tile + NIN;                  // [IY z][2 kWT]: y low-pass then y high-pass
  float2* ring = yp + IY * 2 * kWT;         // [F][4][threads], thread-private columns
  __shared__ float flo[F], fhi[F];
  const int tid = threadIdx.x;
  if (tid < F) { flo[tid] = t.lo[F - 1 - tid]; fhi[tid] = t.hi[F - 1 - tid]; }   // reversed: tap j uses f[F-1-j]
  const int cx = out.e[0] / 2, cy = out.e[1] / 2, cz = out.e[2] / 2;
  const int ky0 = blockIdx.x * kWT, kz0 = blockIdx.y * kWT;
  const int v = blockIdx.z / nchunk, ch = blockIdx.z - v * nchunk;
  const int kx0 = ch * kchunk, kx1 = min(cx, kx0 + kchunk);
  const int nxi = in.e[0], nyi = in.e[1], nzi = in.e[2];
  const float2* base = in.p + (long long)v * in.sv;
  int off[PER];   // element offsets inside one plane of one volume (< 2^31, checked by the host)
#pragma unroll
  for (int r = 0; r < PER; ++r) {
    const int e = min(tid + r * kWaveThreads, NIN - 1);
    const int ly = e % IY, lz = e / IY;
    off[r] = msym(2 * ky0 - F + 2 + ly, nyi) * (int)in.s[1] + msym(2 * kz0 - F + 2 + lz, nzi) * (int)in.s[2];
  }
  const int i0 = 2 * kx0 - F + 2, i1 = 2 * kx1 - 1;   // virtual input planes [i0, i1]
  float2 pre[PER];
  {
    const float2* pl = base + (long long)msym(i0, nxi) * in.s[0];
#pragma unroll
    for (int r = 0; r < PER; ++r) pre[r] = pl[off[r]];
  }
  const int ty = tid % kWT, tz = tid / kWT;
  const int ky = ky0 + ty, kz = kz0 + tz;
  for (int i = i0; i <= i1; ++i) {
#pragma unroll
    for (int r = 0; r < PER; ++r)
      if (tid + r * kWaveThreads < NIN) tile[tid + r * kWaveThreads] = pre[r];
    __syncthreads();
    if (i < i1) {
      const float2* pl = base + (long long)msym(i + 1, nxi) * in.s[0];
#pragma unroll
      for (int r = 0; r < PER; ++r) pre[r] = pl[off[r]];
    }
    // y pass: yp[z][b * kWT + k] = sum_j f_b[F-1-j] tile[z][2k + j]
    for (int e = tid; e < IY * 2 * kWT; e += kWaveThreads) {
      const int z = e / (2 * kWT), kk = e - z * 2 * kWT;
      const int b = kk / kWT, k = kk - b * kWT;
      const float* f = b ? fhi : flo;
      const float2* row = tile + z * IY + 2 * k;
      float2 a = make_float2(0.f, 0.f);
#pragma unroll
      for (int j = 0; j < F; ++j) {
        const float2 x = row[j];
        a.x = fmaf(f[j], x.x, a.x);
        a.y = fmaf(f[j], x.y, a.y);
      }
      yp[e] = a;
    }
    __syncthreads();
    // z pass: four yz sub-bands of this thread's (ky, kz) position into the ring
    const int slot = (i - i0) % F;
#pragma unroll
    for (int yb = 0; yb < 2; ++yb) {
      float2 lo = make_float2(0.f, 0.f), hi = make_float2(0.f, 0.f);
#pragma unroll
      for (int j = 0; j < F; ++j) {
        const float2 x = yp[(2 * tz + j) * 2 * kWT + yb * kWT + ty];
        lo.x = fmaf(flo[j], x.x, lo.x); lo.y = fmaf(flo[j], x.y, lo.y);
        hi.x = fmaf(fhi[j], x.x, hi.x); hi.y = fmaf(fhi[j], x.y, hi.y);
      }
      ring[(slot * 4 + yb) * kWaveThreads + tid] = lo;        // (y band, z low)
      ring[(slot * 4 + 2 + yb) * kWaveThreads + tid] = hi;    // (y band, z high)
    }
    // x coefficient kx is complete when plane 2 kx + 1 has arrived
    const int d = i - i0 - (F - 1);
    if (d >= 0 && (d & 1) == 0 && ky < cy && kz < cz) {
      const int kx = kx0 + d / 2;
#pragma unroll
      for (int sb = 0; sb < 4; ++sb) {
        float2 lo = make_float2(0.f, 0.f), hi = make_float2(0.f, 0.f);
#pragma unroll
        for (int j = 0; j < F; ++j) {
          const float2 x = ring[(((d + j) % F) * 4 + sb) * kWaveThreads + tid];
          lo.x = fmaf(flo[j], x.x, lo.x); lo.y = fmaf(flo[j], x.y, lo.y);
          hi.x = fmaf(fhi[j], x.x, hi.x); hi.y = fmaf(fhi[j], x.y, hi.y);
        }
        const int yb = sb & 1, zb = sb >> 1;
        const long long o = (long long)v * out.sv + (long long)(ky + yb * cy) * out.s[1] +
                            (long long)(kz + zb * cz) * out.s[2];
        if (alpha > 0.f) {
          const bool corner = keep_corner && sb == 0;
          if (!corner) {
            const float m = sqrtf(lo.x * lo.x + lo.y * lo.y);
            lo = cscale(lo, m > 0.f ? fmaxf(m - alpha, 0.f) / m : 0.f);
          }
          const float m = sqrtf(hi.x * hi.x + hi.y * hi.y);
          hi = cscale(hi, m > 0.f ? fmaxf(m - alpha, 0.f) / m : 0.f);
        }
        out.p[o + (long long)kx * out.s[0]] = lo;
        out.p[o + (long long)(kx + cx) * out.s[0]] = hi;
      }
    }
  }
}

// ---------------------------------------------------------------------------------------
// Fused one-level synthesis (kernels.cu:215-268 per axis: upsample, filter, keep the centre).
// A CTA owns a kWS x kWS tile of (y, z) output samples of one volume and a chunk of x samples.
// It walks the coefficient planes h along x; for each, the eight sub-band tiles it needs
// (x low / high, yz sub-bands, with the filter halo) are staged, synthesised along z then y,
// and the two resulting sample tiles (x low and x high) go to a per-thread ring of the last
// F/2 planes; x sample s is formed when its last coefficient plane has arrived and stored
// with the optional phase / scale of the caller.
// ---------------------------------------------------------------------------------------
template <int F>
struct SynShape {
  static constexpr int HY = kWS / 2 + F / 2;                          // coefficient rows per sub-band
  static constexpr int NCO = 8 * HY * HY;                             // staged coefficients
  static constexpr int PER = (NCO + kWaveThreads - 1) / kWaveThreads;
  static constexpr int R = F / 2;                                     // ring depth (planes)
  static constexpr int SPT = kWS * kWS / kWaveThreads;                // samples per thread
  static constexpr size_t smem =
      sizeof(float2) * ((size_t)NCO + (size_t)4 * HY * kWS + (size_t)R * 2 * SPT * kWaveThreads);
};

template <int F>
__global__ void __launch_bounds__(kWaveThreads) wave_synthesis_kernel(View in, View out, Taps t, int schunk,
                                                                      int nchunk, StoreXf xf) {
  constexpr int HY = SynShape<F>::HY, NCO = SynShape<F>::NCO, PER = SynShape<F>::PER, R = SynShape<F>::R,
                SPT = SynShape<F>::SPT;
  extern __shared__ float2 wsm[];
  float2* co = wsm;                         // [xb][zb][yb][HY z][HY y]
  float2* zs = co + NCO;                    // [xb][yb][kWS z][HY y]  (z synthesised)
  float2* ring = zs + 4 * HY * kWS;         // [R][xb][SPT][threads]
  __shared__ float flo[F], fhi[F];
  const int tid = threadIdx.x;
  if (tid < F) { flo[tid] = t.lo[tid]; fhi[tid] = t.hi[tid]; }
  const int cx = in.e[0] / 2, cy = in.e[1] / 2, cz = in.e[2] / 2;
  const int nx = out.e[0], ny = out.e[1], nz = out.e[2];
  const int sy0 = blockIdx.x * kWS, sz0 = blockIdx.y * kWS;
  const int v = blockIdx.z / nchunk, ch = blockIdx.z - v * nchunk;
  const int s0 = ch * schunk, s1 = min(nx, s0 + schunk);
  // output sample s takes taps j with idx = (F - 2) + s - j even, 0 <= idx < 2 c: h = idx / 2
  const int hy0 = sy0 / 2, hz0 = sz0 / 2;   // first coefficient row of the tile (y, z)
  const float2* base = in.p + (long long)v * in.sv;
  int off[PER];   // element offsets inside one volume (< 2^31, checked by the host); -1: outside
#pragma unroll
  for (int r = 0; r < PER; ++r) {
    const int e = tid + r * kWaveThreads;
    const int ly = e % HY, rest = e / HY, lz = rest % HY, sb = rest / HY;   // sb = xb*4 + zb*2 + yb
    const int yb = sb & 1, zb = (sb >> 1) & 1, xb = sb >> 2;
    const int h_y = hy0 + ly, h_z = hz0 + lz;
    off[r] = (e < NCO && h_y < cy && h_z < cz)
                 ? (h_y + yb * cy) * (int)in.s[1] + (h_z + zb * cz) * (int)in.s[2] + xb * cx * (int)in.s[0]
                 : -1;
  }
  const int h0 = s0 / 2, h1 = min(cx - 1, (s1 - 1 + F - 2) / 2);
  float2 pre[PER];
  {
    const float2* pl = base + (long long)h0 * in.s[0];
#pragma unroll
    for (int r = 0; r < PER; ++r) pre[r] = off[r] >= 0 ? pl[off[r]] : make_float2(0.f, 0.f);
  }
  for (int h = h0; h <= h1; ++h) {
#pragma unroll
    for (int r = 0; r < PER; ++r)
      if (tid + r * kWaveThreads < NCO) co[tid + r * kWaveThreads] = pre[r];
    __syncthreads();
    if (h < h1) {
      const float2* pl = base + (long long)(h + 1) * in.s[0];
#pragma unroll
      for (int r = 0; r < PER; ++r) pre[r] = off[r] >= 0 ? pl[off[r]] : make_float2(0.f, 0.f);
    }
    // z synthesis: zs[xb][yb][sz][ly] = sum over taps of lo_r * co[xb][0][yb] + hi_r * co[xb][1][yb]
    for (int e = tid; e < 4 * HY * kWS; e += kWaveThreads) {
      const int ly = e % HY, rest = e / HY, sz = rest % kWS, xy = rest / kWS;   // xy = xb * 2 + yb
      const int s = sz0 + sz;
      const int xb = xy >> 1, yb = xy & 1;
      float2 a = make_float2(0.f, 0.f);
#pragma unroll
      for (int jj = 0; jj < F / 2; ++jj) {   // taps with F - 2 + s - j even: j = (s & 1) + 2 jj
        const int j = (s & 1) + 2 * jj;
        const int idx = F - 2 + s - j;
        if (idx >= 0 && idx < 2 * cz) {
          const int lz = idx / 2 - hz0;
          const float2 cl = co[(((xb * 2 + 0) * 2 + yb) * HY + lz) * HY + ly];
          const float2 chh = co[(((xb * 2 + 1) * 2 + yb) * HY + lz) * HY + ly];
          a.x = fmaf(flo[j], cl.x, a.x); a.y = fmaf(flo[j], cl.y, a.y);
          a.x = fmaf(fhi[j], chh.x, a.x); a.y = fmaf(fhi[j], chh.y, a.y);
        }
      }
      zs[e] = a;
    }
    __syncthreads();
    // y synthesis into the ring slot of plane h
    const int slot = h % R;
#pragma unroll
    for (int q = 0; q < SPT; ++q) {
      const int e = tid + q * kWaveThreads;
      const int sy = e % kWS, sz = e / kWS;
      const int s = sy0 + sy;
#pragma unroll
      for (int xb = 0; xb < 2; ++xb) {
        float2 a = make_float2(0.f, 0.f);
#pragma unroll
        for (int jj = 0; jj < F / 2; ++jj) {
          const int j = (s & 1) + 2 * jj;
          const int idx = F - 2 + s - j;
          if (idx >= 0 && idx < 2 * cy) {
            const int ly = idx / 2 - hy0;
            const float2 cl = zs[((xb * 2 + 0) * kWS + sz) * HY + ly];
            const float2 chh = zs[((xb * 2 + 1) * kWS + sz) * HY + ly];
            a.x = fmaf(flo[j], cl.x, a.x); a.y = fmaf(flo[j], cl.y, a.y);
            a.x = fmaf(fhi[j], chh.x, a.x); a.y = fmaf(fhi[j], chh.y, a.y);
          }
        }
        ring[((slot * 2 + xb) * SPT + q) * kWaveThreads + tid] = a;
      }
    }
    // x samples whose last coefficient plane is h: hmax(s) = min(cx - 1, (s + F - 2) / 2) == h
    const int s_hi = (h == cx - 1) ? s1 - 1 : min(s1 - 1, 2 * h - F + 3);
    for (int s = max(s0, 2 * h - F + 2); s <= s_hi; ++s) {
      if (min(cx - 1, (s + F - 2) / 2) != h) continue;
#pragma unroll
      for (int q = 0; q < SPT; ++q) {
        const int e = tid + q * kWaveThreads;
        const int sy = e % kWS, sz = e / kWS;
        const int iy = sy0 + sy, iz = sz0 + sz;
        float2 a = make_float2(0.f, 0.f);
#pragma unroll
        for (int jj = 0; jj < F / 2; ++jj) {
          const int j = (s & 1) + 2 * jj;
          const int idx = F - 2 + s - j;
          if (idx >= 0 && idx < 2 * cx) {
            const int hh = idx / 2;
            const float2 cl = ring[(((hh % R) * 2 + 0) * SPT + q) * kWaveThreads + tid];
            const float2 chh = ring[(((hh % R) * 2 + 1) * SPT + q) * kWaveThreads + tid];
            a.x = fmaf(flo[j], cl.x, a.x); a.y = fmaf(flo[j], cl.y, a.y);
            a.x = fmaf(fhi[j], chh.x, a.x); a.y = fmaf(fhi[j], chh.y, a.y);
          }
        }
        if (iy < ny && iz < nz) {
          if (xf.on) a = cscale(cmul(a, phase_at(xf.ph, xf.g, xf.q0 + v, s, iy, iz)), xf.scale);
          out.p[(long long)v * out.sv + (long long)s * out.s[0] + (long long)iy * out.s[1] + (long long)iz * out.s[2]] = a;
        }
      }
    }
  }
}

// Work array with y fastest, then z, then x, then volume.
View work_view(float2* p, int ex, int ey, int ez) {
  View v;
  v.p = p;
  v.e[0] = ex; v.e[1] = ey; v.e[2] = ez;
  v.s[1] = 1; v.s[2] = ey; v.s[0] = (long long)ey * ez;
  v.sv = (long long)ex * ey * ez;
  return v;
}

unsigned grid_for(long long n) {
  long long b = (n + 255) / 256;
  return (unsigned)std::max<long long>(1, std::min<long long>(b, 148LL * 64));
}

}  // namespace

// Daubechies taps (reconstruction low-pass, sum = sqrt(2)) by spectral factorisation,
// computed in double and cached per order.  See daubechies_host() in host_api.cu.
int daubechies_host(int order, double* h);

int wavelet_plan_init(WaveletPlan* p, int nx, int ny, int nz, int moments, int levels) {
  double h[20];
  LLR_TRY(daubechies_host(moments, h));
  const int F = 2 * moments;
  if (F > 16) return set_error(LLR_ERR_UNSUPPORTED, "wavelet shrink supports Daubechies orders 1..8, not %d", moments);
  p->flen = F;
  for (int k = 0; k < F; ++k) {
    const double lr = h[k];
    const double hr = ((k & 1) ? -1.0 : 1.0) * h[F - 1 - k];
    p->lo_r[k] = (float)lr;
    p->hi_r[k] = (float)hr;
  }
  for (int k = 0; k < F; ++k) {
    p->lo_d[k] = p->lo_r[F - 1 - k];
    p->hi_d[k] = p->hi_r[F - 1 - k];
  }
  p->nx = nx; p->ny = ny; p->nz = nz;
  if (levels <= 0) {
    const int mn = std::min(nx, std::min(ny, nz));
    levels = (mn < F - 1) ? 0 : (int)std::floor(std::log2((double)mn / (double)(F - 1)));
  }
  p->levels = levels;
  p->sizes.assign(3 * (levels + 1), 0);
  p->sizes[0] = nx; p->sizes[1] = ny; p->sizes[2] = nz;
  for (int l = 0; l < levels; ++l)
    for (int a = 0; a < 3; ++a) p->sizes[3 * (l + 1) + a] = (p->sizes[3 * l + a] + F - 1) / 2;
  return LLR_OK;
}

size_t wavelet_workspace_elems(const WaveletPlan& p, int nvol) {
  if (p.levels == 0) return 0;
  size_t per = 0;
  for (int l = 0; l < p.levels; ++l)
    per += (size_t)2 * p.sizes[3 * (l + 1)] * 2 * p.sizes[3 * (l + 1) + 1] * 2 * p.sizes[3 * (l + 1) + 2];
  return per * nvol;
}

namespace {

template <int F>
int launch_analysis(const View& in, const View& out, const Taps& t, int nvol, float alpha, int keep_corner,
                    cudaStream_t s) {
  const int cx = out.e[0] / 2, cy = out.e[1] / 2, cz = out.e[2] / 2;
  const long long tiles = (long long)((cy + kWT - 1) / kWT) * ((cz + kWT - 1) / kWT) * nvol;
  const long long want = std::min<long long>(cx, std::max<long long>(1, (148LL * 8 + tiles - 1) / tiles));
  const int kchunk = std::max((int)((cx + want - 1) / want), std::min(cx, 2 * F));
  const int nchunk = (cx + kchunk - 1) / kchunk;
  if ((long long)nvol * nchunk > 65535) return set_error(LLR_ERR_UNSUPPORTED, "too many wavelet volumes");
  auto kern = wave_analysis_kernel<F>;
  const size_t sm = AnaShape<F>::smem;
  LLR_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  dim3 grid((cy + kWT - 1) / kWT, (cz + kWT - 1) / kWT, nvol * nchunk);
  note_launch();
  kern<<<grid, kWaveThreads, sm, s>>>(in, out, t, kchunk, nchunk, alpha, keep_corner);
  LLR_CUDA_TRY(cudaGetLastError());
  return LLR_OK;
}

template <int F>
int launch_synthesis(const View& in, const View& out, const Taps& t, int nvol, const StoreXf& xf, cudaStream_t s) {
  const int nx = out.e[0], ny = out.e[1], nz = out.e[2];
  const long long tiles = (long long)((ny + kWS - 1) / kWS) * ((nz + kWS - 1) / kWS) * nvol;
  const long long want = std::min<long long>(nx, std::max<long long>(1, (148LL * 8 + tiles - 1) / tiles));
  const int schunk = std::max((int)((nx + want - 1) / want), std::min(nx, 2 * F));
  const int nchunk = (nx + schunk - 1) / schunk;
  if ((long long)nvol * nchunk > 65535) return set_error(LLR_ERR_UNSUPPORTED, "too many wavelet volumes");
  auto kern = wave_synthesis_kernel<F>;
  const size_t sm = SynShape<F>::smem;
  LLR_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  dim3 grid((ny + kWS - 1) / kWS, (nz + kWS - 1) / kWS, nvol * nchunk);
  note_launch();
  kern<<<grid, kWaveThreads, sm, s>>>(in, out, t, schunk, nchunk, xf);
  LLR_CUDA_TRY(cudaGetLastError());
  return LLR_OK;
}

int analysis_level(int F, const View& in, const View& out, const Taps& t, int nvol, float alpha, int keep_corner,
                   cudaStream_t s) {
  switch (F) {
    case 2: return launch_analysis<2>(in, out, t, nvol, alpha, keep_corner, s);
    case 4: return launch_analysis<4>(in, out, t, nvol, alpha, keep_corner, s);
    case 6: return launch_analysis<6>(in, out, t, nvol, alpha, keep_corner, s);
    case 8: return launch_analysis<8>(in, out, t, nvol, alpha, keep_corner, s);
    case 10: return launch_analysis<10>(in, out, t, nvol, alpha, keep_corner, s);
    case 12: return launch_analysis<12>(in, out, t, nvol, alpha, keep_corner, s);
    case 14: return launch_analysis<14>(in, out, t, nvol, alpha, keep_corner, s);
    case 16: return launch_analysis<16>(in, out, t, nvol, alpha, keep_corner, s);
    default: return set_error(LLR_ERR_UNSUPPORTED, "wavelet filter length %d (Daubechies order above 8)", F);
  }
}

int synthesis_level(int F, const View& in, const View& out, const Taps& t, int nvol, const StoreXf& xf,
                    cudaStream_t s) {
  switch (F) {
    case 2: return launch_synthesis<2>(in, out, t, nvol, xf, s);
    case 4: return launch_synthesis<4>(in, out, t, nvol, xf, s);
    case 6: return launch_synthesis<6>(in, out, t, nvol, xf, s);
    case 8: return launch_synthesis<8>(in, out, t, nvol, xf, s);
    case 10: return launch_synthesis<10>(in, out, t, nvol, xf, s);
    case 12: return launch_synthesis<12>(in, out, t, nvol, xf, s);
    case 14: return launch_synthesis<14>(in, out, t, nvol, xf, s);
    case 16: return launch_synthesis<16>(in, out, t, nvol, xf, s);
    default: return set_error(LLR_ERR_UNSUPPORTED, "wavelet filter length %d (Daubechies order above 8)", F);
  }
}

}  // namespace

// Multi-level shrink: per level one fused analysis kernel (shrink fused; the approximation
// of non-final levels is kept for the next level), then per level, coarsest first, one fused
// synthesis kernel writing into the parent's approximation corner (level 0: the volumes,
// with the caller's phase / scale).
int wavelet_denoise_strided_xf(const WaveletPlan& p, float2* data, long long sx, long long sy, long long sz,
                               long long sv, int nvol, float alpha, float2* work, PhaseTab ph, const Geom* g,
                               int q0, float store_scale, cudaStream_t s) {
  Taps td, tr;
  td.F = tr.F = p.flen;
  for (int k = 0; k < p.flen; ++k) {
    td.lo[k] = p.lo_d[k]; td.hi[k] = p.hi_d[k];
    tr.lo[k] = p.lo_r[k]; tr.hi[k] = p.hi_r[k];
  }
  View vol;
  vol.p = data; vol.s[0] = sx; vol.s[1] = sy; vol.s[2] = sz; vol.sv = sv;
  vol.e[0] = p.nx; vol.e[1] = p.ny; vol.e[2] = p.nz;
  if ((long long)(p.nx - 1) * std::llabs(sx) + (long long)(p.ny - 1) * std::llabs(sy) +
          (long long)(p.nz - 1) * std::llabs(sz) >= (1LL << 30))
    return set_error(LLR_ERR_UNSUPPORTED, "wavelet volume of more than 2^30 elements");
  StoreXf none;
  memset(&none, 0, sizeof(none));
  StoreXf xf = none;
  if (g) { xf.on = 1; xf.ph = ph; xf.g = *g; xf.q0 = q0; xf.scale = store_scale; }
  const int L = p.levels;
  if (L == 0) return set_error(LLR_ERR_UNSUPPORTED, "wavelet level count is 0 for this volume");
  std::vector<View> D(L);
  float2* cur = work;
  for (int l = 0; l < L; ++l) {
    const int* c = &p.sizes[3 * (l + 1)];
    D[l] = work_view(cur, 2 * c[0], 2 * c[1], 2 * c[2]);
    cur += (size_t)D[l].sv * nvol;
  }
  View in = vol;
  for (int l = 0; l < L; ++l) {
    const int* c = &p.sizes[3 * (l + 1)];
    LLR_TRY(analysis_level(p.flen, in, D[l], td, nvol, alpha, l < L - 1 ? 1 : 0, s));
    in = D[l];
    in.e[0] = c[0]; in.e[1] = c[1]; in.e[2] = c[2];
  }
  for (int l = L - 1; l >= 0; --l) {
    const int* e = &p.sizes[3 * l];
    View out;
    if (l > 0) {
      out = D[l - 1];
      out.e[0] = e[0]; out.e[1] = e[1]; out.e[2] = e[2];
    } else {
      out = vol;
    }
    LLR_TRY(synthesis_level(p.flen, D[l], out, tr, nvol, l > 0 ? none : xf, s));
  }
  return LLR_OK;
}

int wavelet_denoise_strided(const WaveletPlan& p, float2* data, long long sx, long long sy, long long sz, long long sv,
                            int nvol, float alpha, float2* work, cudaStream_t s) {
  PhaseTab none{nullptr, nullptr, nullptr};
  return wavelet_denoise_strided_xf(p, data, sx, sy, sz, sv, nvol, alpha, work, none, nullptr, 0, 1.f, s);
}

// ---------------------------------------------------------------------------------------
// Single-level, single-axis analysis / synthesis with the reference's argument shapes
// (dwt3_axis / idwt3_axis, kernels.cu:155-348), x-fastest volumes, optional circular
// shift applied per axis.
// ---------------------------------------------------------------------------------------
namespace {

// Taps and shift come from the kernel arguments, or, when d_lo / d_sh are non-null, from
// device memory (the reference's native interface passes device filter and shift pointers,
// kernels.cu:155-156, 215-216).
__device__ __forceinline__ void load_taps_shift(const Taps& t, const float* d_lo, const float* d_hi, const int* d_sh,
                                                int s0, int s1, int s2, float* lo, float* hi, int* sh) {
  if (threadIdx.x < (unsigned)t.F) {
    lo[threadIdx.x] = d_lo ? d_lo[threadIdx.x] : t.lo[threadIdx.x];
    hi[threadIdx.x] = d_hi ? d_hi[threadIdx.x] : t.hi[threadIdx.x];
  }
  if (threadIdx.x == 0) {
    sh[0] = d_sh ? d_sh[0] : s0;
    sh[1] = d_sh ? d_sh[1] : s1;
    sh[2] = d_sh ? d_sh[2] : s2;
  }
  __syncthreads();
}

__global__ void dwt_axis_ref_kernel(const float2* __restrict__ vol, float2* __restrict__ dec, int vx, int vy, int vz,
                                    int dx, int dy, int dz, int axis, Taps t, int s0, int s1, int s2,
                                    const float* d_lo, const float* d_hi, const int* d_sh) {
  __shared__ float lo[20], hi[20];
  __shared__ int sh[3];
  load_taps_shift(t, d_lo, d_hi, d_sh, s0, s1, s2, lo, hi, sh);
  const long long tot = (long long)dx * dy * dz;
  const int vs[3] = {vx, vy, vz};
  const int n = vs[axis];
  const int nc = (n + t.F - 1) / 2;
  for (long long i = blockIdx.x * 256LL + threadIdx.x; i < tot; i += (long long)gridDim.x * 256) {
    int c[3];
    c[0] = (int)(i % dx);
    c[1] = (int)((i / dx) % dy);
    c[2] = (int)(i / ((long long)dx * dy));
    const int cc = c[axis];
    if (cc >= 2 * nc) continue;
    const bool det = cc >= nc;
    const int k = det ? cc - nc : cc;
    const float* f = det ? hi : lo;
    float2 acc = make_float2(0.f, 0.f);
    for (int j = 0; j < t.F; ++j) {
      int p[3] = {c[0], c[1], c[2]};
      p[axis] = sym_index(2 * k - t.F + 2 + j, n);
      // circular shift per axis
      for (int a = 0; a < 3; ++a) {
        int v = (p[a] + sh[a]) % vs[a];
        p[a] = v < 0 ? v + vs[a] : v;
      }
      const float2 x = vol[p[0] + (long long)vx * (p[1] + (long long)vy * p[2])];
      const float w = f[t.F - 1 - j];
      acc.x = fmaf(w, x.x, acc.x);
      acc.y = fmaf(w, x.y, acc.y);
    }
    dec[i] = acc;
  }
}

__global__ void idwt_axis_ref_kernel(float2* __restrict__ vol, const float2* __restrict__ dec, int vx, int vy, int vz,
                                     int dx, int dy, int dz, int axis, Taps t, int s0, int s1, int s2,
                                     const float* d_lo, const float* d_hi, const int* d_sh) {
  __shared__ float lo[20], hi[20];
  __shared__ int sh[3];
  load_taps_shift(t, d_lo, d_hi, d_sh, s0, s1, s2, lo, hi, sh);
  const long long tot = (long long)vx * vy * vz;
  const int ds[3] = {dx, dy, dz};
  const int vs[3] = {vx, vy, vz};
  const int nc = ds[axis] / 2;
  const int start = t.F - 2;
  for (long long i = blockIdx.x * 256LL + threadIdx.x; i < tot; i += (long long)gridDim.x * 256) {
    int c[3];
    c[0] = (int)(i % vx);
    c[1] = (int)((i / vx) % vy);
    c[2] = (int)(i / ((long long)vx * vy));
    const int s = c[axis];
    float2 acc = make_float2(0.f, 0.f);
    for (int j = 0; j < t.F; ++j) {
      const int idx = start + s - j;
      if (idx >= 0 && idx < 2 * nc && (idx & 1) == 0) {
        int p[3] = {c[0], c[1], c[2]};
        p[axis] = idx >> 1;
        const float2 av = dec[p[0] + (long long)dx * (p[1] + (long long)dy * p[2])];
        p[axis] = (idx >> 1) + nc;
        const float2 dv = dec[p[0] + (long long)dx * (p[1] + (long long)dy * p[2])];
        acc.x = fmaf(lo[j], av.x, acc.x); acc.y = fmaf(lo[j], av.y, acc.y);
        acc.x = fmaf(hi[j], dv.x, acc.x); acc.y = fmaf(hi[j], dv.y, acc.y);
      }
    }
    int p[3];
    for (int a = 0; a < 3; ++a) {
      int v = (c[a] + sh[a]) % vs[a];
      p[a] = v < 0 ? v + vs[a] : v;
    }
    vol[p[0] + (long long)vx * (p[1] + (long long)vy * p[2])] = acc;
  }
}

}  // namespace

int launch_dwt_axis_ref(const float2* vol, float2* dec, const uint32_t* vs, const uint32_t* ds, int axis,
                        const float* lo, const float* hi, int F, const int* sh, int inverse, cudaStream_t s,
                        const float* d_lo, const float* d_hi, const int* d_sh) {
  if (F < 2 || F > 20) return set_error(LLR_ERR_INVALID, "filter length %d outside [2, 20]", F);
  Taps t;
  t.F = F;
  for (int k = 0; k < F; ++k) {
    t.lo[k] = lo ? lo[k] : 0.f;
    t.hi[k] = hi ? hi[k] : 0.f;
  }
  const int s0 = sh ? sh[0] : 0, s1 = sh ? sh[1] : 0, s2 = sh ? sh[2] : 0;
  if (!inverse) {
    const long long tot = (long long)ds[0] * ds[1] * ds[2];
    note_launch();
    dwt_axis_ref_kernel<<<grid_for(tot), 256, 0, s>>>(vol, dec, vs[0], vs[1], vs[2], ds[0], ds[1], ds[2], axis, t, s0,
                                                      s1, s2, d_lo, d_hi, d_sh);
  } else {
    const long long tot = (long long)vs[0] * vs[1] * vs[2];
    note_launch();
    idwt_axis_ref_kernel<<<grid_for(tot), 256, 0, s>>>(const_cast<float2*>(vol), dec, vs[0], vs[1], vs[2], ds[0],
                                                       ds[1], ds[2], axis, t, s0, s1, s2, d_lo, d_hi, d_sh);
  }
  LLR_CUDA_TRY(cudaGetLastError());
  return LLR_OK;
}

}  // namespace llr
