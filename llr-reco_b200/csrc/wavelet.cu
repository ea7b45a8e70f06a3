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

// Analysis along `axis`: out extent 2*nc on that axis; optional shrink of everything
// except (when keep_corner) the approximation corner [0, nc_x) x [0, nc_y) x [0, nc_z).
__global__ void __launch_bounds__(256) analysis_kernel(View in, View out, int axis, int nc, Taps t, int nvol,
                                                       float alpha, int keep_corner, int ncx, int ncy, int ncz) {
  const long long ey = out.e[1], ez = out.e[2], ex = out.e[0];
  const long long tot = ex * ey * ez * nvol;
  const int n = in.e[axis];
  const int F = t.F;
  for (long long i = blockIdx.x * 256LL + threadIdx.x; i < tot; i += (long long)gridDim.x * 256) {
    long long r = i;
    const int iy = (int)(r % ey); r /= ey;
    const int iz = (int)(r % ez); r /= ez;
    const int ix = (int)(r % ex);
    const int v = (int)(r / ex);
    int c[3] = {ix, iy, iz};
    const int cc = c[axis];
    const bool det = cc >= nc;
    const int k = det ? cc - nc : cc;
    const float* f = det ? t.hi : t.lo;
    long long base = v * in.sv;
    for (int a = 0; a < 3; ++a)
      if (a != axis) base += (long long)c[a] * in.s[a];
    const long long st = in.s[axis];
    float2 acc = make_float2(0.f, 0.f);
    const int i0 = 2 * k - F + 2;
    for (int j = 0; j < F; ++j) {
      const int si = sym_index(i0 + j, n);
      const float2 x = in.p[base + (long long)si * st];
      const float w = f[F - 1 - j];
      acc.x = fmaf(w, x.x, acc.x);
      acc.y = fmaf(w, x.y, acc.y);
    }
    if (alpha > 0.f) {
      const bool corner = keep_corner && ix < ncx && iy < ncy && iz < ncz;
      if (!corner) {
        const float mag = sqrtf(acc.x * acc.x + acc.y * acc.y);
        const float sc = (mag > 0.f) ? fmaxf(mag - alpha, 0.f) / mag : 0.f;
        acc = cscale(acc, sc);
      }
    }
    out.p[v * out.sv + (long long)ix * out.s[0] + (long long)iy * out.s[1] + (long long)iz * out.s[2]] = acc;
  }
}

// Synthesis along `axis`: in extent 2*nc on that axis, out extent n_out.
__global__ void __launch_bounds__(256) synthesis_kernel(View in, View out, int axis, int nc, Taps t, int nvol,
                                                        StoreXf xf) {
  const long long ey = out.e[1], ez = out.e[2], ex = out.e[0];
  const long long tot = ex * ey * ez * nvol;
  const int F = t.F;
  const int start = F - 2;
  for (long long i = blockIdx.x * 256LL + threadIdx.x; i < tot; i += (long long)gridDim.x * 256) {
    long long r = i;
    const int iy = (int)(r % ey); r /= ey;
    const int iz = (int)(r % ez); r /= ez;
    const int ix = (int)(r % ex);
    const int v = (int)(r / ex);
    int c[3] = {ix, iy, iz};
    const int s = c[axis];
    long long base = v * in.sv;
    for (int a = 0; a < 3; ++a)
      if (a != axis) base += (long long)c[a] * in.s[a];
    const long long st = in.s[axis];
    float2 acc = make_float2(0.f, 0.f);
    const int cidx = start + s;
    for (int j = 0; j < F; ++j) {
      const int idx = cidx - j;
      if (idx >= 0 && idx < 2 * nc && (idx & 1) == 0) {
        const int h = idx >> 1;
        const float2 av = in.p[base + (long long)h * st];
        const float2 dv = in.p[base + (long long)(h + nc) * st];
        acc.x = fmaf(t.lo[j], av.x, acc.x); acc.y = fmaf(t.lo[j], av.y, acc.y);
        acc.x = fmaf(t.hi[j], dv.x, acc.x); acc.y = fmaf(t.hi[j], dv.y, acc.y);
      }
    }
    if (xf.on) acc = cscale(cmul(acc, phase_at(xf.ph, xf.g, xf.q0 + v, ix, iy, iz)), xf.scale);
    out.p[v * out.sv + (long long)ix * out.s[0] + (long long)iy * out.s[1] + (long long)iz * out.s[2]] = acc;
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
  for (int l = 0; l < p.levels; ++l) {
    const size_t d = (size_t)2 * p.sizes[3 * (l + 1)] * 2 * p.sizes[3 * (l + 1) + 1] * 2 * p.sizes[3 * (l + 1) + 2];
    per += d;
  }
  const int* e0 = &p.sizes[0];
  const int* c0 = &p.sizes[3];
  per += (size_t)2 * c0[0] * e0[1] * e0[2];          // T1
  per += (size_t)2 * c0[0] * 2 * c0[1] * e0[2];      // T2
  return per * nvol;
}

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
  StoreXf none;
  memset(&none, 0, sizeof(none));
  StoreXf xf = none;
  if (g) { xf.on = 1; xf.ph = ph; xf.g = *g; xf.q0 = q0; xf.scale = store_scale; }
  const int L = p.levels;
  if (L == 0) return set_error(LLR_ERR_UNSUPPORTED, "wavelet level count is 0 for this volume");
  // carve the workspace
  std::vector<View> D(L);
  float2* cur = work;
  for (int l = 0; l < L; ++l) {
    const int* c = &p.sizes[3 * (l + 1)];
    D[l] = work_view(cur, 2 * c[0], 2 * c[1], 2 * c[2]);
    cur += (size_t)D[l].sv * nvol;
  }
  const int* e0 = &p.sizes[0];
  const int* c0 = &p.sizes[3];
  float2* t1base = cur;
  float2* t2base = t1base + (size_t)2 * c0[0] * e0[1] * e0[2] * nvol;

  // analysis
  View in = vol;
  for (int l = 0; l < L; ++l) {
    const int* e = &p.sizes[3 * l];
    const int* c = &p.sizes[3 * (l + 1)];
    View T1 = work_view(t1base, 2 * c[0], e[1], e[2]);
    View T2 = work_view(t2base, 2 * c[0], 2 * c[1], e[2]);
    note_launch();
    analysis_kernel<<<grid_for((long long)T1.sv * nvol), 256, 0, s>>>(in, T1, 0, c[0], td, nvol, 0.f, 0, 0, 0, 0);
    note_launch();
    analysis_kernel<<<grid_for((long long)T2.sv * nvol), 256, 0, s>>>(T1, T2, 1, c[1], td, nvol, 0.f, 0, 0, 0, 0);
    const int last = (l == L - 1);
    note_launch();
    analysis_kernel<<<grid_for((long long)D[l].sv * nvol), 256, 0, s>>>(T2, D[l], 2, c[2], td, nvol, alpha, !last,
                                                                         c[0], c[1], c[2]);
    LLR_CUDA_TRY(cudaGetLastError());
    // next input: approximation corner of D[l]
    in = D[l];
    in.e[0] = c[0]; in.e[1] = c[1]; in.e[2] = c[2];
  }
  // synthesis
  for (int l = L - 1; l >= 0; --l) {
    const int* e = &p.sizes[3 * l];
    const int* c = &p.sizes[3 * (l + 1)];
    View T1 = work_view(t1base, 2 * c[0], e[1], e[2]);
    View T2 = work_view(t2base, 2 * c[0], 2 * c[1], e[2]);
    note_launch();
    synthesis_kernel<<<grid_for((long long)T2.sv * nvol), 256, 0, s>>>(D[l], T2, 2, c[2], tr, nvol, none);
    note_launch();
    synthesis_kernel<<<grid_for((long long)T1.sv * nvol), 256, 0, s>>>(T2, T1, 1, c[1], tr, nvol, none);
    View out;
    if (l > 0) {
      out = D[l - 1];
      out.e[0] = e[0]; out.e[1] = e[1]; out.e[2] = e[2];
      note_launch();
      synthesis_kernel<<<grid_for((long long)e[0] * e[1] * e[2] * nvol), 256, 0, s>>>(T1, out, 0, c[0], tr, nvol, none);
    } else {
      out = vol;
      note_launch();
      synthesis_kernel<<<grid_for((long long)e[0] * e[1] * e[2] * nvol), 256, 0, s>>>(T1, out, 0, c[0], tr, nvol, xf);
    }
    LLR_CUDA_TRY(cudaGetLastError());
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
