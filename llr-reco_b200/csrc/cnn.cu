// Learned warm start: a small 3-D residual CNN (conv3d 3x3x3, zero padding, ReLU between
// layers, out = in + net(in)) with hand-written forward, backward-data and backward-weight
// kernels, mean-squared-error loss and Adam.  BF16 weights feed the convolutions with FP32
// accumulation; the optimizer keeps FP32 master weights.
//
// Activations are channels-last FP32, voxel v = x + nx (y + ny z) (the reference image order,
// x fastest).  Forward:  y[v][co] = b[co] + sum_{tap, ci} W[tap][ci][co] x[v + d(tap) - 1][ci],
// tap = dx + 3 (dy + 3 dz).  The input gradient is the same convolution of dy with
// W'[tap][co][ci] = W[26 - tap][ci][co]; the weight gradient is a reduction over voxels with
// per-CTA partial sums added in a fixed order (deterministic).
//
// The network runs on subspace coefficients: 2 r real channels per voxel (re/im of c = x S,
// S the nq x r temporal subspace, dti_subspace.rs:141-166); the warm-start image is c S^H
// (dti_subspace.rs:172-207).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>
#include <algorithm>

#include "llr_common.cuh"
#include "llr_internal.h"

struct llr_cnn {
  int device;
  int n_layers;
  std::vector<int> cin, cout;
  std::vector<long long> w_off, b_off;   // offsets of W and b in the flat parameter array
  long long n_params;
  float* d_master;                       // FP32 parameters (W [27][cin][cout], then b [cout])
  float* d_grad;
  float* d_m;
  float* d_v;
  uint16_t* d_wb;                        // BF16 W per layer, same layout as the master
  uint16_t* d_wt;                        // BF16 W' per layer: [tap][cout][cin], taps flipped
  long long step;
  // activation workspace (grown on demand)
  long long cap_vox;
  std::vector<float*> act;               // act[l]: input of layer l (act[0] = network input)
  float* d_g0;
  float* d_g1;                           // gradient ping-pong buffers
  float* d_out;
  float* d_part;                         // weight-gradient partial sums
  long long part_cap;
  double* d_loss;                        // loss partial sums
  int loss_cap;
};

namespace llr {

namespace {

constexpr int kTX = 8, kTY = 8, kTZ = 4;                      // output tile
constexpr int kHX = kTX + 2, kHY = kTY + 2, kHZ = kTZ + 2;     // input halo tile
constexpr int kHV = kHX * kHY * kHZ;
constexpr int kTV = kTX * kTY * kTZ;
constexpr int kConvThreads = 128;                              // two voxels (z, z + 2) per thread
constexpr int kWgThreads = 288;

__host__ __device__ constexpr int odd_pitch(int c) { return c | 1; }
__host__ __device__ constexpr int pad4(int c) { return (c + 3) & ~3; }

__device__ __forceinline__ float bf16_to_f32(uint16_t h) { return __uint_as_float((uint32_t)h << 16); }

__host__ __device__ __forceinline__ uint16_t f32_to_bf16(float f) {
#ifdef __CUDA_ARCH__
  uint32_t u = __float_as_uint(f);
#else
  uint32_t u;
  memcpy(&u, &f, 4);
#endif
  if ((u & 0x7f800000u) == 0x7f800000u) return (uint16_t)((u >> 16) | ((u & 0xffffu) ? 0x40u : 0u));
  u += 0x7fffu + ((u >> 16) & 1u);   // round to nearest even
  return (uint16_t)(u >> 16);
}

struct TileGeo {
  int nx, ny, nz, tx, ty;   // volume and tile counts along x, y
  __device__ void origin(long long tile, int& ox, int& oy, int& oz) const {
    const int ix = (int)(tile % tx);
    const long long r = tile / tx;
    const int iy = (int)(r % ty);
    const int iz = (int)(r / ty);
    ox = ix * kTX; oy = iy * kTY; oz = iz * kTZ;
  }
};

// halo tile of C channels -> s[hv * CP + c], zero outside the volume
template <int C>
__device__ __forceinline__ void load_halo(const float* __restrict__ x, float* s, const TileGeo& G, int ox, int oy,
                                          int oz) {
  constexpr int CP = odd_pitch(C);
  for (int i = threadIdx.x; i < kHV * C; i += blockDim.x) {
    const int hv = i / C, c = i - hv * C;
    const int hx = hv % kHX, hy = (hv / kHX) % kHY, hz = hv / (kHX * kHY);
    const int gx = ox + hx - 1, gy = oy + hy - 1, gz = oz + hz - 1;
    float v = 0.f;
    if (gx >= 0 && gx < G.nx && gy >= 0 && gy < G.ny && gz >= 0 && gz < G.nz)
      v = x[((long long)gx + (long long)G.nx * (gy + (long long)G.ny * gz)) * C + c];
    s[hv * CP + c] = v;
  }
}

// y = [add +] act(b + conv(x, W)); W in BF16 [27][CIN][COUT].
template <int CIN, int COUT>
__global__ void __launch_bounds__(kConvThreads) conv3d_kernel(const float* __restrict__ x, const uint16_t* __restrict__ wb,
                                                              const float* __restrict__ bias, const float* __restrict__ add,
                                                              float* __restrict__ y, TileGeo G, int relu) {
  constexpr int CP = odd_pitch(CIN), COP = pad4(COUT);
  extern __shared__ __align__(16) float smem_f[];
  float* s_w = smem_f;                    // [27][CIN][COP]
  float* s_in = smem_f + 27 * CIN * COP;  // [kHV][CP]
  for (int i = threadIdx.x; i < 27 * CIN * COP; i += blockDim.x) {
    const int co = i % COP, tc = i / COP;
    s_w[i] = co < COUT ? bf16_to_f32(wb[tc * COUT + co]) : 0.f;
  }
  int ox, oy, oz;
  G.origin(blockIdx.x, ox, oy, oz);
  load_halo<CIN>(x, s_in, G, ox, oy, oz);
  __syncthreads();
  const int t = threadIdx.x;
  const int lx = t & 7, ly = (t >> 3) & 7, lz = t >> 6;
  float acc0[COP], acc1[COP];
#pragma unroll
  for (int c = 0; c < COP; ++c) {
    const float b0 = (bias && c < COUT) ? bias[c] : 0.f;
    acc0[c] = b0;
    acc1[c] = b0;
  }
  for (int dz = 0; dz < 3; ++dz)
    for (int dy = 0; dy < 3; ++dy)
#pragma unroll 1
      for (int dx = 0; dx < 3; ++dx) {
        const int hv0 = ((lz + dz) * kHY + (ly + dy)) * kHX + lx + dx;
        const float* p0 = s_in + hv0 * CP;
        const float* p1 = p0 + 2 * kHX * kHY * CP;
        const float* pw = s_w + (dx + 3 * (dy + 3 * dz)) * CIN * COP;
#pragma unroll 4
        for (int ci = 0; ci < CIN; ++ci) {
          const float xa = p0[ci], xb = p1[ci];
          const float4* w4 = reinterpret_cast<const float4*>(pw + ci * COP);
#pragma unroll
          for (int c4 = 0; c4 < COP / 4; ++c4) {
            const float4 w = w4[c4];
            acc0[4 * c4 + 0] = fmaf(xa, w.x, acc0[4 * c4 + 0]);
            acc0[4 * c4 + 1] = fmaf(xa, w.y, acc0[4 * c4 + 1]);
            acc0[4 * c4 + 2] = fmaf(xa, w.z, acc0[4 * c4 + 2]);
            acc0[4 * c4 + 3] = fmaf(xa, w.w, acc0[4 * c4 + 3]);
            acc1[4 * c4 + 0] = fmaf(xb, w.x, acc1[4 * c4 + 0]);
            acc1[4 * c4 + 1] = fmaf(xb, w.y, acc1[4 * c4 + 1]);
            acc1[4 * c4 + 2] = fmaf(xb, w.z, acc1[4 * c4 + 2]);
            acc1[4 * c4 + 3] = fmaf(xb, w.w, acc1[4 * c4 + 3]);
          }
        }
      }
  auto store = [&](const float (&a)[COP], int gz) {
    const int gx = ox + lx, gy = oy + ly;
    if (gx >= G.nx || gy >= G.ny || gz >= G.nz) return;
    const long long v = (long long)gx + (long long)G.nx * (gy + (long long)G.ny * gz);
#pragma unroll
    for (int c = 0; c < COUT; ++c) {
      float val = a[c];
      if (relu) val = fmaxf(val, 0.f);
      if (add) val += add[v * COUT + c];
      y[v * COUT + c] = val;
    }
  };
  store(acc0, oz + lz);
  store(acc1, oz + lz + 2);
}

// Partial weight (and bias) gradients of one conv layer over the CTA's tiles:
// dW[tap][ci][co] = sum_v x[v + d(tap) - 1][ci] dy[v][co], db[co] = sum_v dy[v][co].
template <int CIN, int COUT>
__global__ void __launch_bounds__(kWgThreads) conv3d_wgrad_kernel(const float* __restrict__ x,
                                                                  const float* __restrict__ dy, float* __restrict__ part,
                                                                  TileGeo G, long long ntiles) {
  constexpr int CP = odd_pitch(CIN), COP = pad4(COUT);
  constexpr int NP = 27 * CIN;
  constexpr int PPT = (NP + kWgThreads - 1) / kWgThreads;
  extern __shared__ __align__(16) float smem_f[];
  float* s_dy = smem_f;              // [kTV][COP]
  float* s_in = smem_f + kTV * COP;  // [kHV][CP]
  const int t = threadIdx.x;
  int hoff[PPT], cidx[PPT];
#pragma unroll
  for (int k = 0; k < PPT; ++k) {
    const int p = t + kWgThreads * k;
    const int tap = p < NP ? p / CIN : 0;
    cidx[k] = p < NP ? p - tap * CIN : -1;
    const int dx = tap % 3, dyy = (tap / 3) % 3, dz = tap / 9;
    hoff[k] = (dz * kHY + dyy) * kHX + dx;
  }
  float acc[PPT][COUT];
#pragma unroll
  for (int k = 0; k < PPT; ++k)
#pragma unroll
    for (int c = 0; c < COUT; ++c) acc[k][c] = 0.f;
  float dbacc = 0.f;
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    int ox, oy, oz;
    G.origin(tile, ox, oy, oz);
    __syncthreads();
    load_halo<CIN>(x, s_in, G, ox, oy, oz);
    for (int i = t; i < kTV * COP; i += blockDim.x) {
      const int lv = i / COP, c = i - lv * COP;
      const int gx = ox + (lv & 7), gy = oy + ((lv >> 3) & 7), gz = oz + (lv >> 6);
      float v = 0.f;
      if (c < COUT && gx < G.nx && gy < G.ny && gz < G.nz)
        v = dy[((long long)gx + (long long)G.nx * (gy + (long long)G.ny * gz)) * COUT + c];
      s_dy[i] = v;
    }
    __syncthreads();
#pragma unroll 1
    for (int lv = 0; lv < kTV; ++lv) {
      const int hb = ((lv >> 6) * kHY + ((lv >> 3) & 7)) * kHX + (lv & 7);
      float d[COP];
#pragma unroll
      for (int c4 = 0; c4 < COP / 4; ++c4) {
        const float4 w = reinterpret_cast<const float4*>(s_dy + lv * COP)[c4];
        d[4 * c4] = w.x; d[4 * c4 + 1] = w.y; d[4 * c4 + 2] = w.z; d[4 * c4 + 3] = w.w;
      }
#pragma unroll
      for (int k = 0; k < PPT; ++k) {
        if (cidx[k] < 0) continue;
        const float xv = s_in[(hb + hoff[k]) * CP + cidx[k]];
#pragma unroll
        for (int c = 0; c < COUT; ++c) acc[k][c] = fmaf(xv, d[c], acc[k][c]);
      }
      if (t < COUT) dbacc += s_dy[lv * COP + t];
    }
  }
  float* P = part + (long long)blockIdx.x * (NP * COUT + COUT);
#pragma unroll
  for (int k = 0; k < PPT; ++k) {
    const int p = t + kWgThreads * k;
    if (p < NP)
#pragma unroll
      for (int c = 0; c < COUT; ++c) P[(long long)p * COUT + c] = acc[k][c];
  }
  if (t < COUT) P[NP * COUT + t] = dbacc;
}

// out[i] = sum over `nb` partial blocks (fixed order), i < n
__global__ void reduce_partials_kernel(const float* __restrict__ part, int nb, long long n, float* __restrict__ out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int b = 0; b < nb; ++b) s += part[(long long)b * n + i];
    out[i] = (float)s;
  }
}

__global__ void relu_mask_kernel(float* __restrict__ g, const float* __restrict__ a, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    if (!(a[i] > 0.f)) g[i] = 0.f;
}

// g = 2 (out - tgt) / n; per-CTA partial sum of (out - tgt)^2 in FP64
__global__ void __launch_bounds__(256) mse_kernel(const float* __restrict__ out, const float* __restrict__ tgt,
                                                  float* __restrict__ g, long long n, double* part) {
  __shared__ double sh[8];
  double s = 0.0;
  const float sc = 2.f / (float)n;
  for (long long i = blockIdx.x * 256LL + threadIdx.x; i < n; i += (long long)gridDim.x * 256) {
    const float d = out[i] - tgt[i];
    s += (double)d * d;
    g[i] = sc * d;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < 8; ++w) t += sh[w];
    part[blockIdx.x] = t;
  }
}

__global__ void adam_kernel(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, long long n, float lr, float b1, float b2, float eps, float c1,
                            float c2) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
  }
}

// BF16 copies of one layer's weights: wb = W, wt[tap][co][ci] = W[26 - tap][ci][co]
__global__ void pack_weights_kernel(const float* __restrict__ W, uint16_t* __restrict__ wb, uint16_t* __restrict__ wt,
                                    int cin, int cout) {
  const int n = 27 * cin * cout;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int co = i % cout, r = i / cout, ci = r % cin, tap = r / cin;
    const uint16_t h = f32_to_bf16(W[i]);
    wb[i] = h;
    wt[((26 - tap) * cout + co) * cin + ci] = h;
  }
}

// counter-based normal draws (Box-Muller on SplitMix64 uniforms)
__global__ void init_weights_kernel(float* __restrict__ W, int n, float stdv, uint64_t seed, uint64_t stream) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint64_t a = llr_rng_u64(seed, stream, 2ull * i), b = llr_rng_u64(seed, stream, 2ull * i + 1);
    const double u1 = ((double)(a >> 11) + 0.5) * (1.0 / 9007199254740992.0);
    const double u2 = (double)(b >> 11) * (1.0 / 9007199254740992.0);
    W[i] = (float)(stdv * sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2));
  }
}

// chan[v][2k + {0, 1}] = scale * (re, im) of sum_q x[v + V q] S[q + nq k]
__global__ void subspace_channels_kernel(const float2* __restrict__ x, long long V, int nq, const float2* __restrict__ S,
                                         int r, float scale, float* __restrict__ chan) {
  extern __shared__ float2 sS[];
  for (int i = threadIdx.x; i < nq * r; i += blockDim.x) sS[i] = S[i];
  __syncthreads();
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < V; v += (long long)gridDim.x * blockDim.x) {
    float2 c[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) c[k] = make_float2(0.f, 0.f);
    for (int q = 0; q < nq; ++q) {
      const float2 xv = x[v + V * q];
#pragma unroll
      for (int k = 0; k < 16; ++k)
        if (k < r) cfma(c[k], xv, sS[q + nq * k]);
    }
#pragma unroll
    for (int k = 0; k < 16; ++k)
      if (k < r) {
        chan[v * 2 * r + 2 * k] = scale * c[k].x;
        chan[v * 2 * r + 2 * k + 1] = scale * c[k].y;
      }
  }
}

// x[v + V q] (+)= (1 / scale) sum_k c_k conj(S[q + nq k])
__global__ void subspace_image_kernel(const float* __restrict__ chan, long long V, int nq, const float2* __restrict__ S,
                                      int r, float inv_scale, float2* __restrict__ x, int accumulate) {
  extern __shared__ float2 sS[];
  for (int i = threadIdx.x; i < nq * r; i += blockDim.x) sS[i] = S[i];
  __syncthreads();
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < V; v += (long long)gridDim.x * blockDim.x) {
    float2 c[16];
#pragma unroll
    for (int k = 0; k < 16; ++k)
      c[k] = k < r ? make_float2(chan[v * 2 * r + 2 * k] * inv_scale, chan[v * 2 * r + 2 * k + 1] * inv_scale)
                   : make_float2(0.f, 0.f);
    for (int q = 0; q < nq; ++q) {
      float2 acc = make_float2(0.f, 0.f);
#pragma unroll
      for (int k = 0; k < 16; ++k)
        if (k < r) cfma_cb(acc, c[k], sS[q + nq * k]);
      if (accumulate) acc = cadd(acc, x[v + V * q]);
      x[v + V * q] = acc;
    }
  }
}

int grid_1d(long long n, int threads = 256) {
  return (int)std::max<long long>(1, std::min<long long>((n + threads - 1) / threads, 148LL * 16));
}

bool conv_shape_ok(int cin, int cout) {
  return (cin == 14 && cout == 32) || (cin == 32 && cout == 32) || (cin == 32 && cout == 14);
}

template <int CIN, int COUT>
size_t conv_smem() {
  return sizeof(float) * (27 * CIN * pad4(COUT) + kHV * odd_pitch(CIN));
}
template <int CIN, int COUT>
size_t wgrad_smem() {
  return sizeof(float) * (kTV * pad4(COUT) + kHV * odd_pitch(CIN));
}

TileGeo tile_geo(const int* dims) {
  TileGeo G;
  G.nx = dims[0]; G.ny = dims[1]; G.nz = dims[2];
  G.tx = (G.nx + kTX - 1) / kTX;
  G.ty = (G.ny + kTY - 1) / kTY;
  return G;
}
long long tile_count(const int* dims) {
  return (long long)((dims[0] + kTX - 1) / kTX) * ((dims[1] + kTY - 1) / kTY) * ((dims[2] + kTZ - 1) / kTZ);
}

template <int CIN, int COUT>
int conv_inst(const float* x, const uint16_t* w, const float* b, const float* add, float* y, const int* dims, int relu,
              cudaStream_t s) {
  const size_t smem = conv_smem<CIN, COUT>();
  auto k = conv3d_kernel<CIN, COUT>;
  LLR_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const long long nt = tile_count(dims);
  note_launch();
  k<<<(unsigned)nt, kConvThreads, smem, s>>>(x, w, b, add, y, tile_geo(dims), relu);
  LLR_CUDA_TRY(cudaGetLastError());
  return LLR_OK;
}

int conv(int cin, int cout, const float* x, const uint16_t* w, const float* b, const float* add, float* y,
         const int* dims, int relu, cudaStream_t s) {
  if (cin == 14 && cout == 32) return conv_inst<14, 32>(x, w, b, add, y, dims, relu, s);
  if (cin == 32 && cout == 32) return conv_inst<32, 32>(x, w, b, add, y, dims, relu, s);
  if (cin == 32 && cout == 14) return conv_inst<32, 14>(x, w, b, add, y, dims, relu, s);
  return set_error(LLR_ERR_UNSUPPORTED, "conv3d %d -> %d channels is not built", cin, cout);
}

template <int CIN, int COUT>
int wgrad_inst(const float* x, const float* dy, float* part, long long part_cap, float* out, const int* dims,
               cudaStream_t s) {
  const size_t smem = wgrad_smem<CIN, COUT>();
  auto k = conv3d_wgrad_kernel<CIN, COUT>;
  LLR_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int dev = 0, nsm = 0;
  LLR_CUDA_TRY(cudaGetDevice(&dev));
  LLR_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  const long long nt = tile_count(dims);
  const long long per = 27LL * CIN * COUT + COUT;
  const int grid = (int)std::max<long long>(1, std::min<long long>(std::min<long long>(nt, 2LL * nsm), part_cap / per));
  note_launch();
  k<<<grid, kWgThreads, smem, s>>>(x, dy, part, tile_geo(dims), nt);
  LLR_CUDA_TRY(cudaGetLastError());
  note_launch();
  reduce_partials_kernel<<<grid_1d(per), 256, 0, s>>>(part, grid, per, out);
  LLR_CUDA_TRY(cudaGetLastError());
  return LLR_OK;
}

int wgrad(int cin, int cout, const float* x, const float* dy, float* part, long long cap, float* out, const int* dims,
          cudaStream_t s) {
  if (cin == 14 && cout == 32) return wgrad_inst<14, 32>(x, dy, part, cap, out, dims, s);
  if (cin == 32 && cout == 32) return wgrad_inst<32, 32>(x, dy, part, cap, out, dims, s);
  if (cin == 32 && cout == 14) return wgrad_inst<32, 14>(x, dy, part, cap, out, dims, s);
  return set_error(LLR_ERR_UNSUPPORTED, "conv3d %d -> %d channels is not built", cin, cout);
}

int pack_all(llr_cnn* n, cudaStream_t s) {
  long long wt_off = 0;
  for (int l = 0; l < n->n_layers; ++l) {
    note_launch();
    pack_weights_kernel<<<grid_1d(27LL * n->cin[l] * n->cout[l]), 256, 0, s>>>(
        n->d_master + n->w_off[l], n->d_wb + wt_off, n->d_wt + wt_off, n->cin[l], n->cout[l]);
    LLR_CUDA_TRY(cudaGetLastError());
    wt_off += 27LL * n->cin[l] * n->cout[l];
  }
  return LLR_OK;
}

long long wtab_off(const llr_cnn* n, int l) {
  long long o = 0;
  for (int i = 0; i < l; ++i) o += 27LL * n->cin[i] * n->cout[i];
  return o;
}

int ensure_workspace(llr_cnn* n, long long vox) {
  if (vox <= n->cap_vox) return LLR_OK;
  for (int l = 1; l < (int)n->act.size(); ++l) if (n->act[l]) cudaFree(n->act[l]);   // act[0] is the caller's
  if (n->d_g0) cudaFree(n->d_g0);
  if (n->d_g1) cudaFree(n->d_g1);
  if (n->d_out) cudaFree(n->d_out);
  n->act.assign(n->n_layers, nullptr);
  n->d_g0 = n->d_g1 = n->d_out = nullptr;
  n->cap_vox = 0;
  int cmax = 0;
  for (int l = 0; l < n->n_layers; ++l) cmax = std::max(cmax, std::max(n->cin[l], n->cout[l]));
  for (int l = 1; l < n->n_layers; ++l)
    LLR_CUDA_TRY(cudaMalloc((void**)&n->act[l], sizeof(float) * vox * n->cin[l]));
  LLR_CUDA_TRY(cudaMalloc((void**)&n->d_g0, sizeof(float) * vox * cmax));
  LLR_CUDA_TRY(cudaMalloc((void**)&n->d_g1, sizeof(float) * vox * cmax));
  LLR_CUDA_TRY(cudaMalloc((void**)&n->d_out, sizeof(float) * vox * n->cout.back()));
  n->cap_vox = vox;
  return LLR_OK;
}

// forward through every layer; act[l] keeps each layer's input (act[0] = in)
int forward(llr_cnn* n, const float* in, float* out, const int* dims, cudaStream_t s) {
  n->act[0] = const_cast<float*>(in);
  for (int l = 0; l < n->n_layers; ++l) {
    const bool last = l + 1 == n->n_layers;
    float* y = last ? out : n->act[l + 1];
    LLR_TRY(conv(n->cin[l], n->cout[l], n->act[l], n->d_wb + wtab_off(n, l), n->d_master + n->b_off[l],
                 last ? in : nullptr, y, dims, last ? 0 : 1, s));
  }
  return LLR_OK;
}

int check_dims(const int* dims) {
  if (!dims || dims[0] < 1 || dims[1] < 1 || dims[2] < 1) return set_error(LLR_ERR_INVALID, "bad volume dims");
  return LLR_OK;
}

}  // namespace

}  // namespace llr

using namespace llr;

extern "C" {

int llr_cnn_create(int32_t n_layers, const int32_t* channels, int32_t device, uint64_t seed, llr_cnn** out) {
  if (!out || !channels || n_layers < 1) return set_error(LLR_ERR_INVALID, "bad network description");
  *out = nullptr;
  if (channels[0] != channels[n_layers]) return set_error(LLR_ERR_INVALID, "residual network: in and out channels differ");
  for (int l = 0; l < n_layers; ++l)
    if (!conv_shape_ok(channels[l], channels[l + 1]))
      return set_error(LLR_ERR_UNSUPPORTED, "conv3d %d -> %d channels is not built (14->32, 32->32, 32->14)",
                       channels[l], channels[l + 1]);
  LLR_CUDA_TRY(cudaSetDevice(device));
  llr_cnn* n = new (std::nothrow) llr_cnn();
  if (!n) return set_error(LLR_ERR_NOMEM, "host allocation failed");
  n->device = device;
  n->n_layers = n_layers;
  long long off = 0, wtot = 0;
  for (int l = 0; l < n_layers; ++l) {
    n->cin.push_back(channels[l]);
    n->cout.push_back(channels[l + 1]);
    n->w_off.push_back(off);
    off += 27LL * channels[l] * channels[l + 1];
    n->b_off.push_back(off);
    off += channels[l + 1];
    wtot += 27LL * channels[l] * channels[l + 1];
  }
  n->n_params = off;
  n->act.assign(n_layers, nullptr);
  auto fail = [&](int st) { llr_cnn_destroy(n); return st; };
  cudaError_t e = cudaSuccess;
  if (e == cudaSuccess) e = cudaMalloc((void**)&n->d_master, sizeof(float) * off);
  if (e == cudaSuccess) e = cudaMalloc((void**)&n->d_grad, sizeof(float) * off);
  if (e == cudaSuccess) e = cudaMalloc((void**)&n->d_m, sizeof(float) * off);
  if (e == cudaSuccess) e = cudaMalloc((void**)&n->d_v, sizeof(float) * off);
  if (e == cudaSuccess) e = cudaMalloc((void**)&n->d_wb, sizeof(uint16_t) * wtot);
  if (e == cudaSuccess) e = cudaMalloc((void**)&n->d_wt, sizeof(uint16_t) * wtot);
  n->loss_cap = 148 * 16;
  if (e == cudaSuccess) e = cudaMalloc((void**)&n->d_loss, sizeof(double) * n->loss_cap);
  long long maxw = 0;
  for (int l = 0; l < n_layers; ++l) maxw = std::max(maxw, 27LL * channels[l] * channels[l + 1] + channels[l + 1]);
  n->part_cap = maxw * 2 * 148;
  if (e == cudaSuccess) e = cudaMalloc((void**)&n->d_part, sizeof(float) * n->part_cap);
  if (e != cudaSuccess) return fail(cuda_error(e, "cudaMalloc", __FILE__, __LINE__));
  e = cudaMemset(n->d_master, 0, sizeof(float) * off);
  if (e == cudaSuccess) e = cudaMemset(n->d_m, 0, sizeof(float) * off);
  if (e == cudaSuccess) e = cudaMemset(n->d_v, 0, sizeof(float) * off);
  if (e == cudaSuccess) e = cudaMemset(n->d_grad, 0, sizeof(float) * off);
  if (e != cudaSuccess) return fail(cuda_error(e, "cudaMemset", __FILE__, __LINE__));
  // He-normal weights (the last layer scaled by 0.1 so that the network starts near identity)
  for (int l = 0; l < n_layers; ++l) {
    const int nw = 27 * channels[l] * channels[l + 1];
    float sd = (float)std::sqrt(2.0 / (27.0 * channels[l]));
    if (l + 1 == n_layers) sd *= 0.1f;
    note_launch();
    init_weights_kernel<<<grid_1d(nw), 256>>>(n->d_master + n->w_off[l], nw, sd, seed, 0x434E4EULL + l);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(cuda_error(e, "init_weights_kernel", __FILE__, __LINE__));
  }
  int st = pack_all(n, nullptr);
  if (st == LLR_OK) {
    e = cudaDeviceSynchronize();
    if (e != cudaSuccess) st = cuda_error(e, "cudaDeviceSynchronize", __FILE__, __LINE__);
  }
  if (st != LLR_OK) return fail(st);
  *out = n;
  return LLR_OK;
}

int llr_cnn_destroy(llr_cnn* n) {
  if (!n) return LLR_OK;
  cudaSetDevice(n->device);
  for (int l = 1; l < (int)n->act.size(); ++l) if (n->act[l]) cudaFree(n->act[l]);
  for (void* p : {(void*)n->d_master, (void*)n->d_grad, (void*)n->d_m, (void*)n->d_v, (void*)n->d_wb, (void*)n->d_wt,
                  (void*)n->d_g0, (void*)n->d_g1, (void*)n->d_out, (void*)n->d_part, (void*)n->d_loss})
    if (p) cudaFree(p);
  delete n;
  return LLR_OK;
}

int llr_cnn_param_count(const llr_cnn* n, int64_t* count) {
  if (!n || !count) return set_error(LLR_ERR_INVALID, "null pointer");
  *count = n->n_params;
  return LLR_OK;
}

int llr_cnn_get_params(llr_cnn* n, float* host) {
  if (!n || !host) return set_error(LLR_ERR_INVALID, "null pointer");
  LLR_CUDA_TRY(cudaSetDevice(n->device));
  LLR_CUDA_TRY(cudaMemcpy(host, n->d_master, sizeof(float) * n->n_params, cudaMemcpyDeviceToHost));
  return LLR_OK;
}

int llr_cnn_set_params(llr_cnn* n, const float* host) {
  if (!n || !host) return set_error(LLR_ERR_INVALID, "null pointer");
  LLR_CUDA_TRY(cudaSetDevice(n->device));
  LLR_CUDA_TRY(cudaMemcpy(n->d_master, host, sizeof(float) * n->n_params, cudaMemcpyHostToDevice));
  LLR_TRY(pack_all(n, nullptr));
  LLR_CUDA_TRY(cudaDeviceSynchronize());
  return LLR_OK;
}

int llr_cnn_get_grads(llr_cnn* n, float* host) {
  if (!n || !host) return set_error(LLR_ERR_INVALID, "null pointer");
  LLR_CUDA_TRY(cudaSetDevice(n->device));
  LLR_CUDA_TRY(cudaMemcpy(host, n->d_grad, sizeof(float) * n->n_params, cudaMemcpyDeviceToHost));
  return LLR_OK;
}

int llr_cnn_forward_dev(llr_cnn* n, const float* d_in, float* d_out, const int32_t* dims, void* stream) {
  if (!n || !d_in || !d_out) return set_error(LLR_ERR_INVALID, "null pointer");
  LLR_TRY(check_dims(dims));
  LLR_CUDA_TRY(cudaSetDevice(n->device));
  LLR_TRY(ensure_workspace(n, (long long)dims[0] * dims[1] * dims[2]));
  return forward(n, d_in, d_out, dims, (cudaStream_t)stream);
}

int llr_cnn_loss_grad_dev(llr_cnn* n, const float* d_in, const float* d_target, const int32_t* dims, double* loss,
                          void* stream) {
  if (!n || !d_in || !d_target) return set_error(LLR_ERR_INVALID, "null pointer");
  LLR_TRY(check_dims(dims));
  LLR_CUDA_TRY(cudaSetDevice(n->device));
  cudaStream_t s = (cudaStream_t)stream;
  const long long vox = (long long)dims[0] * dims[1] * dims[2];
  LLR_TRY(ensure_workspace(n, vox));
  LLR_TRY(forward(n, d_in, n->d_out, dims, s));
  const long long nout = vox * n->cout.back();
  const int lg = std::min(n->loss_cap, grid_1d(nout));
  note_launch();
  mse_kernel<<<lg, 256, 0, s>>>(n->d_out, d_target, n->d_g0, nout, n->d_loss);
  LLR_CUDA_TRY(cudaGetLastError());
  // out = in + f(in): dL/df = dL/dout; walk the layers backwards
  float* g = n->d_g0;
  float* gn = n->d_g1;
  for (int l = n->n_layers - 1; l >= 0; --l) {
    LLR_TRY(wgrad(n->cin[l], n->cout[l], n->act[l], g, n->d_part, n->part_cap, n->d_grad + n->w_off[l], dims, s));
    if (l == 0) break;
    // dL/d act[l] = conv(g, W') masked by the ReLU that produced act[l]
    LLR_TRY(conv(n->cout[l], n->cin[l], g, n->d_wt + wtab_off(n, l), nullptr, nullptr, gn, dims, 0, s));
    const long long na = vox * n->cin[l];
    note_launch();
    relu_mask_kernel<<<grid_1d(na), 256, 0, s>>>(gn, n->act[l], na);
    LLR_CUDA_TRY(cudaGetLastError());
    std::swap(g, gn);
  }
  if (loss) {
    std::vector<double> h((size_t)lg);
    LLR_CUDA_TRY(cudaMemcpyAsync(h.data(), n->d_loss, sizeof(double) * lg, cudaMemcpyDeviceToHost, s));
    LLR_CUDA_TRY(cudaStreamSynchronize(s));
    double t = 0.0;
    for (double v : h) t += v;
    *loss = t / (double)nout;
  }
  return LLR_OK;
}

int llr_cnn_adam_step(llr_cnn* n, float lr, float beta1, float beta2, float eps, void* stream) {
  if (!n) return set_error(LLR_ERR_INVALID, "null network");
  LLR_CUDA_TRY(cudaSetDevice(n->device));
  cudaStream_t s = (cudaStream_t)stream;
  n->step += 1;
  const float c1 = (float)(1.0 / (1.0 - std::pow((double)beta1, (double)n->step)));
  const float c2 = (float)(1.0 / (1.0 - std::pow((double)beta2, (double)n->step)));
  note_launch();
  adam_kernel<<<grid_1d(n->n_params), 256, 0, s>>>(n->d_master, n->d_grad, n->d_m, n->d_v, n->n_params, lr, beta1,
                                                   beta2, eps, c1, c2);
  LLR_CUDA_TRY(cudaGetLastError());
  return pack_all(n, s);
}

int llr_cnn_train_step_dev(llr_cnn* n, const float* d_in, const float* d_target, const int32_t* dims, float lr,
                           double* loss, void* stream) {
  LLR_TRY(llr_cnn_loss_grad_dev(n, d_in, d_target, dims, loss, stream));
  return llr_cnn_adam_step(n, lr, 0.9f, 0.999f, 1e-8f, stream);
}

int llr_subspace_channels_dev(const llr_cf32* d_x, const int32_t* vol, int32_t nq, const llr_cf32* d_S, int32_t srank,
                              float scale, float* d_chan, void* stream) {
  if (!d_x || !vol || !d_S || !d_chan || nq < 1 || srank < 1 || srank > 16)
    return set_error(LLR_ERR_INVALID, "bad subspace channel arguments (1 <= srank <= 16)");
  const long long V = (long long)vol[0] * vol[1] * vol[2];
  note_launch();
  subspace_channels_kernel<<<grid_1d(V), 256, sizeof(float2) * nq * srank, (cudaStream_t)stream>>>(
      (const float2*)d_x, V, nq, (const float2*)d_S, srank, scale, d_chan);
  LLR_CUDA_TRY(cudaGetLastError());
  return LLR_OK;
}

int llr_subspace_image_dev(const float* d_chan, const int32_t* vol, int32_t nq, const llr_cf32* d_S, int32_t srank,
                           float scale, int32_t accumulate, llr_cf32* d_x, void* stream) {
  if (!d_x || !vol || !d_S || !d_chan || nq < 1 || srank < 1 || srank > 16 || !(scale != 0.f))
    return set_error(LLR_ERR_INVALID, "bad subspace image arguments (1 <= srank <= 16, scale != 0)");
  const long long V = (long long)vol[0] * vol[1] * vol[2];
  note_launch();
  subspace_image_kernel<<<grid_1d(V), 256, sizeof(float2) * nq * srank, (cudaStream_t)stream>>>(
      d_chan, V, nq, (const float2*)d_S, srank, 1.f / scale, (float2*)d_x, accumulate ? 1 : 0);
  LLR_CUDA_TRY(cudaGetLastError());
  return LLR_OK;
}

}  // extern "C"
