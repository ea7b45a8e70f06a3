// Learned warm start: a small 3-D residual CNN (conv3d 3x3x3, zero padding, ReLU between
// layers, out = in + net(in)) with hand-written forward, backward-data and backward-weight
// kernels, mean-squared-error loss and Adam.  BF16 weights feed the convolutions with FP32
// accumulation on the tensor cores: forward and backward-data as tcgen05 kind::f16 MMAs with
// the activations split into three BF16 planes, the weight gradient as 3xTF32 MMAs; the
// optimizer keeps FP32 master weights.
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

#include <cuda_bf16.h>

#include "llr_common.cuh"
#include "llr_internal.h"
#include "llr_umma.cuh"

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
  int* d_err;                            // set by a conv kernel whose bounded tensor-core wait ran out
};

namespace llr {

namespace {

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

// ---------------------------------------------------------------------------------------
// Geometry shared by the tensor-core conv kernels.
// ---------------------------------------------------------------------------------------
constexpr int kCvThreads = 256;
constexpr int kCvTX = 8, kCvTY = 4, kCvTZ = 4;                  // weight-gradient tile: 128 voxels
constexpr int kCvHX = kCvTX + 2, kCvHY = kCvTY + 2, kCvHZ = kCvTZ + 2;
constexpr int kCvHV = kCvHX * kCvHY * kCvHZ;
constexpr int kCvPlane = 128 * 128;                              // one 128 x 32 TF32 operand plane (bytes)

__host__ __device__ constexpr int cv_np(int cout) { return cout <= 16 ? 16 : 32; }

// ---------------------------------------------------------------------------------------
// conv3d forward (and backward-data: the same convolution with W') as an implicit GEMM on
// the tensor cores, tcgen05 kind::f16 with BF16 operands and FP32 accumulation in tensor
// memory.
//
// A CTA owns tiles of 128 output voxels, 8 (x) x 16 (y) x 1 (z); row a = x + 8 y of the
// 128 x COUT accumulator.  The tile's input halo (10 x 18 x 3 voxels, all channels) is
// written once into shared memory in the unswizzled K-major operand layout: channel chunk c
// (8 BF16 = 16 B) of halo voxel h at byte c * CS + 16 h.  The operand of tap (dx, dy, dz) is
// then the same array read from voxel dx + 10 (dy + 18 dz) on: 8 consecutive x form one core
// matrix (128 contiguous bytes), the 16 rows y step by 10 voxels (SBO = 160 B) and the K
// chunks by CS (LBO).  There is no per-tap copy and no per-tap barrier: once the halo is in
// place one thread issues the MMAs of all 27 taps back to back.
//
// FP32 accuracy: each activation is split x = b1 + b2 + b3 into three BF16 planes (b1 the
// BF16 rounding of x, b2 of x - b1, b3 of the rest: ~24 significant bits in all); the weights
// are BF16 and exact.  D += b1 W + b2 W + b3 W, three MMAs per K step of 16 channels.
//
// Pipeline: the next tile's FP32 halo is copied with cp.async (zero fill outside the volume
// and for padding channels) into a staging buffer while the current tile's MMAs run, and two
// accumulators in tensor memory let the epilogue of tile i - 1 (tcgen05.ld, bias, ReLU,
// residual, store) run beside the MMAs of tile i.  Every mbarrier wait is bounded; one that
// runs out sets the error flag and the CTA stops.
// ---------------------------------------------------------------------------------------
constexpr int kFwTX = 8, kFwTY = 16;                             // forward tile: 128 voxels of one z plane
constexpr int kFwHX = kFwTX + 2, kFwHY = kFwTY + 2, kFwHZ = 3;
constexpr int kFwNV = kFwHX * kFwHY * kFwHZ;                       // 540 halo voxels
constexpr int kFwCS = kFwNV * 16;                                  // bytes of one 8-channel chunk of a plane

template <int CIN, int COUT>
struct CvLayout {
  static constexpr int NP = cv_np(COUT);                           // accumulator columns (N)
  static constexpr int KC = (CIN + 15) / 16 * 2;                   // 8-channel chunks, K padded to 16
  static constexpr int KS = KC / 2;                                // K steps of 16 channels per tap
  static constexpr int RC = 2 * KC;                                // 4-channel chunks of the FP32 halo
  static constexpr int NPL = 3;                                    // BF16 planes per activation
  static constexpr int WT = KC * NP * 16;                          // bytes of one tap's weights
  static constexpr size_t PB = (size_t)KC * kFwCS;                 // bytes of one BF16 plane
  static constexpr size_t off_hdr = 0;                             // mbarriers, TMEM address
  static constexpr size_t off_pl = 1024;                           // NPL BF16 planes
  static constexpr size_t off_w = off_pl + NPL * PB;               // 27 taps of weights
  static constexpr size_t off_raw = off_w + (size_t)27 * WT;       // FP32 halo staging, chunk r at r NV 16
  static constexpr size_t total = off_raw + (size_t)RC * kFwNV * 16;
};

struct CvGeo {
  int nx, ny, nz, tx, ty;
  long long ntiles;
};

// x = b1 + b2 + b3 for two values, as three packed BF16 pairs (low half = first value)
__device__ __forceinline__ void split3_bf16(float a, float b, uint32_t& p1, uint32_t& p2, uint32_t& p3) {
  const __nv_bfloat162 h1 = __floats2bfloat162_rn(a, b);
  const float2 f1 = __bfloat1622float2(h1);
  const float ra = a - f1.x, rb = b - f1.y;
  const __nv_bfloat162 h2 = __floats2bfloat162_rn(ra, rb);
  const float2 f2 = __bfloat1622float2(h2);
  const __nv_bfloat162 h3 = __floats2bfloat162_rn(ra - f2.x, rb - f2.y);
  p1 = *reinterpret_cast<const uint32_t*>(&h1);
  p2 = *reinterpret_cast<const uint32_t*>(&h2);
  p3 = *reinterpret_cast<const uint32_t*>(&h3);
}

// any of the 256 worker threads (warps 0-7, named barrier 1) has v set; all of them get the answer
__device__ __forceinline__ bool workers_any(bool v) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\tbar.red.or.pred q, 1, 256, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}" : "=r"(r) : "r"((uint32_t)v) : "memory");
  return r != 0;
}

__device__ __forceinline__ void mbar_arrive(uint32_t mbar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(mbar) : "memory");
}

constexpr int kFwWorkers = 256, kFwThreads = kFwWorkers + 32;   // warps 0-7 workers, warp 8 issues the MMAs

template <int CIN, int COUT>
__global__ void __launch_bounds__(kFwThreads, 1) conv3d_tc_kernel(const float* __restrict__ x,
                                                                  const uint16_t* __restrict__ wb,
                                                                  const float* __restrict__ bias,
                                                                  const float* __restrict__ add, float* __restrict__ y,
                                                                  CvGeo G, int relu, int* err) {
  using Lay = CvLayout<CIN, COUT>;
  constexpr int NP = Lay::NP, KS = Lay::KS, RC = Lay::RC, NPL = Lay::NPL;
  constexpr uint32_t idesc = umma_idesc_bf16(128, NP);
  constexpr uint32_t kCols = 2 * NP;                               // two accumulators: 32 or 64 columns
  static_assert(NPL == 3, "the operand split writes three planes");
  static_assert(KS <= 4, "mbarrier slots");
  extern __shared__ __align__(1024) unsigned char smem[];
  // mbarriers: conv_full[s] (workers -> MMA warp: K step s of the planes written), mma_done[s]
  // (MMA warp -> workers: K step s read), acc_full[a] / acc_empty[a] per accumulator, drain
  unsigned long long* mb = reinterpret_cast<unsigned long long*>(smem + Lay::off_hdr);
  unsigned long long* conv_full = mb;
  unsigned long long* mma_done = mb + 4;
  unsigned long long* acc_full = mb + 8;
  unsigned long long* acc_empty = mb + 10;
  unsigned long long* drain = mb + 12;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + Lay::off_hdr + 128);
  unsigned char* pl = smem + Lay::off_pl;
  unsigned char* wsm = smem + Lay::off_w;
  unsigned char* raw = smem + Lay::off_raw;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int b = 0; b < 13; ++b) {
      const uint32_t cnt = (b < 4 || b == 10 || b == 11) ? (uint32_t)kFwWorkers : 1u;
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&mb[b])), "r"(cnt));
    }
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  // weights W[tap][ci][co] (BF16) -> tap block, chunk ci / 8, row co, element ci % 8;
  // padding rows (co >= COUT) and columns (ci >= CIN) stay zero
  for (int i = tid; i < 27 * Lay::WT / 16; i += kFwThreads) reinterpret_cast<uint4*>(wsm)[i] = make_uint4(0u, 0u, 0u, 0u);
  __syncthreads();
  for (int i = tid; i < 27 * CIN * COUT; i += kFwThreads) {
    const int tap = i / (CIN * COUT), r = i - tap * (CIN * COUT), ci = r / COUT, co = r - ci * COUT;
    *reinterpret_cast<uint16_t*>(wsm + tap * Lay::WT + (ci >> 3) * NP * 16 + co * 16 + (ci & 7) * 2) = wb[i];
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = *tmem_slot;
  // tile i of this CTA is blockIdx.x + i gridDim.x
  const long long n = (long long)blockIdx.x < G.ntiles ? (G.ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  bool failed = false;

  if (warp < 8) {
    // FP32 halo of tile t into the staging buffer (4-channel chunk r of halo voxel h at
    // (r NV + h) 16 bytes), zero outside the volume and for channels >= CIN
    constexpr int VW = CIN % 4 == 0 ? 4 : 1, PER = 4 * RC / VW;
    auto load_raw = [&](long long t) {
      const int hx0 = (int)(t % G.tx) * kFwTX - 1;
      const long long rt = t / G.tx;
      const int hy0 = (int)(rt % G.ty) * kFwTY - 1, hz0 = (int)(rt / G.ty) - 1;
      for (int i = tid; i < kFwNV * PER; i += kFwWorkers) {
        const int h = i / PER, c = (i - h * PER) * VW;
        const int hx = h % kFwHX, hy = (h / kFwHX) % kFwHY, hz = h / (kFwHX * kFwHY);
        const int gx = hx0 + hx, gy = hy0 + hy, gz = hz0 + hz;
        const bool in = c < CIN && gx >= 0 && gx < G.nx && gy >= 0 && gy < G.ny && gz >= 0 && gz < G.nz;
        const float* src = in ? x + ((long long)gx + (long long)G.nx * (gy + (long long)G.ny * gz)) * CIN + c : x;
        const uint32_t dst = smem_u32(raw + ((size_t)(c >> 2) * kFwNV + h) * 16 + (c & 3) * 4);
        if constexpr (VW == 4)
          asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(in ? 16 : 0) : "memory");
        else
          asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(dst), "l"(src), "r"(in ? 4 : 0) : "memory");
      }
      asm volatile("cp.async.commit_group;" ::: "memory");
    };
    // K step s of the staging buffer -> the three BF16 planes (item = 8 channels of one voxel)
    auto convert = [&](int s) {
      for (int i = tid; i < 2 * kFwNV; i += kFwWorkers) {
        const int c = 2 * s + (i >= kFwNV ? 1 : 0), h = i - (i >= kFwNV ? kFwNV : 0);
        const float4 v0 = *reinterpret_cast<const float4*>(raw + ((size_t)(2 * c) * kFwNV + h) * 16);
        const float4 v1 = *reinterpret_cast<const float4*>(raw + ((size_t)(2 * c + 1) * kFwNV + h) * 16);
        uint4 q1, q2, q3;
        split3_bf16(v0.x, v0.y, q1.x, q2.x, q3.x);
        split3_bf16(v0.z, v0.w, q1.y, q2.y, q3.y);
        split3_bf16(v1.x, v1.y, q1.z, q2.z, q3.z);
        split3_bf16(v1.z, v1.w, q1.w, q2.w, q3.w);
        unsigned char* o = pl + (size_t)c * kFwCS + (size_t)h * 16;
        *reinterpret_cast<uint4*>(o) = q1;
        *reinterpret_cast<uint4*>(o + Lay::PB) = q2;
        *reinterpret_cast<uint4*>(o + 2 * Lay::PB) = q3;
      }
    };
    // accumulator of tile j -> y: warp w reads TMEM lanes 32 (w & 3) .. + 31 (tile rows) and
    // the column half w >> 2; returns false when the wait for the MMAs ran out
    constexpr int HC = NP / 2;
    const int q = warp & 3, hs = warp >> 2;
    float bz[HC];
#pragma unroll
    for (int j = 0; j < HC; ++j) bz[j] = (bias && hs * HC + j < COUT) ? bias[hs * HC + j] : 0.f;
    auto epilogue = [&](long long j) -> bool {
      const uint32_t acc = (uint32_t)(j & 1);
      const bool ok = mbar_wait(smem_u32(&acc_full[acc]), (uint32_t)((j >> 1) & 1));
      if (workers_any(!ok)) return false;
      asm volatile("tcgen05.fence::after_thread_sync;");
      uint32_t r[HC];
      const uint32_t taddr = tmem + ((uint32_t)(32 * q) << 16) + acc * NP + hs * HC;
      if constexpr (HC == 16) {
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
              "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
            : "r"(taddr));
      } else {
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                     : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                     : "r"(taddr));
      }
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;");
      mbar_arrive(smem_u32(&acc_empty[acc]));   // the MMA warp may reuse this accumulator
      const long long t = (long long)blockIdx.x + j * gridDim.x;
      const int a = 32 * q + lane;
      const int gx = (int)(t % G.tx) * kFwTX + (a & 7);
      const long long rt = t / G.tx;
      const int gy = (int)(rt % G.ty) * kFwTY + (a >> 3), gz = (int)(rt / G.ty);
      if (gx < G.nx && gy < G.ny) {
        const long long v = (long long)gx + (long long)G.nx * (gy + (long long)G.ny * gz);
        float o[HC];
#pragma unroll
        for (int k = 0; k < HC; ++k) {
          float val = __uint_as_float(r[k]) + bz[k];
          if (relu) val = fmaxf(val, 0.f);
          o[k] = val;
        }
        if constexpr (COUT == 2 * HC && HC % 4 == 0) {   // whole 16-byte groups of this voxel's channels
          float4* yp = reinterpret_cast<float4*>(y + v * COUT + hs * HC);
          const float4* ap = add ? reinterpret_cast<const float4*>(add + v * COUT + hs * HC) : nullptr;
#pragma unroll
          for (int k = 0; k < HC / 4; ++k) {
            float4 w4 = make_float4(o[4 * k], o[4 * k + 1], o[4 * k + 2], o[4 * k + 3]);
            if (ap) {
              const float4 a4 = ap[k];
              w4.x += a4.x; w4.y += a4.y; w4.z += a4.z; w4.w += a4.w;
            }
            yp[k] = w4;
          }
        } else {
#pragma unroll
          for (int k = 0; k < HC; ++k) {
            const int c = hs * HC + k;
            if (c < COUT) y[v * COUT + c] = o[k] + (add ? add[v * COUT + c] : 0.f);
          }
        }
      }
      return true;
    };

    if (n > 0) load_raw(blockIdx.x);
    for (long long i = 0; i < n && !failed; ++i) {
      asm volatile("cp.async.wait_all;" ::: "memory");
      asm volatile("bar.sync 1, 256;" ::: "memory");
      for (int s = 0; s < KS; ++s) {
        if (i > 0) {   // the MMAs of tile i - 1 no longer read K step s of the planes
          const bool ok = mbar_wait(smem_u32(&mma_done[s]), (uint32_t)((i - 1) & 1));
          if (workers_any(!ok)) { failed = true; break; }
        }
        convert(s);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_arrive(smem_u32(&conv_full[s]));
      }
      if (failed) break;
      asm volatile("bar.sync 1, 256;" ::: "memory");   // every worker is done with the staging buffer
      if (i + 1 < n) load_raw((long long)blockIdx.x + (i + 1) * gridDim.x);
      if (i > 0 && !epilogue(i - 1)) failed = true;
    }
    if (!failed && n > 0 && !epilogue(n - 1)) failed = true;
    asm volatile("cp.async.wait_all;" ::: "memory");
  } else if (lane == 0) {
    const uint64_t a0 = umma_desc_kmajor(smem_u32(pl), kFwCS, kFwHX * 16);
    const uint64_t b0 = umma_desc_kmajor(smem_u32(wsm), NP * 16, 128);
    for (long long i = 0; i < n && !failed; ++i) {
      const uint32_t acc = (uint32_t)(i & 1);
      if (i >= 2 && !mbar_wait(smem_u32(&acc_empty[acc]), (uint32_t)(((i - 2) >> 1) & 1))) { failed = true; break; }
      const uint32_t d = tmem + acc * NP;
      for (int s = 0; s < KS; ++s) {
        if (!mbar_wait(smem_u32(&conv_full[s]), (uint32_t)(i & 1))) { failed = true; break; }
        asm volatile("tcgen05.fence::after_thread_sync;");
        // descriptor start addresses advance in 16-byte units
        const uint64_t as = a0 + (uint64_t)((s * 2 * kFwCS) >> 4), bs = b0 + (uint64_t)((s * 2 * NP * 16) >> 4);
#pragma unroll 1
        for (int dzy = 0; dzy < 9; ++dzy) {   // dy + 3 dz
          const uint32_t vrow = (uint32_t)(kFwHX * (dzy % 3 + kFwHY * (dzy / 3)));
#pragma unroll
          for (int dx = 0; dx < 3; ++dx) {
            const uint64_t db = bs + (uint64_t)(((3 * dzy + dx) * Lay::WT) >> 4);
#pragma unroll
            for (int p = 0; p < NPL; ++p) {
              const uint64_t da = as + (uint64_t)((p * Lay::PB) >> 4) + vrow + dx;
              umma_bf16(d, da, db, idesc, (s > 0 || dzy > 0 || dx > 0 || p > 0) ? 1u : 0u);
            }
          }
        }
        umma_commit(smem_u32(&mma_done[s]));
      }
      if (failed) break;
      umma_commit(smem_u32(&acc_full[acc]));
    }
  }
  if (failed && err) atomicExch(err, 1);
  __syncthreads();
  // nothing may still write an accumulator when tensor memory is released
  if (warp == 8 && lane == 0) umma_commit(smem_u32(drain));
  mbar_wait(smem_u32(drain), 0u);
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols));
}

// ---------------------------------------------------------------------------------------
// Weight gradient on the tensor cores: D[(tap, ci)][co] = sum_v x[v + d(tap)][ci] dy[v][co]
// as MT = ceil(27 CIN / 128) GEMMs of M = 128 rows (tap, ci), N = COUT (padded to 16 / 32),
// K = voxels, accumulated in tensor memory over every tile the CTA visits (MT x N columns).
// Per 128-voxel tile the input halo and the tile's dy are staged once; dy goes to TF32 hi / lo
// B planes (N rows x 32 voxels per K chunk), and for each (K chunk, M tile) the tap-shifted
// input rows are written as hi / lo A planes (double-buffered) and multiplied with 3xTF32
// (hi hi + hi lo + lo hi).  At the end each CTA writes its partial sums (and the bias
// gradient, summed in FP32 from the staged dy); a fixed-order reduction adds the CTAs.
// ---------------------------------------------------------------------------------------
template <int CIN, int COUT>
struct WgLayout {
  static constexpr int NP = cv_np(COUT);
  static constexpr int HP = CIN | 1;
  static constexpr int MT = (27 * CIN + 127) / 128;
  static constexpr int TCOLS = MT * NP <= 32 ? 32 : MT * NP <= 64 ? 64 : MT * NP <= 128 ? 128 : 256;
  static constexpr size_t off_hdr = 0;
  static constexpr size_t off_b = 1024;                              // 4 K chunks x (hi, lo) x NP x 128 B
  static constexpr size_t off_a = off_b + (size_t)8 * NP * 128;       // 2 buffers x (hi, lo)
  static constexpr size_t off_halo = off_a + (size_t)4 * kCvPlane;
  static constexpr size_t off_dy = off_halo + sizeof(float) * (size_t)kCvHV * HP;
  static constexpr size_t total = off_dy + sizeof(float) * 128 * COUT;
};

template <int CIN, int COUT>
__global__ void __launch_bounds__(kCvThreads, 1) conv3d_wgrad_tc_kernel(const float* __restrict__ x,
                                                                        const float* __restrict__ dy,
                                                                        float* __restrict__ part, CvGeo G, int* err) {
  using Lay = WgLayout<CIN, COUT>;
  constexpr int NP = Lay::NP, HP = Lay::HP, MT = Lay::MT, ROWS = 27 * CIN;
  constexpr uint32_t idesc = umma_idesc_tf32(128, NP);
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned long long* mbar = reinterpret_cast<unsigned long long*>(smem + Lay::off_hdr);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + Lay::off_hdr + 32);
  unsigned char* bsm = smem + Lay::off_b;
  unsigned char* asm_ = smem + Lay::off_a;
  float* halo = reinterpret_cast<float*>(smem + Lay::off_halo);
  float* sdy = reinterpret_cast<float*>(smem + Lay::off_dy);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"((uint32_t)Lay::TCOLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int b = 0; b < 3; ++b) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[b])));
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  for (int i = tid; i < (int)((Lay::off_halo - Lay::off_b) / 16); i += kCvThreads)
    reinterpret_cast<float4*>(bsm)[i] = make_float4(0.f, 0.f, 0.f, 0.f);
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = *tmem_slot;
  uint32_t phase[3] = {0u, 0u, 0u};
  bool used[2] = {false, false};
  bool failed = false, first = true;
  int gpar = 0;
  float dbacc = 0.f;
  for (long long tile = blockIdx.x; tile < G.ntiles && !failed; tile += gridDim.x) {
    const int ox = (int)(tile % G.tx) * kCvTX;
    const long long rt = tile / G.tx;
    const int oy = (int)(rt % G.ty) * kCvTY, oz = (int)(rt / G.ty) * kCvTZ;
    for (int i = tid; i < kCvHV * CIN; i += kCvThreads) {
      const int hv = i / CIN, c = i - hv * CIN;
      const int hx = hv % kCvHX, hy = (hv / kCvHX) % kCvHY, hz = hv / (kCvHX * kCvHY);
      const int gx = ox + hx - 1, gy = oy + hy - 1, gz = oz + hz - 1;
      float v = 0.f;
      if (gx >= 0 && gx < G.nx && gy >= 0 && gy < G.ny && gz >= 0 && gz < G.nz)
        v = x[((long long)gx + (long long)G.nx * (gy + (long long)G.ny * gz)) * CIN + c];
      halo[hv * HP + c] = v;
    }
    for (int i = tid; i < 128 * COUT; i += kCvThreads) {   // dy of the tile's voxels -> B planes (row co, column voxel)
      const int a = i / COUT, c = i - a * COUT;
      const int gx = ox + (a & 7), gy = oy + ((a >> 3) & 3), gz = oz + (a >> 5);
      float v = 0.f;
      if (gx < G.nx && gy < G.ny && gz < G.nz) v = dy[((long long)gx + (long long)G.nx * (gy + (long long)G.ny * gz)) * COUT + c];
      sdy[i] = v;
      const int kc = a >> 5, kv = a & 31;
      unsigned char* bh = bsm + (size_t)kc * 2 * NP * 128;
      const uint32_t h = tf32_rna(v);
      const int o = op_offset(c, kv);
      *reinterpret_cast<uint32_t*>(bh + o) = h;
      *reinterpret_cast<float*>(bh + NP * 128 + o) = v - __uint_as_float(h);
    }
    __syncthreads();
    if (tid < COUT)
      for (int a = 0; a < 128; ++a) dbacc += sdy[a * COUT + tid];
    for (int kc = 0; kc < 4 && !failed; ++kc) {
      for (int mt = 0; mt < MT; ++mt) {
        const int b = gpar;
        if (used[b]) {
          const bool ok = mbar_wait(smem_u32(&mbar[b]), phase[b]);
          phase[b] ^= 1u;
          if (__syncthreads_or(!ok)) { failed = true; break; }
        }
        unsigned char* hi = asm_ + (size_t)b * 2 * kCvPlane;
        unsigned char* lo = hi + kCvPlane;
        for (int e = tid; e < 128 * 32; e += kCvThreads) {   // row r = (tap, ci), column kv = voxel 32 kc + kv
          const int rl = e >> 5, kv = e & 31;
          const int r = mt * 128 + rl;
          float v = 0.f;
          if (r < ROWS) {
            const int tap = r / CIN, ci = r - tap * CIN;
            const int dx = tap % 3, dyy = (tap / 3) % 3, dz = tap / 9;
            const int a = 32 * kc + kv;
            const int lx = a & 7, ly = (a >> 3) & 3, lz = a >> 5;
            v = halo[((lx + dx) + kCvHX * ((ly + dyy) + kCvHY * (lz + dz))) * HP + ci];
          }
          const uint32_t h = tf32_rna(v);
          const int o = op_offset(rl, kv);
          *reinterpret_cast<uint32_t*>(hi + o) = h;
          *reinterpret_cast<float*>(lo + o) = v - __uint_as_float(h);
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
          asm volatile("tcgen05.fence::after_thread_sync;");
          const uint32_t ah = smem_u32(hi), al = smem_u32(lo);
          const uint32_t bh = smem_u32(bsm + (size_t)kc * 2 * NP * 128), bl = bh + NP * 128;
          const uint32_t d = tmem + (uint32_t)(mt * NP);
#pragma unroll
          for (int st = 0; st < 4; ++st) {
            const uint64_t dah = umma_desc_sw128(ah + st * 32), dal = umma_desc_sw128(al + st * 32);
            const uint64_t dbh = umma_desc_sw128(bh + st * 32), dbl = umma_desc_sw128(bl + st * 32);
            umma_tf32(d, dah, dbh, idesc, (first && kc == 0 && st == 0) ? 0u : 1u);
            umma_tf32(d, dah, dbl, idesc, 1u);
            umma_tf32(d, dal, dbh, idesc, 1u);
          }
          umma_commit(smem_u32(&mbar[b]));
          if (kc == 3 && mt == MT - 1) umma_commit(smem_u32(&mbar[2]));
        }
        used[b] = true;
        gpar ^= 1;
      }
    }
    if (failed) break;
    first = false;
    {   // the next tile overwrites the B planes and the halo: this tile's MMAs must be done
      const bool ok = mbar_wait(smem_u32(&mbar[2]), phase[2]);
      phase[2] ^= 1u;
      for (int bb = 0; bb < 2; ++bb)
        if (used[bb]) {
          mbar_wait(smem_u32(&mbar[bb]), phase[bb]);
          phase[bb] ^= 1u;
          used[bb] = false;
        }
      if (__syncthreads_or(!ok)) { failed = true; break; }
    }
  }
  float* P = part + (long long)blockIdx.x * (ROWS * COUT + COUT);
  if (!failed) {
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (warp < 4) {
      for (int mt = 0; mt < MT; ++mt) {
        uint32_t r[NP];
        const uint32_t taddr = tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(mt * NP);
        if constexpr (NP == 32) {
          asm volatile(
              "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
              "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
              : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
                "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
                "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
              : "r"(taddr));
        } else {
          asm volatile(
              "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
              : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                "=r"(r[15])
              : "r"(taddr));
        }
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        const int row = mt * 128 + 32 * warp + lane;
        if (row < ROWS) {
#pragma unroll
          for (int c = 0; c < COUT; ++c) P[(long long)row * COUT + c] = first ? 0.f : __uint_as_float(r[c]);
        }
      }
    }
    if (tid < COUT) P[ROWS * COUT + tid] = dbacc;
  }
  if (failed && tid == 0 && err) atomicExch(err, 1);
  if (tid == 0) umma_commit(smem_u32(&mbar[2]));
  mbar_wait(smem_u32(&mbar[2]), phase[2]);
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)Lay::TCOLS));
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

// Unit phase of a reference value (1 for 0): the demodulation factor of one voxel and volume.
__device__ __forceinline__ float2 unit_phase(float2 r) {
  const float m2 = r.x * r.x + r.y * r.y;
  if (!(m2 > 0.f)) return make_float2(1.f, 0.f);
  const float inv = rsqrtf(m2);
  return make_float2(r.x * inv, r.y * inv);
}

// chan[v][2k + {0, 1}] = scale * (re, im) of sum_q u*[v + V q] x[v + V q] S[q + nq k], with u the unit
// phase of the reference image `ph` (u = 1 when ph is null)
__global__ void subspace_channels_kernel(const float2* __restrict__ x, long long V, int nq, const float2* __restrict__ S,
                                         int r, float scale, const float2* __restrict__ ph, float* __restrict__ chan) {
  extern __shared__ float2 sS[];
  for (int i = threadIdx.x; i < nq * r; i += blockDim.x) sS[i] = S[i];
  __syncthreads();
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < V; v += (long long)gridDim.x * blockDim.x) {
    float2 c[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) c[k] = make_float2(0.f, 0.f);
    for (int q = 0; q < nq; ++q) {
      float2 xv = x[v + V * q];
      if (ph) xv = cmulc(unit_phase(ph[v + V * q]), xv);
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

// x[v + V q] (+)= u[v + V q] (1 / scale) sum_k c_k conj(S[q + nq k]), u as above
__global__ void subspace_image_kernel(const float* __restrict__ chan, long long V, int nq, const float2* __restrict__ S,
                                      int r, float inv_scale, const float2* __restrict__ ph, float2* __restrict__ x,
                                      int accumulate) {
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
      if (ph) acc = cmul(unit_phase(ph[v + V * q]), acc);
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
int conv_inst(const float* x, const uint16_t* w, const float* b, const float* add, float* y, const int* dims, int relu,
              int* err, cudaStream_t s) {
  const size_t smem = CvLayout<CIN, COUT>::total;
  static_assert(CvLayout<CIN, COUT>::total <= 227 * 1024, "conv operands exceed shared memory");
  if (CIN % 4 == 0 && (reinterpret_cast<uintptr_t>(x) & 15) != 0)
    return set_error(LLR_ERR_INVALID, "conv3d input must be 16-byte aligned for %d channels", CIN);
  auto k = conv3d_tc_kernel<CIN, COUT>;
  LLR_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int dev = 0, nsm = 0;
  LLR_CUDA_TRY(cudaGetDevice(&dev));
  LLR_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  CvGeo G;
  G.nx = dims[0]; G.ny = dims[1]; G.nz = dims[2];
  G.tx = (G.nx + kFwTX - 1) / kFwTX;
  G.ty = (G.ny + kFwTY - 1) / kFwTY;
  G.ntiles = (long long)G.tx * G.ty * G.nz;
  const long long grid = std::min<long long>(G.ntiles, nsm);
  note_launch();
  k<<<(unsigned)grid, kFwThreads, smem, s>>>(x, w, b, add, y, G, relu, err);
  LLR_CUDA_TRY(cudaGetLastError());
  return LLR_OK;
}

int conv(int cin, int cout, const float* x, const uint16_t* w, const float* b, const float* add, float* y,
         const int* dims, int relu, int* err, cudaStream_t s) {
  if (cin == 14 && cout == 32) return conv_inst<14, 32>(x, w, b, add, y, dims, relu, err, s);
  if (cin == 32 && cout == 32) return conv_inst<32, 32>(x, w, b, add, y, dims, relu, err, s);
  if (cin == 32 && cout == 14) return conv_inst<32, 14>(x, w, b, add, y, dims, relu, err, s);
  return set_error(LLR_ERR_UNSUPPORTED, "conv3d %d -> %d channels is not built", cin, cout);
}

template <int CIN, int COUT>
int wgrad_inst(const float* x, const float* dy, float* part, long long part_cap, float* out, const int* dims, int* err,
               cudaStream_t s) {
  const size_t smem = WgLayout<CIN, COUT>::total;
  static_assert(WgLayout<CIN, COUT>::total <= 227 * 1024, "wgrad operands exceed shared memory");
  auto k = conv3d_wgrad_tc_kernel<CIN, COUT>;
  LLR_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int dev = 0, nsm = 0;
  LLR_CUDA_TRY(cudaGetDevice(&dev));
  LLR_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  CvGeo G;
  G.nx = dims[0]; G.ny = dims[1]; G.nz = dims[2];
  G.tx = (G.nx + kCvTX - 1) / kCvTX;
  G.ty = (G.ny + kCvTY - 1) / kCvTY;
  G.ntiles = (long long)G.tx * G.ty * ((G.nz + kCvTZ - 1) / kCvTZ);
  const long long per = 27LL * CIN * COUT + COUT;
  const int grid = (int)std::max<long long>(1, std::min<long long>(std::min<long long>(G.ntiles, nsm), part_cap / per));
  note_launch();
  k<<<grid, kCvThreads, smem, s>>>(x, dy, part, G, err);
  LLR_CUDA_TRY(cudaGetLastError());
  note_launch();
  reduce_partials_kernel<<<grid_1d(per), 256, 0, s>>>(part, grid, per, out);
  LLR_CUDA_TRY(cudaGetLastError());
  return LLR_OK;
}

int wgrad(int cin, int cout, const float* x, const float* dy, float* part, long long cap, float* out, const int* dims,
          int* err, cudaStream_t s) {
  if (cin == 14 && cout == 32) return wgrad_inst<14, 32>(x, dy, part, cap, out, dims, err, s);
  if (cin == 32 && cout == 32) return wgrad_inst<32, 32>(x, dy, part, cap, out, dims, err, s);
  if (cin == 32 && cout == 14) return wgrad_inst<32, 14>(x, dy, part, cap, out, dims, err, s);
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
                 last ? in : nullptr, y, dims, last ? 0 : 1, n->d_err, s));
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
  if (e == cudaSuccess) e = cudaMalloc((void**)&n->d_err, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(n->d_err, 0, sizeof(int));
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
                  (void*)n->d_g0, (void*)n->d_g1, (void*)n->d_out, (void*)n->d_part, (void*)n->d_loss,
                  (void*)n->d_err})
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
    LLR_TRY(wgrad(n->cin[l], n->cout[l], n->act[l], g, n->d_part, n->part_cap, n->d_grad + n->w_off[l], dims,
                  n->d_err, s));
    if (l == 0) break;
    // dL/d act[l] = conv(g, W') masked by the ReLU that produced act[l]
    LLR_TRY(conv(n->cout[l], n->cin[l], g, n->d_wt + wtab_off(n, l), nullptr, nullptr, gn, dims, 0, n->d_err, s));
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
    int herr = 0;
    LLR_CUDA_TRY(cudaMemcpy(&herr, n->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (herr) return set_error(LLR_ERR_CUDA, "a tensor-core wait in a conv3d kernel timed out");
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
                              float scale, const llr_cf32* d_phase_ref, float* d_chan, void* stream) {
  if (!d_x || !vol || !d_S || !d_chan || nq < 1 || srank < 1 || srank > 16)
    return set_error(LLR_ERR_INVALID, "bad subspace channel arguments (1 <= srank <= 16)");
  const long long V = (long long)vol[0] * vol[1] * vol[2];
  note_launch();
  subspace_channels_kernel<<<grid_1d(V), 256, sizeof(float2) * nq * srank, (cudaStream_t)stream>>>(
      (const float2*)d_x, V, nq, (const float2*)d_S, srank, scale, (const float2*)d_phase_ref, d_chan);
  LLR_CUDA_TRY(cudaGetLastError());
  return LLR_OK;
}

int llr_subspace_image_dev(const float* d_chan, const int32_t* vol, int32_t nq, const llr_cf32* d_S, int32_t srank,
                           float scale, const llr_cf32* d_phase_ref, int32_t accumulate, llr_cf32* d_x, void* stream) {
  if (!d_x || !vol || !d_S || !d_chan || nq < 1 || srank < 1 || srank > 16 || !(scale != 0.f))
    return set_error(LLR_ERR_INVALID, "bad subspace image arguments (1 <= srank <= 16, scale != 0)");
  const long long V = (long long)vol[0] * vol[1] * vol[2];
  note_launch();
  subspace_image_kernel<<<grid_1d(V), 256, sizeof(float2) * nq * srank, (cudaStream_t)stream>>>(
      d_chan, V, nq, (const float2*)d_S, srank, 1.f / scale, (const float2*)d_phase_ref, (float2*)d_x,
      accumulate ? 1 : 0);
  LLR_CUDA_TRY(cudaGetLastError());
  return LLR_OK;
}

}  // extern "C"
