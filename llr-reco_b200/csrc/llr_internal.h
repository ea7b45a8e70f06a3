// Internal declarations shared by the library translation units.
#pragma once

#include <cufft.h>
#include <vector>
#include <mutex>

#include "llr_common.cuh"

namespace llr {

constexpr int kLlrThreads = 256;

// Where the Casorati matrices of one prox launch come from and go to.
struct BlockSource {
  int kind;            // 0: contiguous (m, n, batch) matrices; 1: planar volume blocks
  float2* data;
  long long nblocks;
  // kind 1 only
  Geom g;
  int bx, by, bz;      // block size
  int gx, gy, gz;      // blocks per axis
  int sx, sy, sz;      // explicit shift (used when it_ptr == nullptr)
  const long long* it_ptr;  // device iteration counter; shift drawn on device when set
  unsigned long long seed;
  int mx, my, mz;      // max random shift per axis
  float load_scale;    // value = raw * load_scale * conj(phase)
  PhaseTab ph;         // phase tables (null members: identity)
  int store_phase;     // 1: stored value = value * phase; 0: stored value = value
  float store_scale;   // stored value additionally scaled by this factor
  int ph_uniform;      // every volume has the same phase tables (per-row phase suffices)
  const int* blk_list; // optional list of block indices (with blk_count) instead of 0..nblocks-1
  const int* blk_count;
  int ox, oy, oz;      // offset added to the (drawn or explicit) shift: one phase of an overlapping grid
  float2* out;         // null: results go back to `data`; else to `out` (same layout; planar only)
  int accumulate;      // with `out`: out += result (zero results are skipped) instead of out = result
};

struct ProxOp {
  int m, n;
  int mode;            // LLR_PROX_HARD_RANK / LLR_PROX_SOFT_THRESH
  int rank;
  float lambda;
  float* block_stat;   // when non-null: write the largest Gram eigenvalue, skip the update
  int eig_solver;      // 0: tridiagonal, one warp per block; 1: Jacobi
  int* fb_list;        // blocks handed to the Jacobi kernel (capacity nblocks)
  int* fb_count;
  float2* gram;        // optional scratch, nblocks * gram_stride: selects the split Gram/eigen path
  long long gram_stride;   // float2 per block in `gram` (prox_gram_stride(n))
  int* blk_ra;         // split path: kept count per block (+1 int: the eigen kernel's queue)
  int gram_mode;       // 0: 3xTF32 on tensor cores (tcgen05) where 2n <= 128; 1: FP32 FMA
  int* err;            // device flag set when a bounded wait gives up (never expected)
  int defer_zero = 0;  // 1: the apply kernel leaves blocks with r_a = 0 unwritten; the fused
                       // FFT that follows in the same iteration zero-fills them as it loads
  float2* vwide = nullptr;  // 64 < n <= 128: per-CTA eigenvector scratch of the wide Jacobi kernel,
  int vwide_ctas = 0;       // vwide_ctas * wide_v_stride() float2
  double* blk_nuc = nullptr;   // soft threshold: per block sum over its singular values s of
                               // (s - lambda)+ in FP64, the nuclear norm of the block's prox output
                               // (the regulariser term of the objective); blocks left at 0 keep none
};

// Widest Casorati column count of the prox kernels, and the per-CTA eigenvector scratch the
// wide (64 < n <= 128) Jacobi kernel needs, in float2.
constexpr int kProxMaxN = 128;
__host__ __device__ inline long long wide_v_stride() { return (long long)kProxMaxN * (kProxMaxN + 1); }
int wide_jacobi_ctas();   // CTAs of the wide Jacobi kernel on the current device

// Kept eigenvectors per block that the warp eigen kernel hands to the apply kernel.
constexpr int kFacCols = 8;

// Per-block scratch of the split prox path, in float2: the packed Gram matrix n(n+1)/2,
// overwritten by the eigen factor (n x kFacCols eigenvectors, then kFacCols gains).
inline long long prox_gram_stride(int n) {
  const long long p = (long long)n * (n + 1) / 2, f = (long long)n * kFacCols + kFacCols;
  return p > f ? p : f;
}

bool fft_dc_supported(int ny, int nz);
std::vector<float2> fft_dc_twiddles(int ny, int nz);
int fft_dc_grid(int ny, int nz);
int launch_fft_dc(float2* u, const float2* yhat, const int* pos, const long long* off, const float2* twiddle,
                  const Geom& g, double* partials, int grid, const int* zero_ra, const BlockSource* zsrc,
                  cudaStream_t s);
int launch_diff_norm(const float2* a, const float2* b, long long n, double* part_d, double* part_b, int nblocks,
                     cudaStream_t s);
int launch_llr_eig_warp(const ProxOp& op, long long nblocks, cudaStream_t stream);

int launch_llr_prox(const BlockSource& src, const ProxOp& op, cudaStream_t stream);
bool llr_prox_supported(int m, int n);
bool prox_needs_wide_fallback(int m, int n);   // n <= 64 whose blocks the Jacobi kernel cannot stage
bool llr_gram_tc_supported(int m, int n);
int launch_llr_gram_tc(const BlockSource& src, const ProxOp& op, cudaStream_t stream);

struct SubspaceOp {
  int m, nq, srank;
  int mode, rank;
  float lambda;
  const float2* S;     // nq x srank column-major
  float2* coef_out = nullptr;  // when set (planar source): store the coefficient volumes LR(X S)
                               // (planar, srank volumes, image space) here instead of X'
};
int launch_llr_prox_subspace(const BlockSource& src, const SubspaceOp& op, cudaStream_t stream);
// x(., q) = (sum_k c(., k) conj(S[q, k])) * phase(q, .) * scale, planar volumes (nq from srank)
int launch_subspace_expand(const float2* coef, float2* x, const float2* S, int srank, const Geom& g, PhaseTab ph,
                           int store_phase, int ph_uniform, float scale, cudaStream_t s);

// layout / transform kernels (signal_model.cu)
int launch_ref_to_planar(const float2* ref, float2* planar, const Geom& g, float scale, PhaseTab ph,
                         int phase_sign, cudaStream_t s);
int launch_planar_to_ref(const float2* planar, float2* ref, const Geom& g, float scale, PhaseTab ph,
                         int phase_sign, cudaStream_t s);
int launch_scale_uncovered(float2* data, const Geom& g, const int* grid_cover, const long long* it_ptr,
                           unsigned long long seed, const int shift[3], const int maxs[3], float scale,
                           PhaseTab ph, int conj_phase, cudaStream_t s);

// wavelet (wavelet.cu)
struct WaveletPlan {
  int nx, ny, nz;      // volume size (in the storage axis order used by the caller)
  int levels;
  int flen;
  float lo_d[20], hi_d[20], lo_r[20], hi_r[20];
  std::vector<int> sizes;   // per level l: input extents (3 ints) ; level count + 1 entries
};
int wavelet_plan_init(WaveletPlan* p, int nx, int ny, int nz, int moments, int levels);
size_t wavelet_workspace_elems(const WaveletPlan& p, int nvol);
// Denoise nvol volumes stored with element (ix,iy,iz,v) at ix*sx + iy*sy + iz*sz + v*sv.
int wavelet_denoise_strided(const WaveletPlan& p, float2* data, long long sx, long long sy, long long sz,
                            long long sv, int nvol, float alpha, float2* work, cudaStream_t s);

// plan cache for stand-alone signal-model calls
int get_c2c_plan(int rank, const long long* n, long long batch, cufftHandle* out);
int cufft_error(cufftResult r, const char* what);

}  // namespace llr

// -------------------------------------------------------------------------------------
// context
// -------------------------------------------------------------------------------------
struct llr_ctx {
  llr_config cfg;
  int device;
  cudaStream_t stream;
  bool own_stream;
  Geom g;
  int m;                    // voxels per block
  int gx, gy, gz;           // block grid
  long long nblocks;
  // state
  bool have_kspace;
  bool have_image;
  bool hybrid;              // line-structured measurements: x-transform eliminated
  bool fused_fft;           // hybrid and the (y, z) plane fits fft_dc_kernel
  int fft_grid;             // fft_dc_kernel CTAs (= residual partials)
  float2* d_fft_tw;         // fft_dc_kernel twiddle table
  float load_scale;         // 1 / N_t
  // device buffers
  float2* d_x;              // iterate (planar, raw convention)
  float2* d_work;           // E-sized scratch
  float2* d_yhat;           // hybrid: compact sampled lines; general: full planar
  int* d_samp_pos;          // hybrid: sampled (ky + ny*kz) per volume, concatenated
  long long* d_samp_off;    // hybrid: nq + 1 offsets into d_samp_pos
  std::vector<long long> h_samp_off;
  long long n_samp_lines;
  float2* d_ph_ksp;         // (nx + ny + nz) * nq  image-domain phase  e^{+i theta_ksp}
  float2* d_ph_img;         // (nx + ny + nz) * nq  k-domain phase      e^{+i theta_img}
  float2* d_S;              // subspace (nq x srank)
  double* d_partials;
  int n_partials;
  double* d_hist;
  long long hist_cap;
  double* d_obj;            // objective per iteration (FP64; NaN where the model has none)
  double* d_blk_nuc;        // per-block nuclear-norm terms of the current iteration's prox
  int obj_mode;             // 0: no objective, 1: data term only (hard rank), 2: data + lambda nuclear
  long long* d_iter;
  long long h_iter;         // host mirror (valid after sync)
  float* d_block_stat;
  int* d_fb;                // Jacobi fallback block list (nblocks) + count
  float2* d_gram;           // per-block packed Gram matrices (split prox path)
  int* d_blk_ra;            // per-block kept count of the split prox path + queue counter
  int* d_err;               // device error flag of the prox kernels
  int ph_uniform;           // all volumes share the image-domain phase tables
  float2* d_vwide;          // eigenvector scratch of the wide (64 < nq <= 128) Jacobi kernel
  int vwide_ctas;
  std::vector<int> phase_off;   // overlapping blocks: 3 offsets per phase (empty: non-overlapping)
  float2* d_wavelet_work;
  size_t wavelet_work_elems;
  llr::WaveletPlan wplan;
  bool wavelet_on;
  // FFT
  cufftHandle plan_fwd;     // hybrid: 2-D over (z, y) per plane; general: 3-D
  bool have_plan;
  void* d_fft_work;
  size_t fft_work_bytes;
  // graph
  cudaGraph_t graph;
  cudaGraphExec_t graph_exec;
  bool have_graph;
  cudaGraphExec_t stage_exec[5];
  bool have_stages;
  int launches_per_iter;   // library kernels one iteration launches (counted at capture)
  // measurement stats
  double total_energy;
  double undersampling;
  std::vector<float> lin_ksp, lin_img;   // nq * 3
};

namespace llr {
int ctx_enqueue_iteration(llr_ctx* ctx, cudaStream_t s);
int ctx_prox(llr_ctx* ctx, cudaStream_t s, const int* explicit_shift, float* block_stat);
int check_device_error(llr_ctx* ctx);
PhaseTab ctx_phase(const llr_ctx* ctx, const float2* base, bool with_x);
}
