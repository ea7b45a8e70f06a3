// Device-resident reconstruction context: the replacement of llr_recon_exec's loop
// (lib.rs:113-363) with every buffer on the GPU and one CUDA graph per iteration.
//
// Iterate convention.  Between iterations d_x holds the raw inverse-FFT output w in the
// planar layout; the image is x = (1/N_t) e^{-i theta_ksp} w (N_t = ny*nz on the hybrid
// path, nx*ny*nz on the element-wise path).  The LLR gather applies that map on load
// and its scatter stores e^{+i theta_ksp} x, which is exactly the forward FFT's input, so
// neither ramp nor scaling needs a pass of its own.
#include <cstdio>
#include <cstring>
#include <cmath>
#include <algorithm>
#include <new>

#include "llr_internal.h"

namespace llr {

int launch_dc_hybrid(float2* u, const float2* yhat, const int* pos, const long long* off, const Geom& g, int max_lines,
                     double* partials, int n_part_x, int replace_only, cudaStream_t s);
int launch_dc_full(float2* u, const float2* yhat, long long n, double* partials, int nblocks, int replace_only,
                   cudaStream_t s);
int launch_objective(const double* blk_nuc, long long nb, double lam, const double* hist, double* obj, long long cap,
                     const long long* it, cudaStream_t s);
int launch_finalize(const double* partials, int np, double scale, double* hist, long long cap, long long* it,
                    int advance, double* out, cudaStream_t s);
int launch_line_nnz(const float2* y, long long nlines, int nx, int* cnt, cudaStream_t s);
int launch_energy(const float2* y, long long n, double* part_e, double* part_n, int nblocks, cudaStream_t s);
int launch_gather_lines(const float2* yh, float2* yhat, const int* pos, const long long* off, const Geom& g,
                        PhaseTab ph_img, float scale, cudaStream_t s);
int launch_prep_full(float2* y, const Geom& g, PhaseTab ph_img, float scale, cudaStream_t s);
int launch_phase_x(float2* x, const Geom& g, int nvol, const float2* tx, int sign, float scale, cudaStream_t s);
int launch_scale(float2* x, long long n, float sc, cudaStream_t s);
void phase_tables_host(const int dims[3], int nvol, const float* corr, float2* out);
int wavelet_denoise_strided_xf(const WaveletPlan& p, float2* data, long long sx, long long sy, long long sz,
                               long long sv, int nvol, float alpha, float2* work, PhaseTab ph, const Geom* g,
                               int q0, float store_scale, cudaStream_t s);

namespace {
constexpr int kPartX = 64;          // DC partial blocks per volume (hybrid)
constexpr int kPartFull = 1184;     // DC partial blocks (element-wise)
constexpr long long kHistCap = 1 << 16;

int ensure_no_capture(llr_ctx* c) {
  cudaStreamCaptureStatus st;
  LLR_CUDA_TRY(cudaStreamIsCapturing(c->stream, &st));
  if (st != cudaStreamCaptureStatusNone) return set_error(LLR_ERR_STATE, "context stream is being captured");
  return LLR_OK;
}

void drop_graph(llr_ctx* c) {
  if (c->have_graph) {
    cudaGraphExecDestroy(c->graph_exec);
    cudaGraphDestroy(c->graph);
    c->have_graph = false;
  }
  if (c->have_stages) {
    for (int i = 0; i < 5; ++i)
      if (c->stage_exec[i]) cudaGraphExecDestroy(c->stage_exec[i]);
    c->have_stages = false;
  }
}

int exec_fft(llr_ctx* c, float2* d, int dir, cudaStream_t s) {
  cufftResult r = cufftSetStream(c->plan_fwd, s);
  if (r != CUFFT_SUCCESS) return cufft_error(r, "cufftSetStream");
  r = cufftExecC2C(c->plan_fwd, (cufftComplex*)d, (cufftComplex*)d, dir);
  if (r != CUFFT_SUCCESS) return cufft_error(r, "cufftExecC2C");
  return LLR_OK;
}

int upload_tables(llr_ctx* c) {
  const int dims[3] = {c->g.nx, c->g.ny, c->g.nz};
  const size_t nt = (size_t)c->g.nq * (c->g.nx + c->g.ny + c->g.nz);
  std::vector<float2> h(2 * nt);
  phase_tables_host(dims, c->g.nq, c->lin_ksp.data(), h.data());
  phase_tables_host(dims, c->g.nq, c->lin_img.data(), h.data() + nt);
  c->ph_uniform = 1;
  for (int q = 1; q < c->g.nq; ++q)
    for (int a = 0; a < 3; ++a)
      if (c->lin_ksp[3 * q + a] != c->lin_ksp[a]) c->ph_uniform = 0;
  LLR_CUDA_TRY(cudaMemcpyAsync(c->d_ph_ksp, h.data(), sizeof(float2) * nt, cudaMemcpyHostToDevice, c->stream));
  LLR_CUDA_TRY(cudaMemcpyAsync(c->d_ph_img, h.data() + nt, sizeof(float2) * nt, cudaMemcpyHostToDevice, c->stream));
  LLR_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return LLR_OK;
}

template <class T>
int dalloc(T** p, size_t n) {
  *p = nullptr;
  if (n == 0) n = 1;
  LLR_CUDA_TRY(cudaMalloc((void**)p, n * sizeof(T)));
  return LLR_OK;
}

void dfree(void* p) {
  if (p) cudaFree(p);
}

int make_plan(llr_ctx* c) {
  if (c->have_plan) {
    cufftDestroy(c->plan_fwd);
    c->have_plan = false;
  }
  cufftResult r = cufftCreate(&c->plan_fwd);
  if (r != CUFFT_SUCCESS) return cufft_error(r, "cufftCreate");
  c->have_plan = true;
  r = cufftSetAutoAllocation(c->plan_fwd, 0);
  if (r != CUFFT_SUCCESS) return cufft_error(r, "cufftSetAutoAllocation");
  size_t ws = 0;
  if (c->hybrid) {
    long long n[2] = {c->g.nz, c->g.ny};
    r = cufftMakePlanMany64(c->plan_fwd, 2, n, nullptr, 1, c->g.nyz, nullptr, 1, c->g.nyz, CUFFT_C2C,
                            (long long)c->g.nx * c->g.nq, &ws);
  } else {
    long long n[3] = {c->g.nx, c->g.nz, c->g.ny};
    r = cufftMakePlanMany64(c->plan_fwd, 3, n, nullptr, 1, c->g.V, nullptr, 1, c->g.V, CUFFT_C2C, c->g.nq, &ws);
  }
  if (r != CUFFT_SUCCESS) return cufft_error(r, "cufftMakePlanMany64");
  if (ws > c->fft_work_bytes) {
    dfree(c->d_fft_work);
    c->d_fft_work = nullptr;
    LLR_CUDA_TRY(cudaMalloc(&c->d_fft_work, ws));
    c->fft_work_bytes = ws;
  }
  r = cufftSetWorkArea(c->plan_fwd, c->d_fft_work);
  if (r != CUFFT_SUCCESS) return cufft_error(r, "cufftSetWorkArea");
  return LLR_OK;
}

}  // namespace

int check_device_error(llr_ctx* c) {
  int h = 0;
  LLR_CUDA_TRY(cudaMemcpy(&h, c->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (h != 0) return set_error(LLR_ERR_CUDA, "a tensor-core wait in the prox kernel timed out (device flag %d)", h);
  return LLR_OK;
}

PhaseTab ctx_phase(const llr_ctx* c, const float2* base, bool with_x) {
  PhaseTab t;
  t.x = with_x ? base : nullptr;
  t.y = base + (size_t)c->g.nq * c->g.nx;
  t.z = t.y + (size_t)c->g.nq * c->g.ny;
  return t;
}

static BlockSource make_source(llr_ctx* c, const int* explicit_shift, float store_scale_unused) {
  (void)store_scale_unused;
  BlockSource s;
  memset(&s, 0, sizeof(s));
  s.kind = 1;
  s.data = c->d_x;
  s.nblocks = c->nblocks;
  s.g = c->g;
  s.bx = c->cfg.block_size[0]; s.by = c->cfg.block_size[1]; s.bz = c->cfg.block_size[2];
  s.gx = c->gx; s.gy = c->gy; s.gz = c->gz;
  s.seed = c->cfg.seed;
  s.mx = c->cfg.max_rand_shift[0] > 0 ? c->cfg.max_rand_shift[0] : c->g.nx;
  s.my = c->cfg.max_rand_shift[1] > 0 ? c->cfg.max_rand_shift[1] : c->g.ny;
  s.mz = c->cfg.max_rand_shift[2] > 0 ? c->cfg.max_rand_shift[2] : c->g.nz;
  if (explicit_shift) {
    s.it_ptr = nullptr;
    s.sx = explicit_shift[0]; s.sy = explicit_shift[1]; s.sz = explicit_shift[2];
  } else {
    s.it_ptr = c->d_iter;
  }
  s.load_scale = c->load_scale;
  s.ph = ctx_phase(c, c->d_ph_ksp, !c->hybrid);
  s.store_phase = 1;
  s.store_scale = 1.f;
  s.ph_uniform = c->ph_uniform;
  s.blk_list = nullptr;
  s.blk_count = nullptr;
  return s;
}

// Inside an iteration whose DC stage is the fused FFT kernel, the prox leaves blocks whose output
// is zero (every singular value below the threshold) unwritten, and the fused kernel zero-fills
// them as it loads its planes: their bytes are neither written nor read.  Only the split prox
// path (warp eigen kernel + apply kernel) reports such blocks, and nothing may read the iterate
// between the two stages (no wavelet stage).
static bool defer_zero_blocks(const llr_ctx* c) {
  return c->fused_fft && !c->wavelet_on && c->phase_off.empty() && c->cfg.subspace_rank == 0 && c->cfg.eig_solver == 0 &&
         c->d_gram != nullptr && c->d_blk_ra != nullptr && c->g.nq <= 64 &&
         (long long)c->gy * c->gz <= 4096;
}

// Inside an iteration with a subspace and wavelet_space == 1, the prox stores the subspace
// coefficient volumes LR(X S) in d_work, the wavelet shrinks those srank volumes, and an expand
// kernel writes X = C S^H (the FFT input) back to d_x.
static bool coef_mode(const llr_ctx* c) {
  return c->cfg.subspace_rank > 0 && c->wavelet_on && c->cfg.wavelet_space == 1;
}

// One prox pass on d_x.  standalone == true keeps the raw convention (used by single-step
// entry points); otherwise the output is the FFT input (or the image, if the wavelet runs).
static int prox_pass(llr_ctx* c, cudaStream_t s, const int* explicit_shift, bool standalone, float* block_stat) {
  BlockSource src = make_source(c, explicit_shift, 1.f);
  if (standalone) {
    src.store_phase = 1;
    src.store_scale = 1.f / c->load_scale;
  } else {
    src.store_phase = c->wavelet_on ? 0 : 1;
    src.store_scale = 1.f;
  }
  if (c->cfg.subspace_rank > 0 && !block_stat) {
    SubspaceOp op;
    op.m = c->m; op.nq = c->g.nq; op.srank = c->cfg.subspace_rank;
    op.mode = c->cfg.prox_mode; op.rank = c->cfg.rank; op.lambda = c->cfg.lambda;
    op.S = c->d_S;
    if (!standalone && coef_mode(c)) {
      op.coef_out = c->d_work;
      return launch_llr_prox_subspace(src, op, s);   // the blocks tile the volume (validated)
    }
    LLR_TRY(launch_llr_prox_subspace(src, op, s));
  } else {
    ProxOp op;
    op.m = c->m; op.n = c->g.nq; op.mode = c->cfg.prox_mode; op.rank = c->cfg.rank; op.lambda = c->cfg.lambda;
    op.block_stat = block_stat;
    op.eig_solver = c->cfg.eig_solver;
    op.fb_list = c->d_fb;
    op.fb_count = c->d_fb + std::max<long long>(1, c->nblocks);
    op.gram = c->d_gram;
    op.gram_stride = prox_gram_stride(c->g.nq);
    op.blk_ra = c->d_blk_ra;
    op.gram_mode = c->cfg.gram_mode;
    op.err = c->d_err;
    op.defer_zero = (!standalone && !block_stat && !explicit_shift && defer_zero_blocks(c)) ? 1 : 0;
    op.vwide = c->d_vwide;
    op.vwide_ctas = c->vwide_ctas;
    if (c->obj_mode == 2 && !standalone && !block_stat && !explicit_shift) {
      LLR_CUDA_TRY(cudaMemsetAsync(c->d_blk_nuc, 0, sizeof(double) * (size_t)std::max<long long>(1, c->nblocks), s));
      op.blk_nuc = c->d_blk_nuc;
    }
    if (!c->phase_off.empty() && !block_stat) {
      // overlapping blocks: every phase of the strided grid is a non-overlapping tiling at the
      // shift plus the phase offset; the mean of the phases goes to d_work, then back to d_x
      const int P = (int)c->phase_off.size() / 3;
      for (int p = 0; p < P; ++p) {
        BlockSource ps = src;
        ps.ox = c->phase_off[3 * p]; ps.oy = c->phase_off[3 * p + 1]; ps.oz = c->phase_off[3 * p + 2];
        ps.out = c->d_work;
        ps.accumulate = p > 0;
        ps.store_scale = src.store_scale / (float)P;
        LLR_TRY(launch_llr_prox(ps, op, s));
      }
      LLR_CUDA_TRY(cudaMemcpyAsync(c->d_x, c->d_work, sizeof(float2) * (size_t)c->g.V * c->g.nq,
                                   cudaMemcpyDeviceToDevice, s));
      return LLR_OK;   // the blocks tile the volume (validated)
    }
    LLR_TRY(launch_llr_prox(src, op, s));
  }
  if (block_stat || standalone) return LLR_OK;
  const int cover[3] = {c->gx * c->cfg.block_size[0], c->gy * c->cfg.block_size[1], c->gz * c->cfg.block_size[2]};
  if (cover[0] < c->g.nx || cover[1] < c->g.ny || cover[2] < c->g.nz) {
    const int maxs[3] = {src.mx, src.my, src.mz};
    LLR_TRY(launch_scale_uncovered(c->d_x, c->g, cover, explicit_shift ? nullptr : c->d_iter, c->cfg.seed,
                                   explicit_shift, maxs, c->load_scale, src.ph, c->wavelet_on ? 1 : 0, s));
  }
  return LLR_OK;
}

// Wavelet shrink on the image held in d_x; stores e^{+i theta_ksp} x * store_scale.  In an
// iteration in coefficient mode: shrink the coefficient volumes in d_work, then expand them into
// d_x as the FFT input.
static int wavelet_pass(llr_ctx* c, cudaStream_t s, float store_scale, bool in_iteration = false) {
  const long long sx = c->g.nyz, sy = 1, sz = c->g.ny, sv = c->g.V;
  if (in_iteration && coef_mode(c)) {
    const int sr = c->cfg.subspace_rank;
    const int nb = std::max(1, (int)(c->wavelet_work_elems / wavelet_workspace_elems(c->wplan, 1)));
    PhaseTab none{nullptr, nullptr, nullptr};
    for (int k0 = 0; k0 < sr; k0 += nb)
      LLR_TRY(wavelet_denoise_strided_xf(c->wplan, c->d_work + (size_t)k0 * c->g.V, sx, sy, sz, sv,
                                         std::min(nb, sr - k0), c->cfg.wavelet_alpha, c->d_wavelet_work, none,
                                         nullptr, 0, 1.f, s));
    return launch_subspace_expand(c->d_work, c->d_x, c->d_S, sr, c->g, ctx_phase(c, c->d_ph_ksp, !c->hybrid), 1,
                                  c->ph_uniform, store_scale, s);
  }
  const int nb = std::max(1, (int)(c->wavelet_work_elems / wavelet_workspace_elems(c->wplan, 1)));
  PhaseTab ph = ctx_phase(c, c->d_ph_ksp, !c->hybrid);
  for (int q0 = 0; q0 < c->g.nq; q0 += nb) {
    const int nv = std::min(nb, c->g.nq - q0);
    LLR_TRY(wavelet_denoise_strided_xf(c->wplan, c->d_x + (size_t)q0 * c->g.V, sx, sy, sz, sv, nv,
                                       c->cfg.wavelet_alpha, c->d_wavelet_work, ph, &c->g, q0, store_scale, s));
  }
  return LLR_OK;
}

static int dc_pass(llr_ctx* c, cudaStream_t s, int replace_only) {
  if (c->hybrid) {
    return launch_dc_hybrid(c->d_x, c->d_yhat, c->d_samp_pos, c->d_samp_off, c->g, 0, c->d_partials, kPartX,
                            replace_only, s);
  }
  return launch_dc_full(c->d_x, c->d_yhat, c->g.V * c->g.nq, c->d_partials, kPartFull, replace_only, s);
}

static int n_partials(const llr_ctx* c) { return c->hybrid ? kPartX * c->g.nq : kPartFull; }

// Residual of iteration k from the DC partials into the history (advancing the counter), then
// the objective of the prox output of the same iteration.
static int finalize_iteration(llr_ctx* c, int np, cudaStream_t s) {
  LLR_TRY(launch_finalize(c->d_partials, np, (double)c->load_scale, c->d_hist, c->hist_cap, c->d_iter, 1, nullptr, s));
  if (c->obj_mode == 0) return LLR_OK;
  return launch_objective(c->obj_mode == 2 ? c->d_blk_nuc : nullptr, std::max<long long>(1, c->nblocks),
                          (double)c->cfg.lambda, c->d_hist, c->d_obj, c->hist_cap, c->d_iter, s);
}

// Forward 2-D DFT, DC with residual, inverse 2-D DFT in one kernel; residual finalized.
static int fused_dc_pass(llr_ctx* c, cudaStream_t s, double* out) {
  const bool zf = defer_zero_blocks(c);
  const BlockSource zsrc = make_source(c, nullptr, 1.f);
  LLR_TRY(launch_fft_dc(c->d_x, c->d_yhat, c->d_samp_pos, c->d_samp_off, c->d_fft_tw, c->g, c->d_partials,
                        c->fft_grid, zf ? c->d_blk_ra : nullptr, zf ? &zsrc : nullptr, s));
  if (!out) return finalize_iteration(c, c->fft_grid, s);
  return launch_finalize(c->d_partials, c->fft_grid, (double)c->load_scale, nullptr, 0, nullptr, 0, out, s);
}

int ctx_enqueue_iteration(llr_ctx* c, cudaStream_t s) {
  LLR_TRY(prox_pass(c, s, nullptr, false, nullptr));
  if (c->wavelet_on) LLR_TRY(wavelet_pass(c, s, 1.f, true));
  if (c->fused_fft) return fused_dc_pass(c, s, nullptr);
  LLR_TRY(exec_fft(c, c->d_x, CUFFT_FORWARD, s));
  LLR_TRY(dc_pass(c, s, 0));
  LLR_TRY(finalize_iteration(c, n_partials(c), s));
  LLR_TRY(exec_fft(c, c->d_x, CUFFT_INVERSE, s));
  return LLR_OK;
}

}  // namespace llr

using namespace llr;

extern "C" {

int llr_ctx_create(const llr_config* cfg, llr_ctx** out) {
  if (!out) return set_error(LLR_ERR_INVALID, "null output pointer");
  *out = nullptr;
  LLR_TRY(llr_config_validate(cfg));
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) return set_error(LLR_ERR_NO_DEVICE, "no CUDA device available");
  if (cfg->device < 0 || cfg->device >= ndev) return set_error(LLR_ERR_INVALID, "device %d out of range", cfg->device);
  LLR_CUDA_TRY(cudaSetDevice(cfg->device));
  llr_ctx* c = new (std::nothrow) llr_ctx();
  if (!c) return set_error(LLR_ERR_NOMEM, "host allocation failed");
  c->cfg = *cfg;
  c->device = cfg->device;
  c->g.nx = cfg->vol_size[0]; c->g.ny = cfg->vol_size[1]; c->g.nz = cfg->vol_size[2]; c->g.nq = cfg->nq;
  c->g.nyz = (long long)c->g.ny * c->g.nz;
  c->g.V = (long long)c->g.nx * c->g.nyz;
  c->m = cfg->block_size[0] * cfg->block_size[1] * cfg->block_size[2];
  c->gx = c->g.nx / cfg->block_size[0];
  c->gy = c->g.ny / cfg->block_size[1];
  c->gz = c->g.nz / cfg->block_size[2];
  c->nblocks = (long long)c->gx * c->gy * c->gz;
  c->lin_ksp.assign((size_t)3 * c->g.nq, 0.f);
  c->lin_img.assign((size_t)3 * c->g.nq, 0.f);
  c->load_scale = 1.f;
  int st = LLR_OK;
  auto fail = [&](int s) { llr_ctx_destroy(c); return s; };
  if (cfg->subspace_rank == 0 && !llr_prox_supported(c->m, c->g.nq))
    return fail(set_error(LLR_ERR_UNSUPPORTED, "Casorati %d x %d exceeds the fused prox kernel (n <= 64, m*n*8 + "
                                               "2*64*65*8 <= 227 KiB)", c->m, c->g.nq));
  e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) return fail(cuda_error(e, "cudaStreamCreate", __FILE__, __LINE__));
  c->own_stream = true;
  const size_t E = (size_t)c->g.V * c->g.nq;
  const size_t nt = (size_t)c->g.nq * (c->g.nx + c->g.ny + c->g.nz);
  if ((st = dalloc(&c->d_x, E))) return fail(st);
  if ((st = dalloc(&c->d_work, E))) return fail(st);
  if ((st = dalloc(&c->d_ph_ksp, nt))) return fail(st);
  if ((st = dalloc(&c->d_ph_img, nt))) return fail(st);
  c->n_partials = std::max(kPartFull, kPartX * c->g.nq) + 8;
  if ((st = dalloc(&c->d_partials, (size_t)c->n_partials))) return fail(st);
  c->hist_cap = kHistCap;
  if ((st = dalloc(&c->d_hist, (size_t)c->hist_cap))) return fail(st);
  if ((st = dalloc(&c->d_obj, (size_t)c->hist_cap))) return fail(st);
  if ((st = dalloc(&c->d_blk_nuc, (size_t)std::max<long long>(1, c->nblocks)))) return fail(st);
  if ((st = dalloc(&c->d_iter, 1))) return fail(st);
  if ((st = dalloc(&c->d_block_stat, (size_t)std::max<long long>(1, c->nblocks)))) return fail(st);
  if ((st = dalloc(&c->d_fb, (size_t)std::max<long long>(1, c->nblocks) + 1))) return fail(st);
  if ((st = dalloc(&c->d_err, 1))) return fail(st);
  if (cfg->subspace_rank == 0 && (c->g.nq > 64 || prox_needs_wide_fallback(c->m, c->g.nq))) {
    c->vwide_ctas = wide_jacobi_ctas();
    if ((st = dalloc(&c->d_vwide, (size_t)c->vwide_ctas * (size_t)wide_v_stride()))) return fail(st);
  }
  {
    int per[3], P = 1;
    for (int a = 0; a < 3; ++a) {
      const int b = cfg->block_size[a], st2 = cfg->block_stride[a];
      per[a] = (st2 > 0 && st2 < b) ? b / st2 : 1;
      P *= per[a];
    }
    if (P > 1)
      for (int pz = 0; pz < per[2]; ++pz)
        for (int py = 0; py < per[1]; ++py)
          for (int px = 0; px < per[0]; ++px) {
            c->phase_off.push_back(px * (per[0] > 1 ? cfg->block_stride[0] : 0));
            c->phase_off.push_back(py * (per[1] > 1 ? cfg->block_stride[1] : 0));
            c->phase_off.push_back(pz * (per[2] > 1 ? cfg->block_stride[2] : 0));
          }
  }
  e = cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream);
  if (e != cudaSuccess) return fail(cuda_error(e, "cudaMemsetAsync", __FILE__, __LINE__));
  if (cfg->subspace_rank == 0 && c->g.nq <= 64 &&
      ((st = dalloc(&c->d_gram, (size_t)std::max<long long>(1, c->nblocks) * (size_t)prox_gram_stride(c->g.nq))) ||
       (st = dalloc(&c->d_blk_ra, (size_t)std::max<long long>(1, c->nblocks) + 1))))
    return fail(st);
  e = cudaMemsetAsync(c->d_iter, 0, sizeof(long long), c->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(c->d_hist, 0, sizeof(double) * c->hist_cap, c->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(c->d_obj, 0xFF, sizeof(double) * c->hist_cap, c->stream);   // NaN
  if (e == cudaSuccess) e = cudaMemsetAsync(c->d_x, 0, sizeof(float2) * E, c->stream);
  if (e != cudaSuccess) return fail(cuda_error(e, "cudaMemsetAsync", __FILE__, __LINE__));
  if (cfg->subspace_rank > 0 && (st = dalloc(&c->d_S, (size_t)c->g.nq * cfg->subspace_rank))) return fail(st);
  if (cfg->fft_mode == 0 && fft_dc_supported(c->g.ny, c->g.nz)) {   // fused FFT + DC twiddles (FP64-computed)
    const std::vector<float2> tw = fft_dc_twiddles(c->g.ny, c->g.nz);
    c->fft_grid = fft_dc_grid(c->g.ny, c->g.nz);
    if (c->fft_grid > 0) {
      if ((st = dalloc(&c->d_fft_tw, tw.size()))) return fail(st);
      e = cudaMemcpy(c->d_fft_tw, tw.data(), sizeof(float2) * tw.size(), cudaMemcpyHostToDevice);
      if (e != cudaSuccess) return fail(cuda_error(e, "cudaMemcpy", __FILE__, __LINE__));
    }
  }
  c->wavelet_on = false;
  if (cfg->wavelet_alpha > 0.f) {
    if ((st = wavelet_plan_init(&c->wplan, c->g.nx, c->g.ny, c->g.nz, cfg->wavelet_moments, cfg->wavelet_levels)))
      return fail(st);
    if (c->wplan.levels > 0) {
      const size_t per = wavelet_workspace_elems(c->wplan, 1);
      const size_t budget = std::max(per, (size_t)(4ull << 30) / sizeof(float2));
      int nb = (int)std::min<size_t>((size_t)c->g.nq, budget / per);
      nb = std::max(nb, 1);
      c->wavelet_work_elems = per * nb;
      if ((st = dalloc(&c->d_wavelet_work, c->wavelet_work_elems))) return fail(st);
      c->wavelet_on = true;
    }
  }
  // The objective 0.5 ||M A x - y||^2 + lambda sum_b ||X_b||_* is the function the iteration
  // minimises when the prox is the exact soft threshold of one tiling and nothing else acts on
  // the iterate; hard rank keeps the data term (the rank constraint holds by construction).
  // Overlapping tilings, wavelets and the subspace model have no such single objective here.
  const bool plain = cfg->subspace_rank == 0 && !c->wavelet_on && c->phase_off.empty();
  c->obj_mode = !plain ? 0 : (cfg->prox_mode == LLR_PROX_SOFT_THRESH ? 2 : 1);
  if ((st = upload_tables(c))) return fail(st);
  c->h_iter = 0;
  *out = c;
  return LLR_OK;
}

int llr_ctx_destroy(llr_ctx* c) {
  if (!c) return LLR_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  drop_graph(c);
  if (c->have_plan) cufftDestroy(c->plan_fwd);
  dfree(c->d_x); dfree(c->d_work); dfree(c->d_yhat); dfree(c->d_samp_pos); dfree(c->d_samp_off);
  dfree(c->d_ph_ksp); dfree(c->d_ph_img); dfree(c->d_S); dfree(c->d_partials); dfree(c->d_hist); dfree(c->d_iter);
  dfree(c->d_obj); dfree(c->d_blk_nuc);
  dfree(c->d_block_stat); dfree(c->d_fb); dfree(c->d_gram); dfree(c->d_blk_ra); dfree(c->d_fft_tw); dfree(c->d_err); dfree(c->d_vwide); dfree(c->d_wavelet_work); dfree(c->d_fft_work);
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return LLR_OK;
}

int llr_ctx_set_stream(llr_ctx* c, void* stream) {
  if (!c) return set_error(LLR_ERR_INVALID, "null context");
  LLR_CUDA_TRY(cudaSetDevice(c->device));
  LLR_CUDA_TRY(cudaStreamSynchronize(c->stream));
  if (!stream) return LLR_OK;
  if (c->own_stream) cudaStreamDestroy(c->stream);
  c->stream = (cudaStream_t)stream;
  c->own_stream = false;
  drop_graph(c);
  return LLR_OK;
}

int llr_ctx_get_config(const llr_ctx* c, llr_config* out) {
  if (!c || !out) return set_error(LLR_ERR_INVALID, "null pointer");
  *out = c->cfg;
  return LLR_OK;
}

int llr_set_linear_corrections(llr_ctx* c, const float* lk, const float* li) {
  if (!c) return set_error(LLR_ERR_INVALID, "null context");
  if (c->have_kspace) return set_error(LLR_ERR_STATE, "set linear corrections before uploading k-space");
  LLR_CUDA_TRY(cudaSetDevice(c->device));
  for (size_t i = 0; i < c->lin_ksp.size(); ++i) {
    c->lin_ksp[i] = lk ? lk[i] : 0.f;
    c->lin_img[i] = li ? li[i] : 0.f;
  }
  return upload_tables(c);
}

static int upload_kspace_device(llr_ctx* c) {
  // d_work holds y in the reference layout.
  cudaStream_t s = c->stream;
  const Geom& g = c->g;
  const long long E = g.V * g.nq;
  drop_graph(c);
  // measurement statistics (lib.rs:409-417)
  LLR_TRY(launch_energy(c->d_work, E, c->d_partials, c->d_partials + 512, 512, s));
  std::vector<double> hp(1024);
  LLR_CUDA_TRY(cudaMemcpyAsync(hp.data(), c->d_partials, sizeof(double) * 1024, cudaMemcpyDeviceToHost, s));
  // per-line non-zero counts
  const long long nlines = g.nyz * g.nq;
  int* d_cnt = nullptr;
  LLR_TRY(dalloc(&d_cnt, (size_t)nlines));
  int st = launch_line_nnz(c->d_work, nlines, g.nx, d_cnt, s);
  std::vector<int> cnt((size_t)nlines);
  if (st == LLR_OK) {
    cudaError_t e = cudaMemcpyAsync(cnt.data(), d_cnt, sizeof(int) * nlines, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) st = cuda_error(e, "line count copy", __FILE__, __LINE__);
  }
  dfree(d_cnt);
  if (st) return st;
  double en = 0, nnz = 0;
  for (int i = 0; i < 512; ++i) { en += hp[i]; nnz += hp[512 + i]; }
  c->total_energy = en;
  c->undersampling = nnz > 0 ? (double)E / nnz : INFINITY;
  bool structured = true;
  long long nsamp = 0;
  for (long long i = 0; i < nlines; ++i) {
    if (cnt[i] != 0 && cnt[i] != g.nx) structured = false;
    nsamp += cnt[i] != 0;
  }
  dfree(c->d_yhat); c->d_yhat = nullptr;
  dfree(c->d_samp_pos); c->d_samp_pos = nullptr;
  dfree(c->d_samp_off); c->d_samp_off = nullptr;
  c->hybrid = structured;
  c->fused_fft = structured && c->cfg.fft_mode == 0 && c->d_fft_tw != nullptr;
  PhaseTab ph_img_full = ctx_phase(c, c->d_ph_img, true);
  if (structured) {
    // sampled (ky + ny*kz) per volume
    std::vector<int> pos;
    pos.reserve((size_t)std::max<long long>(nsamp, 1));
    c->h_samp_off.assign((size_t)g.nq + 1, 0);
    for (int q = 0; q < g.nq; ++q) {
      c->h_samp_off[q] = (long long)pos.size();
      for (long long p = 0; p < g.nyz; ++p)
        if (cnt[(size_t)(p + g.nyz * q)] != 0) pos.push_back((int)p);
    }
    c->h_samp_off[g.nq] = (long long)pos.size();
    c->n_samp_lines = (long long)pos.size();
    LLR_TRY(dalloc(&c->d_samp_pos, pos.size()));
    LLR_TRY(dalloc(&c->d_samp_off, (size_t)g.nq + 1));
    LLR_CUDA_TRY(cudaMemcpyAsync(c->d_samp_pos, pos.data(), sizeof(int) * pos.size(), cudaMemcpyHostToDevice, s));
    LLR_CUDA_TRY(cudaMemcpyAsync(c->d_samp_off, c->h_samp_off.data(), sizeof(long long) * (g.nq + 1),
                                 cudaMemcpyHostToDevice, s));
    // y_h = A_x^H y along x: e^{+i theta_img,x} -> IFFT_x -> e^{-i theta_ksp,x} / sqrt(nx)
    LLR_TRY(launch_phase_x(c->d_work, g, g.nq, c->d_ph_img, +1, 1.f, s));
    cufftHandle px;
    long long n1[1] = {g.nx};
    LLR_TRY(get_c2c_plan(1, n1, g.nyz * g.nq, &px));
    cufftResult r = cufftSetStream(px, s);
    if (r != CUFFT_SUCCESS) return cufft_error(r, "cufftSetStream");
    r = cufftExecC2C(px, (cufftComplex*)c->d_work, (cufftComplex*)c->d_work, CUFFT_INVERSE);
    if (r != CUFFT_SUCCESS) return cufft_error(r, "cufftExecC2C (x)");
    LLR_TRY(launch_phase_x(c->d_work, g, g.nq, c->d_ph_ksp, -1, (float)(1.0 / std::sqrt((double)g.nx)), s));
    PhaseTab none{nullptr, nullptr, nullptr};
    LLR_TRY(launch_ref_to_planar(c->d_work, c->d_x, g, 1.f, none, 0, s));
    LLR_TRY(dalloc(&c->d_yhat, (size_t)std::max<long long>(1, c->n_samp_lines * g.nx)));
    LLR_TRY(launch_gather_lines(c->d_x, c->d_yhat, c->d_samp_pos, c->d_samp_off, g, ctx_phase(c, c->d_ph_img, false),
                                (float)std::sqrt((double)g.nyz), s));
    c->load_scale = (float)(1.0 / (double)g.nyz);
  } else {
    LLR_TRY(dalloc(&c->d_yhat, (size_t)E));
    PhaseTab none{nullptr, nullptr, nullptr};
    LLR_TRY(launch_ref_to_planar(c->d_work, c->d_yhat, g, 1.f, none, 0, s));
    LLR_TRY(launch_prep_full(c->d_yhat, g, ph_img_full, (float)std::sqrt((double)g.V), s));
    c->load_scale = (float)(1.0 / (double)g.V);
  }
  LLR_TRY(make_plan(c));
  LLR_CUDA_TRY(cudaStreamSynchronize(s));
  c->have_kspace = true;
  c->have_image = false;
  return LLR_OK;
}

int llr_upload_kspace(llr_ctx* c, const llr_cf32* y) {
  if (!c || !y) return set_error(LLR_ERR_INVALID, "null pointer");
  LLR_CUDA_TRY(cudaSetDevice(c->device));
  LLR_TRY(ensure_no_capture(c));
  const size_t bytes = sizeof(float2) * (size_t)c->g.V * c->g.nq;
  LLR_CUDA_TRY(cudaMemcpyAsync(c->d_work, y, bytes, cudaMemcpyHostToDevice, c->stream));
  return upload_kspace_device(c);
}

int llr_upload_kspace_dev(llr_ctx* c, const llr_cf32* d_y) {
  if (!c || !d_y) return set_error(LLR_ERR_INVALID, "null pointer");
  LLR_CUDA_TRY(cudaSetDevice(c->device));
  LLR_TRY(ensure_no_capture(c));
  const size_t bytes = sizeof(float2) * (size_t)c->g.V * c->g.nq;
  LLR_CUDA_TRY(cudaMemcpyAsync(c->d_work, d_y, bytes, cudaMemcpyDeviceToDevice, c->stream));
  return upload_kspace_device(c);
}

int llr_upload_subspace(llr_ctx* c, const llr_cf32* S) {
  if (!c || !S) return set_error(LLR_ERR_INVALID, "null pointer");
  if (c->cfg.subspace_rank <= 0) return set_error(LLR_ERR_STATE, "context was created without a subspace rank");
  LLR_CUDA_TRY(cudaSetDevice(c->device));
  LLR_CUDA_TRY(cudaMemcpyAsync(c->d_S, S, sizeof(float2) * (size_t)c->g.nq * c->cfg.subspace_rank,
                               cudaMemcpyHostToDevice, c->stream));
  LLR_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return LLR_OK;
}

int llr_init_zero_filled(llr_ctx* c) {
  if (!c) return set_error(LLR_ERR_INVALID, "null context");
  if (!c->have_kspace) return set_error(LLR_ERR_STATE, "upload k-space first");
  LLR_CUDA_TRY(cudaSetDevice(c->device));
  cudaStream_t s = c->stream;
  if (c->hybrid) LLR_CUDA_TRY(cudaMemsetAsync(c->d_x, 0, sizeof(float2) * (size_t)c->g.V * c->g.nq, s));
  LLR_TRY(dc_pass(c, s, 1));
  LLR_TRY(exec_fft(c, c->d_x, CUFFT_INVERSE, s));
  LLR_CUDA_TRY(cudaMemsetAsync(c->d_iter, 0, sizeof(long long), s));
  LLR_CUDA_TRY(cudaStreamSynchronize(s));
  c->h_iter = 0;
  c->have_image = true;
  return LLR_OK;
}

static int upload_image_common(llr_ctx* c) {
  PhaseTab ph = ctx_phase(c, c->d_ph_ksp, !c->hybrid);
  LLR_TRY(launch_ref_to_planar(c->d_work, c->d_x, c->g, 1.f / c->load_scale, ph, +1, c->stream));
  LLR_CUDA_TRY(cudaStreamSynchronize(c->stream));
  c->have_image = true;
  return LLR_OK;
}

int llr_upload_image(llr_ctx* c, const llr_cf32* x) {
  if (!c || !x) return set_error(LLR_ERR_INVALID, "null pointer");
  if (!c->have_kspace) return set_error(LLR_ERR_STATE, "upload k-space first (it fixes the iterate convention)");
  LLR_CUDA_TRY(cudaSetDevice(c->device));
  LLR_CUDA_TRY(cudaMemcpyAsync(c->d_work, x, sizeof(float2) * (size_t)c->g.V * c->g.nq, cudaMemcpyHostToDevice,
                               c->stream));
  return upload_image_common(c);
}

int llr_upload_image_dev(llr_ctx* c, const llr_cf32* d_x) {
  if (!c || !d_x) return set_error(LLR_ERR_INVALID, "null pointer");
  if (!c->have_kspace) return set_error(LLR_ERR_STATE, "upload k-space first (it fixes the iterate convention)");
  LLR_CUDA_TRY(cudaSetDevice(c->device));
  LLR_CUDA_TRY(cudaMemcpyAsync(c->d_work, d_x, sizeof(float2) * (size_t)c->g.V * c->g.nq, cudaMemcpyDeviceToDevice,
                               c->stream));
  return upload_image_common(c);
}

int llr_download_image_dev(llr_ctx* c, llr_cf32* d_out) {
  if (!c || !d_out) return set_error(LLR_ERR_INVALID, "null pointer");
  if (!c->have_image) return set_error(LLR_ERR_STATE, "no image: call llr_init_zero_filled or llr_upload_image");
  LLR_CUDA_TRY(cudaSetDevice(c->device));
  PhaseTab ph = ctx_phase(c, c->d_ph_ksp, !c->hybrid);
  LLR_TRY(launch_planar_to_ref(c->d_x, (float2*)d_out, c->g, c->load_scale, ph, -1, c->stream));
  LLR_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return LLR_OK;
}

int llr_download_image(llr_ctx* c, llr_cf32* x) {
  if (!c || !x) return set_error(LLR_ERR_INVALID, "null pointer");
  if (!c->have_image) return set_error(LLR_ERR_STATE, "no image: call llr_init_zero_filled or llr_upload_image");
  LLR_CUDA_TRY(cudaSetDevice(c->device));
  PhaseTab ph = ctx_phase(c, c->d_ph_ksp, !c->hybrid);
  LLR_TRY(launch_planar_to_ref(c->d_x, c->d_work, c->g, c->load_scale, ph, -1, c->stream));
  LLR_CUDA_TRY(cudaMemcpyAsync(x, c->d_work, sizeof(float2) * (size_t)c->g.V * c->g.nq, cudaMemcpyDeviceToHost,
                               c->stream));
  LLR_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return LLR_OK;
}

static int build_graph(llr_ctx* c) {
  drop_graph(c);
  cudaStream_t s = c->stream;
  LLR_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  const long long n0 = launch_counter;
  int st = ctx_enqueue_iteration(c, s);
  c->launches_per_iter = (int)(launch_counter - n0);
  cudaGraph_t graph = nullptr;
  cudaError_t e = cudaStreamEndCapture(s, &graph);
  if (st != LLR_OK) {
    if (graph) cudaGraphDestroy(graph);
    return st;
  }
  if (e != cudaSuccess) return cuda_error(e, "cudaStreamEndCapture", __FILE__, __LINE__);
  e = cudaGraphInstantiate(&c->graph_exec, graph, 0);
  if (e != cudaSuccess) {
    cudaGraphDestroy(graph);
    return cuda_error(e, "cudaGraphInstantiate", __FILE__, __LINE__);
  }
  c->graph = graph;
  c->have_graph = true;
  return LLR_OK;
}

static int capture_stage(llr_ctx* c, int stage, cudaGraphExec_t* out) {
  cudaStream_t s = c->stream;
  *out = nullptr;
  LLR_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  int st = LLR_OK;
  switch (stage) {
    case 0: st = prox_pass(c, s, nullptr, false, nullptr); break;
    case 1: if (c->wavelet_on) st = wavelet_pass(c, s, 1.f, true); break;
    case 2: st = c->fused_fft ? fused_dc_pass(c, s, nullptr) : exec_fft(c, c->d_x, CUFFT_FORWARD, s); break;
    case 3:
      if (c->fused_fft) break;
      st = dc_pass(c, s, 0);
      if (st == LLR_OK) st = finalize_iteration(c, n_partials(c), s);
      break;
    case 4: if (!c->fused_fft) st = exec_fft(c, c->d_x, CUFFT_INVERSE, s); break;
  }
  cudaGraph_t graph = nullptr;
  cudaError_t e = cudaStreamEndCapture(s, &graph);
  if (st != LLR_OK) {
    if (graph) cudaGraphDestroy(graph);
    return st;
  }
  if (e != cudaSuccess) return cuda_error(e, "cudaStreamEndCapture", __FILE__, __LINE__);
  e = cudaGraphInstantiate(out, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) return cuda_error(e, "cudaGraphInstantiate", __FILE__, __LINE__);
  return LLR_OK;
}

int llr_iterate_profiled(llr_ctx* c, int32_t n, double* stage_ms, double* total_ms) {
  if (!c) return set_error(LLR_ERR_INVALID, "null context");
  if (n < 1) return set_error(LLR_ERR_INVALID, "need at least one iteration");
  if (!c->have_kspace || !c->have_image) return set_error(LLR_ERR_STATE, "upload k-space and initialise the image");
  if (c->cfg.subspace_rank > 0 && !c->d_S) return set_error(LLR_ERR_STATE, "subspace not uploaded");
  LLR_CUDA_TRY(cudaSetDevice(c->device));
  if (!c->have_stages) {
    const long long n0 = launch_counter;
    for (int i = 0; i < 5; ++i) {
      int st = capture_stage(c, i, &c->stage_exec[i]);
      if (st != LLR_OK) {
        for (int j = 0; j < i; ++j) cudaGraphExecDestroy(c->stage_exec[j]);
        return st;
      }
    }
    c->have_stages = true;
    c->launches_per_iter = (int)(launch_counter - n0);
  }
  std::vector<cudaEvent_t> ev((size_t)n * 6, nullptr);
  int st = LLR_OK;
  for (size_t i = 0; i < ev.size() && st == LLR_OK; ++i) {
    cudaError_t e = cudaEventCreate(&ev[i]);
    if (e != cudaSuccess) st = cuda_error(e, "cudaEventCreate", __FILE__, __LINE__);
  }
  for (int it = 0; it < n && st == LLR_OK; ++it) {
    for (int k = 0; k < 5 && st == LLR_OK; ++k) {
      cudaError_t e = cudaEventRecord(ev[(size_t)it * 6 + k], c->stream);
      if (e == cudaSuccess) e = cudaGraphLaunch(c->stage_exec[k], c->stream);
      if (e != cudaSuccess) st = cuda_error(e, "stage launch", __FILE__, __LINE__);
    }
    if (st == LLR_OK) {
      cudaError_t e = cudaEventRecord(ev[(size_t)it * 6 + 5], c->stream);
      if (e != cudaSuccess) st = cuda_error(e, "cudaEventRecord", __FILE__, __LINE__);
    }
  }
  if (st == LLR_OK) {
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) st = cuda_error(e, "cudaStreamSynchronize", __FILE__, __LINE__);
  }
  if (st == LLR_OK) st = llr::check_device_error(c);
  if (st == LLR_OK) {
    double acc[5] = {0, 0, 0, 0, 0};
    for (int it = 0; it < n; ++it)
      for (int k = 0; k < 5; ++k) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ev[(size_t)it * 6 + k], ev[(size_t)it * 6 + k + 1]);
        acc[k] += ms;
      }
    float tot = 0.f;
    cudaEventElapsedTime(&tot, ev[0], ev[(size_t)(n - 1) * 6 + 5]);
    if (stage_ms)
      for (int k = 0; k < 5; ++k) stage_ms[k] = acc[k];
    if (total_ms) *total_ms = tot;
    c->h_iter += n;
  }
  for (auto e : ev)
    if (e) cudaEventDestroy(e);
  return st;
}

int llr_iterate_timed(llr_ctx* c, int32_t n, double* total_ms) {
  if (!c) return set_error(LLR_ERR_INVALID, "null context");
  LLR_CUDA_TRY(cudaSetDevice(c->device));
  cudaEvent_t a, b;
  LLR_CUDA_TRY(cudaEventCreate(&a));
  LLR_CUDA_TRY(cudaEventCreate(&b));
  int st = LLR_OK;
  cudaError_t e = cudaEventRecord(a, c->stream);
  if (e != cudaSuccess) st = cuda_error(e, "cudaEventRecord", __FILE__, __LINE__);
  if (st == LLR_OK) st = llr_iterate_async(c, n);
  if (st == LLR_OK) {
    e = cudaEventRecord(b, c->stream);
    if (e == cudaSuccess) e = cudaEventSynchronize(b);
    if (e != cudaSuccess) st = cuda_error(e, "cudaEventSynchronize", __FILE__, __LINE__);
  }
  if (st == LLR_OK) st = llr::check_device_error(c);
  if (st == LLR_OK) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    if (total_ms) *total_ms = ms;
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return st;
}

int llr_iterate_async(llr_ctx* c, int32_t n) {
  if (!c) return set_error(LLR_ERR_INVALID, "null context");
  if (n < 0) return set_error(LLR_ERR_INVALID, "negative iteration count");
  if (!c->have_kspace || !c->have_image) return set_error(LLR_ERR_STATE, "upload k-space and initialise the image");
  if (c->cfg.subspace_rank > 0 && !c->d_S) return set_error(LLR_ERR_STATE, "subspace not uploaded");
  LLR_CUDA_TRY(cudaSetDevice(c->device));
  if (!c->have_graph) LLR_TRY(build_graph(c));
  for (int i = 0; i < n; ++i) LLR_CUDA_TRY(cudaGraphLaunch(c->graph_exec, c->stream));
  c->h_iter += n;
  return LLR_OK;
}

int llr_iterate(llr_ctx* c, int32_t n, double* hist) {
  const long long it0 = c ? c->h_iter : 0;
  LLR_TRY(llr_iterate_async(c, n));
  if (hist && n > 0) {
    const long long lo = std::max<long long>(0, it0), hi = std::min<long long>(c->hist_cap, it0 + n);
    for (long long i = 0; i < n; ++i) hist[i] = NAN;
    if (hi > lo)
      LLR_CUDA_TRY(cudaMemcpyAsync(hist + (lo - it0), c->d_hist + lo, sizeof(double) * (hi - lo),
                                   cudaMemcpyDeviceToHost, c->stream));
  }
  LLR_CUDA_TRY(cudaStreamSynchronize(c->stream));
  LLR_TRY(llr::check_device_error(c));
  if (hist && n > 0) {
    const long long lo = std::max<long long>(0, it0), hi = std::min<long long>(c->hist_cap, it0 + n);
    for (long long i = lo; i < hi; ++i)
      if (!std::isfinite(hist[i - it0]))
        return set_error(LLR_ERR_NOT_FINITE, "non-finite data-consistency residual at iteration %lld", i);
  }
  return LLR_OK;
}

int llr_ctx_snapshot(llr_ctx* c, llr_cf32* d_dst) {
  if (!c || !d_dst) return set_error(LLR_ERR_INVALID, "null pointer");
  if (!c->have_image) return set_error(LLR_ERR_STATE, "no image");
  LLR_CUDA_TRY(cudaSetDevice(c->device));
  LLR_CUDA_TRY(cudaMemcpyAsync(d_dst, c->d_x, sizeof(float2) * (size_t)c->g.V * c->g.nq, cudaMemcpyDeviceToDevice,
                               c->stream));
  LLR_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return LLR_OK;
}

int llr_ctx_nrmse(llr_ctx* c, const llr_cf32* d_ref, double* out) {
  if (!c || !d_ref || !out) return set_error(LLR_ERR_INVALID, "null pointer");
  if (!c->have_image) return set_error(LLR_ERR_STATE, "no image");
  LLR_CUDA_TRY(cudaSetDevice(c->device));
  constexpr int nb = 512;
  LLR_TRY(launch_diff_norm(c->d_x, (const float2*)d_ref, c->g.V * c->g.nq, c->d_partials, c->d_partials + nb, nb,
                           c->stream));
  std::vector<double> h(2 * nb);
  LLR_CUDA_TRY(cudaMemcpyAsync(h.data(), c->d_partials, sizeof(double) * 2 * nb, cudaMemcpyDeviceToHost, c->stream));
  LLR_CUDA_TRY(cudaStreamSynchronize(c->stream));
  double d = 0.0, r = 0.0;
  for (int i = 0; i < nb; ++i) { d += h[i]; r += h[nb + i]; }
  *out = r > 0.0 ? std::sqrt(d / r) : INFINITY;
  return LLR_OK;
}

int llr_ctx_kernel_launches(const llr_ctx* c, int32_t* per_iteration) {
  if (!c || !per_iteration) return set_error(LLR_ERR_INVALID, "null pointer");
  if (!c->have_graph && !c->have_stages) return set_error(LLR_ERR_STATE, "no iteration has been captured yet");
  *per_iteration = c->launches_per_iter;
  return LLR_OK;
}

int llr_ctx_fallback_blocks(llr_ctx* c, int64_t* count) {
  if (!c || !count) return set_error(LLR_ERR_INVALID, "null pointer");
  LLR_CUDA_TRY(cudaSetDevice(c->device));
  LLR_CUDA_TRY(cudaStreamSynchronize(c->stream));
  int h = 0;
  if (c->cfg.subspace_rank == 0 && c->cfg.eig_solver != 1)
    LLR_CUDA_TRY(cudaMemcpy(&h, c->d_fb + std::max<long long>(1, c->nblocks), sizeof(int), cudaMemcpyDeviceToHost));
  *count = h;
  return LLR_OK;
}

int llr_get_iteration(const llr_ctx* c, int64_t* it) {
  if (!c || !it) return set_error(LLR_ERR_INVALID, "null pointer");
  *it = c->h_iter;
  return LLR_OK;
}

int llr_set_iteration(llr_ctx* c, int64_t it) {
  if (!c || it < 0) return set_error(LLR_ERR_INVALID, "bad arguments");
  LLR_CUDA_TRY(cudaSetDevice(c->device));
  long long v = it;
  LLR_CUDA_TRY(cudaMemcpyAsync(c->d_iter, &v, sizeof(long long), cudaMemcpyHostToDevice, c->stream));
  LLR_CUDA_TRY(cudaStreamSynchronize(c->stream));
  c->h_iter = it;
  return LLR_OK;
}

int llr_get_residual_history(llr_ctx* c, double* out, int32_t count) {
  if (!c || !out || count < 0) return set_error(LLR_ERR_INVALID, "bad arguments");
  LLR_CUDA_TRY(cudaSetDevice(c->device));
  const long long hi = std::min<long long>(c->h_iter, c->hist_cap);
  const long long lo = std::max<long long>(0, hi - count);
  for (int i = 0; i < count; ++i) out[i] = NAN;
  const long long nn = hi - lo;
  if (nn > 0)
    LLR_CUDA_TRY(cudaMemcpyAsync(out + (count - nn), c->d_hist + lo, sizeof(double) * nn, cudaMemcpyDeviceToHost,
                                 c->stream));
  LLR_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return LLR_OK;
}

int llr_get_objective_history(llr_ctx* c, double* out, int32_t count) {
  if (!c || !out || count < 0) return set_error(LLR_ERR_INVALID, "bad arguments");
  LLR_CUDA_TRY(cudaSetDevice(c->device));
  const long long hi = std::min<long long>(c->h_iter, c->hist_cap);
  const long long lo = std::max<long long>(0, hi - count);
  for (int i = 0; i < count; ++i) out[i] = NAN;
  const long long nn = hi - lo;
  if (nn > 0 && c->obj_mode != 0)
    LLR_CUDA_TRY(cudaMemcpyAsync(out + (count - nn), c->d_obj + lo, sizeof(double) * nn, cudaMemcpyDeviceToHost,
                                 c->stream));
  LLR_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return LLR_OK;
}

int llr_measurement_stats(llr_ctx* c, double* energy, double* us) {
  if (!c) return set_error(LLR_ERR_INVALID, "null context");
  if (!c->have_kspace) return set_error(LLR_ERR_STATE, "upload k-space first");
  if (energy) *energy = c->total_energy;
  if (us) *us = c->undersampling;
  return LLR_OK;
}

int llr_sigma_max(llr_ctx* c, const int32_t* shift, double* out) {
  if (!c || !out) return set_error(LLR_ERR_INVALID, "null pointer");
  if (!c->have_image) return set_error(LLR_ERR_STATE, "no image");
  LLR_CUDA_TRY(cudaSetDevice(c->device));
  const int zero[3] = {0, 0, 0};
  const int* sh = shift ? shift : zero;
  LLR_TRY(prox_pass(c, c->stream, sh, true, c->d_block_stat));
  std::vector<float> h((size_t)std::max<long long>(1, c->nblocks));
  LLR_CUDA_TRY(cudaMemcpyAsync(h.data(), c->d_block_stat, sizeof(float) * c->nblocks, cudaMemcpyDeviceToHost,
                               c->stream));
  LLR_CUDA_TRY(cudaStreamSynchronize(c->stream));
  double mx = 0;
  for (long long i = 0; i < c->nblocks; ++i) mx = std::max(mx, (double)h[i]);
  *out = std::sqrt(mx);
  return LLR_OK;
}

int llr_set_lambda(llr_ctx* c, float lam) {
  if (!c || !(lam >= 0.f)) return set_error(LLR_ERR_INVALID, "bad lambda");
  c->cfg.lambda = lam;
  drop_graph(c);
  return LLR_OK;
}

int llr_ctx_prox_llr(llr_ctx* c, const int32_t* shift) {
  if (!c || !shift) return set_error(LLR_ERR_INVALID, "null pointer");
  if (!c->have_image) return set_error(LLR_ERR_STATE, "no image");
  LLR_CUDA_TRY(cudaSetDevice(c->device));
  LLR_TRY(prox_pass(c, c->stream, shift, true, nullptr));
  LLR_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return LLR_OK;
}

int llr_ctx_wavelet(llr_ctx* c) {
  if (!c) return set_error(LLR_ERR_INVALID, "null context");
  if (!c->have_image) return set_error(LLR_ERR_STATE, "no image");
  if (!c->wavelet_on) return set_error(LLR_ERR_STATE, "wavelet disabled (alpha == 0 or no level fits)");
  LLR_CUDA_TRY(cudaSetDevice(c->device));
  // raw -> image over every voxel, then shrink and store back in the raw convention.
  const int cover[3] = {0, 0, 0};
  const int maxs[3] = {1, 1, 1};
  const int zero[3] = {0, 0, 0};
  PhaseTab ph = ctx_phase(c, c->d_ph_ksp, !c->hybrid);
  LLR_TRY(launch_scale_uncovered(c->d_x, c->g, cover, nullptr, 0, zero, maxs, c->load_scale, ph, 1, c->stream));
  LLR_TRY(wavelet_pass(c, c->stream, 1.f / c->load_scale));
  LLR_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return LLR_OK;
}

int llr_ctx_data_consistency(llr_ctx* c, double* resid) {
  if (!c) return set_error(LLR_ERR_INVALID, "null context");
  if (!c->have_image || !c->have_kspace) return set_error(LLR_ERR_STATE, "no image / k-space");
  LLR_CUDA_TRY(cudaSetDevice(c->device));
  cudaStream_t s = c->stream;
  // raw -> FFT input e^{+i theta} x = raw / N_t
  LLR_TRY(launch_scale(c->d_x, c->g.V * c->g.nq, c->load_scale, s));
  LLR_TRY(exec_fft(c, c->d_x, CUFFT_FORWARD, s));
  LLR_TRY(dc_pass(c, s, 0));
  double* d_out = c->d_partials + c->n_partials - 1;
  LLR_TRY(launch_finalize(c->d_partials, n_partials(c), (double)c->load_scale, nullptr, 0, nullptr, 0, d_out, s));
  LLR_TRY(exec_fft(c, c->d_x, CUFFT_INVERSE, s));
  double h = 0;
  LLR_CUDA_TRY(cudaMemcpyAsync(&h, d_out, sizeof(double), cudaMemcpyDeviceToHost, s));
  LLR_CUDA_TRY(cudaStreamSynchronize(s));
  if (resid) *resid = h;
  return LLR_OK;
}

int llr_ctx_device_bytes(const llr_ctx* c, size_t* bytes) {
  if (!c || !bytes) return set_error(LLR_ERR_INVALID, "null pointer");
  const size_t E = (size_t)c->g.V * c->g.nq;
  size_t b = 2 * E * sizeof(float2);
  b += c->hybrid ? (size_t)c->n_samp_lines * c->g.nx * sizeof(float2) : (c->have_kspace ? E * sizeof(float2) : 0);
  b += c->fft_work_bytes + c->wavelet_work_elems * sizeof(float2);
  if (c->d_gram) b += (size_t)std::max<long long>(1, c->nblocks) * (size_t)prox_gram_stride(c->g.nq) * sizeof(float2);
  if (c->d_vwide) b += (size_t)c->vwide_ctas * (size_t)wide_v_stride() * sizeof(float2);
  *bytes = b;
  return LLR_OK;
}

}  // extern "C"
