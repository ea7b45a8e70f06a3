// Allocation-free variant of the batched hard-rank prox.
//
// llr_low_rank_batch_dev() allocates, with cudaMallocAsync on every call, a per-matrix packed
// Gram buffer and 2 * batch + 2 ints (fallback list and count, kept counts and a queue
// counter), and takes the split path: tensor-core Gram kernel, warp eigen kernel, apply
// kernel.  Some callers cannot let the library allocate: a host that records the call into a
// CUDA graph it owns and replays it under a fixed memory plan, a process whose device memory is
// handed out by another framework's pool, or a real-time loop that must not pay an allocator
// call per invocation.  For them this entry point runs the fused tridiagonal prox kernel, which
// needs no per-matrix scratch, and takes its one piece of scratch -- the list of matrices that
// keep more components than the fused kernel handles (more than 16), finished by the Jacobi
// kernel -- from a file-scope device array.  It calls no cudaMalloc, cudaFree or allocating
// library routine.  The two entry points compute the same operation with different kernels;
// their outputs agree to the low-rank prox tolerance (relative 5e-5 on well-separated spectra).
#include <cstring>
#include <mutex>

#include "llr_internal.h"

namespace llr {

namespace {

// Largest batch the static list can serve: one int per matrix plus the count.  256 KiB of
// device memory on every GPU that loads the library, held until the process exits.
constexpr int kNoAllocMaxBatch = 65536;

static __device__ __align__(256) int g_noalloc_fallback[kNoAllocMaxBatch + 1];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
int* g_noalloc_addr[kMaxDevices] = {nullptr};

// The array's name is only a host-side stand-in in host code; the device address must be
// queried once per device, with that device current.  The cached address belongs to the
// device's primary context: after cudaDeviceReset() on a device the module is loaded again and
// the cache entry for that device is stale, so this entry point must not be used on a device
// that was reset during the process's life.
int noalloc_scratch(int** out) {
  int dev = 0;
  LLR_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return set_error(LLR_ERR_UNSUPPORTED, "device ordinal %d >= %d", dev, kMaxDevices);
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_fallback);
    if (e != cudaSuccess) return cuda_error(e, "cudaGetSymbolAddress", __FILE__, __LINE__);
    g_noalloc_addr[dev] = static_cast<int*>(p);
  }
  *out = g_noalloc_addr[dev];
  return LLR_OK;
}

}  // namespace

}  // namespace llr

using namespace llr;

extern "C" int llr_low_rank_batch_dev_noalloc(int32_t m, int32_t n, int32_t rank, int32_t batch, llr_cf32* d_mats,
                                              void* stream) {
  if (!d_mats || m < 1 || n < 1 || batch < 0) return set_error(LLR_ERR_INVALID, "bad matrix batch arguments");
  if (rank < 1 || rank > n) return set_error(LLR_ERR_INVALID, "rank must be in [1, n] (lib.rs:205-207)");
  if (batch > kNoAllocMaxBatch)
    return set_error(LLR_ERR_INVALID,
                     "batch of %d matrices exceeds the %d that the allocation-free entry point's static list holds; "
                     "split the batch or use llr_low_rank_batch_dev",
                     batch, kNoAllocMaxBatch);
  if (batch == 0) return LLR_OK;
  int* list = nullptr;
  LLR_TRY(noalloc_scratch(&list));
  BlockSource src;
  memset(&src, 0, sizeof(src));
  src.kind = 0;
  src.data = (float2*)d_mats;
  src.nblocks = batch;
  ProxOp op;
  memset(&op, 0, sizeof(op));
  op.m = m;
  op.n = n;
  op.mode = LLR_PROX_HARD_RANK;
  op.rank = rank;
  op.lambda = 0.f;
  op.block_stat = nullptr;
  op.eig_solver = 0;
  op.fb_list = list;                 // the count word (cleared by launch_llr_prox) follows the list
  op.fb_count = list + kNoAllocMaxBatch;
  return launch_llr_prox(src, op, (cudaStream_t)stream);
}
