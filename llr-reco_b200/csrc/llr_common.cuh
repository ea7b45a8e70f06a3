// Shared device/host helpers for the B200 LLR reconstruction library.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

#include "../../include/llr_b200.h"

// ---------------------------------------------------------------------------------------
// error reporting (thread-local message, status codes)
// ---------------------------------------------------------------------------------------
namespace llr {

int set_error(int status, const char* fmt, ...);
int cuda_error(cudaError_t e, const char* what, const char* file, int line);

// Kernel launches issued by the calling thread. Every launch site of the library calls
// note_launch() just before its launch; the iteration graph builder reads the difference
// across its capture to know how many of the library's kernels one iteration runs.
inline thread_local long long launch_counter = 0;
inline void note_launch() { ++launch_counter; }

}  // namespace llr

#define LLR_CUDA_TRY(expr)                                                         \
  do {                                                                             \
    cudaError_t _e = (expr);                                                       \
    if (_e != cudaSuccess) return ::llr::cuda_error(_e, #expr, __FILE__, __LINE__); \
  } while (0)

#define LLR_TRY(expr)            \
  do {                           \
    int _s = (expr);             \
    if (_s != LLR_OK) return _s; \
  } while (0)

#define LLR_CHECK_ARG(cond, msg)                                   \
  do {                                                             \
    if (!(cond)) return ::llr::set_error(LLR_ERR_INVALID, "%s", msg); \
  } while (0)

// ---------------------------------------------------------------------------------------
// complex float2 arithmetic
// ---------------------------------------------------------------------------------------
__host__ __device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// conj(a) * b
__host__ __device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
  return make_float2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
// a * conj(b)
__host__ __device__ __forceinline__ float2 cmul_bc(float2 a, float2 b) {
  return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__host__ __device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
__host__ __device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
__host__ __device__ __forceinline__ float cabs2(float2 a) { return a.x * a.x + a.y * a.y; }

// acc += a * b
__device__ __forceinline__ void cfma(float2& acc, float2 a, float2 b) {
  acc.x = fmaf(a.x, b.x, acc.x);
  acc.x = fmaf(-a.y, b.y, acc.x);
  acc.y = fmaf(a.x, b.y, acc.y);
  acc.y = fmaf(a.y, b.x, acc.y);
}
// acc += conj(a) * b
__device__ __forceinline__ void cfma_ca(float2& acc, float2 a, float2 b) {
  acc.x = fmaf(a.x, b.x, acc.x);
  acc.x = fmaf(a.y, b.y, acc.x);
  acc.y = fmaf(a.x, b.y, acc.y);
  acc.y = fmaf(-a.y, b.x, acc.y);
}
// acc += a * conj(b)
__device__ __forceinline__ void cfma_cb(float2& acc, float2 a, float2 b) {
  acc.x = fmaf(a.x, b.x, acc.x);
  acc.x = fmaf(a.y, b.y, acc.x);
  acc.y = fmaf(a.y, b.x, acc.y);
  acc.y = fmaf(-a.x, b.y, acc.y);
}

// ---------------------------------------------------------------------------------------
// counter-based RNG: SplitMix64 finaliser keyed by (seed, stream, index).  Identical on
// host and device so that shifts drawn inside a CUDA graph match the host/oracle draw.
// ---------------------------------------------------------------------------------------
#define LLR_GOLDEN64 0x9E3779B97F4A7C15ull
#define LLR_SHIFT_STREAM 0x5348ull
#define LLR_MASK_STREAM 0x4D41ull

__host__ __device__ __forceinline__ uint64_t llr_splitmix64(uint64_t x) {
  uint64_t z = x + LLR_GOLDEN64;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__host__ __device__ __forceinline__ uint64_t llr_rng_u64(uint64_t seed, uint64_t stream, uint64_t index) {
  return llr_splitmix64(seed + LLR_GOLDEN64 * ((stream << 32) + index + 1ull));
}

__host__ __device__ __forceinline__ int llr_shift_draw(uint64_t seed, int64_t it, int axis, int maxv) {
  return (int)(llr_rng_u64(seed, LLR_SHIFT_STREAM, (uint64_t)(3 * it + axis)) % (uint64_t)maxv);
}

// ---------------------------------------------------------------------------------------
// geometry shared by kernels
// ---------------------------------------------------------------------------------------
struct Geom {
  int nx, ny, nz, nq;
  long long nyz;   // ny * nz
  long long V;     // nx * ny * nz
};

// Per-axis phase tables, one row per volume: t[q * n + i] = exp(+i theta_a(i)).
struct PhaseTab {
  const float2* x;  // nq * nx  (may be null: identity)
  const float2* y;  // nq * ny
  const float2* z;  // nq * nz
};

__device__ __forceinline__ float2 phase_at(const PhaseTab& t, const Geom& g, int q, int ix, int iy, int iz) {
  float2 p = make_float2(1.f, 0.f);
  if (t.y) p = t.y[(long long)q * g.ny + iy];
  if (t.z) p = cmul(p, t.z[(long long)q * g.nz + iz]);
  if (t.x) p = cmul(p, t.x[(long long)q * g.nx + ix]);
  return p;
}

// Planar (plane-major) internal layout: element (ix, iy, iz, q) at
// iy + ny * (iz + nz * (ix + nx * q)); every (x, q) plane of ny*nz samples is contiguous.
__device__ __forceinline__ long long planar_index(const Geom& g, int ix, int iy, int iz, int q) {
  return (long long)iy + (long long)g.ny * ((long long)iz + (long long)g.nz * ((long long)ix + (long long)g.nx * q));
}
