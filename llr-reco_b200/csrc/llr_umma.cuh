// Shared helpers for the kernels that drive the 5th-generation tensor cores (tcgen05):
// UMMA shared-memory and instruction descriptors (128-byte swizzled and unswizzled K-major), the
// TF32 and BF16 MMAs, commits to mbarriers, bounded mbarrier waits, the TF32 split and the
// 128-byte swizzled operand layout.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace llr {

constexpr unsigned long long kUmmaWaitLimit = 1ull << 22;   // bounded spin: ~seconds, never forever

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// K-major UMMA shared-memory descriptor (sm_100 version 1) with the 128-byte swizzle: rows of
// 128 B (32 TF32 along K), 8-row atoms of 1 KB (SBO = 1 KB), the 16-byte chunk index XORed with
// the row index inside the atom.  Stepping K by 8 TF32 moves the start address by 32 B.
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t saddr) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)1 << 16;                          // LBO: unused for swizzled K-major
  d |= (uint64_t)(1024u >> 4) << 32;               // SBO: next 8-row atom
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)2 << 61;                          // SWIZZLE_128B
  return d;
}

// K-major UMMA shared-memory descriptor without swizzle: core matrices of 8 rows x 16 B stored
// as 128 contiguous bytes (row stride 16 B); lbo = byte step between core matrices along K,
// sbo = byte step between 8-row groups along M / N.  The start address needs 16-byte alignment
// only, so an operand can begin at any 16-byte row of a larger array.
__device__ __forceinline__ uint64_t umma_desc_kmajor(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;                          // SWIZZLE_NONE (layout type 0)
  return d;
}

// Instruction descriptor: BF16 x BF16 -> F32, both operands K-major, M x N.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(uint32_t M, uint32_t N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((N >> 3) << 17) | ((M >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

// Instruction descriptor: TF32 x TF32 -> F32, both operands K-major, M x N.
__host__ __device__ constexpr uint32_t umma_idesc_tf32(uint32_t M, uint32_t N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((N >> 3) << 17) | ((M >> 4) << 24);
}

__device__ __forceinline__ void umma_tf32(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void umma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t mbar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, P1;\n\t}" : "=r"(ok) : "r"(mbar), "r"(parity) : "memory");
  return ok != 0;
}

// Bounded wait; returns false when the limit runs out.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
  for (unsigned long long i = 0; i < kUmmaWaitLimit; ++i)
    if (mbar_try(mbar, parity)) return true;
  return false;
}

// TF32 part of x rounded to nearest (ties away from zero) on the 10-bit mantissa: add half a
// TF32 unit to the magnitude bits and clear the 13 low bits.  Finite inputs only.
__device__ __forceinline__ uint32_t tf32_rna(float x) {
  return (__float_as_uint(x) + 0x1000u) & 0xFFFFE000u;
}

// Byte offset of element (mn, k) of one operand plane (k < 32) in the 128-byte swizzled layout.
__device__ __forceinline__ int op_offset(int mn, int k) {
  return (mn >> 3) * 1024 + (mn & 7) * 128 + ((((k >> 2) ^ mn) & 7) << 4) + ((k & 3) << 2);
}

}  // namespace llr
