// tc.cuh -- split-TF32 operands and tcgen05 MMA helpers shared by the
// fifth-generation tensor-core kernels (legendre_tc.cu, int2e_tc.cu).
//
// Operand planes are canonical K-major with no swizzle: 8-row x 16-byte core
// matrices, K-adjacent ones 128 bytes apart (LBO), 8-row groups kp * 32 bytes
// apart (SBO) for a plane of depth kp TF32 values.  An FP64 value x is split
// into x_hi = tf32(x) and x_lo = tf32(x - x_hi).
#pragma once
#include <cstdint>

#include "common.cuh"
#include "tma.cuh"

namespace td1c {

// byte offset of (row r, depth k) in a canonical K-major plane of depth kp
// (8 x 16-byte core matrices: K-adjacent ones 128 bytes apart, 8-row groups
// kp * 32 bytes apart)
__host__ __device__ __forceinline__ uint32_t tc_off(int r, int k, int kp) {
  return (uint32_t)((r >> 3) * (kp * 32) + (k >> 2) * 128 + (r & 7) * 16 + (k & 3) * 4);
}
__device__ __forceinline__ uint32_t tc_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ void tc_split(double x, uint32_t& hi, uint32_t& lo) {
  hi = tc_tf32((float)x);
  lo = tc_tf32((float)(x - (double)__uint_as_float(hi)));
}
// shared-memory matrix descriptor (sm100): start, LBO, SBO, version 1, no swizzle
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr, uint32_t sbo) {
  return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(sbo >> 4) << 32) | (1ull << 46);
}
__device__ __forceinline__ void tc_mma(uint32_t tmem, uint64_t da, uint64_t db, uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
      "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
}
__device__ __forceinline__ void tc_commit(unsigned long long* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(su32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned long long* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(su32(bar)) : "memory");
}

}  // namespace td1c
