// tma.cuh -- thin wrappers over the sm_90+/sm_100a asynchronous copy engine
// (cp.async.bulk, cp.async.bulk.tensor) and mbarriers, shared by the
// kernels that stage their operands in shared memory.
//
// Every wait on an mbarrier is bounded in time (mbar_wait); callers turn a
// wait that runs out into ST_TIMEOUT instead of spinning forever.  No copy
// here uses cluster multicast.
#pragma once
#include <cuda.h>
#include <cudaTypedefs.h>

#include "common.cuh"

namespace td1c {

__device__ __forceinline__ unsigned su32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(su32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
constexpr unsigned long long TMA_WAIT_NS = 1000000000ull;  // bound of one mbarrier wait: 1 s
// wait for the phase of the given parity; false when TMA_WAIT_NS ran out
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = globaltimer_ns();
  while (globaltimer_ns() - t0 < TMA_WAIT_NS)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// 1-d bulk copy global -> shared (16-byte aligned addresses, size a multiple of 16)
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(su32(dst)),
               "l"(src), "r"(bytes), "r"(su32(bar))
               : "memory");
}
// tiled tensor copies; the x coordinate times the element size is a multiple of 16 bytes
__device__ __forceinline__ void tensor_load_2d(void* dst, const CUtensorMap* tm, int x, int y, unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          su32(dst)),
      "l"(tm), "r"(x), "r"(y), "r"(su32(bar))
      : "memory");
}
__device__ __forceinline__ void tensor_load_3d(void* dst, const CUtensorMap* tm, int x, int y, int z, unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
          su32(dst)),
      "l"(tm), "r"(x), "r"(y), "r"(z), "r"(su32(bar))
      : "memory");
}
__device__ __forceinline__ void tensor_load_4d(void* dst, const CUtensorMap* tm, int x, int y, int z, int w,
                                               unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(
          su32(dst)),
      "l"(tm), "r"(x), "r"(y), "r"(z), "r"(w), "r"(su32(bar))
      : "memory");
}
__device__ __forceinline__ void tensor_store_4d(const CUtensorMap* tm, int x, int y, int z, int w, const void* src) {
  asm volatile("cp.async.bulk.tensor.4d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3, %4}], [%5];" ::"l"(tm), "r"(x),
               "r"(y), "r"(z), "r"(w), "r"(su32(src))
               : "memory");
}
__device__ __forceinline__ void tensor_store_3d(const CUtensorMap* tm, int x, int y, int z, const void* src) {
  asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3}], [%4];" ::"l"(tm), "r"(x),
               "r"(y), "r"(z), "r"(su32(src))
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read_1() { asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_async_global() { asm volatile("fence.proxy.async.global;" ::: "memory"); }

// cuTensorMapEncodeTiled through the runtime's driver entry point (no -lcuda)
inline PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (!encode) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  }
  return encode;
}

// float64 tensor map of rank 2 to 4, no swizzle, out-of-bounds elements read as 0
inline int encode_f64_map(CUtensorMap* tm, const void* base, int rank, const cuuint64_t* dims, const cuuint64_t* strides_bytes,
                          const cuuint32_t* box, const char* what) {
  auto encode = tensor_map_encoder();
  if (!encode) {
    fprintf(stderr, "td1c_b200: cuTensorMapEncodeTiled is not available (%s)\n", what);
    return (int)cudaErrorNotSupported;
  }
  const cuuint32_t estr[4] = {1u, 1u, 1u, 1u};
  CUresult r = encode(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, (cuuint32_t)rank, const_cast<void*>(base), dims, strides_bytes, box,
                      estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    fprintf(stderr, "td1c_b200: cuTensorMapEncodeTiled (%s) failed: %d\n", what, (int)r);
    return (int)cudaErrorInvalidValue;
  }
  return 0;
}

}  // namespace td1c
