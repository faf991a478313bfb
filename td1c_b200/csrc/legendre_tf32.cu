// legendre_tf32.cu -- the mean field's theta <-> l transforms in split TF32 on
// the fifth-generation tensor cores (tcgen05.mma kind::tf32, accumulator in
// tensor memory).
//
// Same contract as legendre_gemm.cu: C[b](M x N) = T[b](M x K) * B[b](K x N)
// with a real Legendre table T and a complex slab B viewed as K rows of N
// reals (pair mode: B = conj(B0) * B1 formed in the loader).  The mixed
// precision form of the pair-density multipoles (ang2sph2, bas_ang2sph2.F90:
// 330-482) and of the pair potentials on the grid (sph2ang2,
// bas_sph2ang2.F90:334-463):
//   every FP64 operand x is split into x_hi = tf32(x) and x_lo = tf32(x - x_hi),
//   and T * B = T_hi B_hi + T_hi B_lo + T_lo B_hi (the lo * lo term dropped),
// three MMAs accumulated in FP32 in tensor memory: about 2^-21 relative per
// product, FP32-class results from TF32 tensor-core throughput.  C is written
// back in FP64, so everything downstream stays FP64.
//
// One CTA of 4 warps per 128 x 128 tile of C; K in chunks of 32.  Per chunk
// the 128 threads convert and stage the table and slab tiles (hi and lo
// planes) in shared memory in the canonical K-major layout without swizzle
// (8 rows x 16 bytes per core matrix; the two core matrices of one 8-deep MMA
// step 128 bytes apart, 8-row groups 1024 bytes apart), one thread issues the
// 4 x 3 MMAs of 128 x 128 x 8 and commits them to an mbarrier, and all threads
// wait on it (bounded) before the next chunk overwrites the tiles.  The
// epilogue reads the accumulator rows (TMEM lane = row) with tcgen05.ld and
// stores FP64.  The tensor-memory columns are allocated by warp 0 and always
// freed; a wait that runs out sets ST_TIMEOUT in the status word and the tile
// is abandoned.
#include "common.cuh"
#include "kernels.cuh"

namespace td1c {

constexpr int LT_BM = 128, LT_BN = 128, LT_BK = 32;
constexpr int LT_TILE = LT_BM * LT_BK * 4;  // bytes of one staged plane (128 rows x 32 tf32)
static_assert(LT_BN == LT_BM, "A and B planes share one size");
constexpr int LT_SMEM = 4 * LT_TILE + 64;  // A hi, A lo, B hi, B lo; then the mbarrier and the TMEM address
constexpr uint32_t LT_TMEM_COLS = 128;     // FP32 accumulator: 128 lanes x 128 columns
constexpr int LT_WAIT_LIMIT = 1 << 22;

// kind::tf32, D F32, A and B TF32 K-major, N = 128, M = 128 (bit layout of the
// tcgen05 instruction descriptor)
constexpr uint32_t LT_IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(LT_BN >> 3) << 17) |
                              ((uint32_t)(LT_BM >> 4) << 24);

// byte offset of element (row r, depth k) of a staged plane
__device__ __forceinline__ uint32_t lt_off(int r, int kg) {  // kg = k / 4: one 16-byte row of a core matrix
  return (uint32_t)((r >> 3) * 1024 + kg * 128 + (r & 7) * 16);
}
__device__ __forceinline__ uint32_t lt_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ void lt_split(double x, uint32_t& hi, uint32_t& lo) {
  hi = lt_tf32((float)x);
  lo = lt_tf32((float)(x - (double)__uint_as_float(hi)));
}
// shared-memory matrix descriptor: start address, LBO 128 B, SBO 1024 B, version 1, no swizzle
__device__ __forceinline__ uint64_t lt_desc(uint32_t saddr) {
  return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(1024 >> 4) << 32) |
         (1ull << 46);
}
__device__ __forceinline__ void lt_mma(uint32_t tmem, uint64_t da, uint64_t db, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
      "l"(da), "l"(db), "r"(LT_IDESC), "r"(accumulate));
}
__device__ __forceinline__ bool lt_wait(uint32_t bar, uint32_t parity) {
  for (int it = 0; it < LT_WAIT_LIMIT; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

template <bool PAIR>
__global__ void __launch_bounds__(128) legendre_tf32_kernel(const LegGemmBatch* __restrict__ batches, int M, int K, int N,
                                                            int* __restrict__ status) {
  extern __shared__ __align__(1024) unsigned char lt_smem[];
  const uint32_t s_base = (uint32_t)__cvta_generic_to_shared(lt_smem);
  const uint32_t sA = s_base, sB = s_base + 2 * LT_TILE;  // [hi | lo] planes each
  const uint32_t bar = s_base + 4 * LT_TILE;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(lt_smem + 4 * LT_TILE + 16);
  const LegGemmBatch bt = batches[blockIdx.z];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.y * LT_BM, n0 = blockIdx.x * LT_BN;

  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(1));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     (uint32_t)__cvta_generic_to_shared(tmem_slot)),
                 "r"(LT_TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  const int nchunk = (K + LT_BK - 1) / LT_BK;  // table rows are padded with zeros to nchunk * 32
  bool ok = true;
  uint32_t parity = 0;  // phase of the last commit
  for (int c = 0; c < nchunk && ok; ++c) {
    const int k0 = c * LT_BK;
    // table tile: thread = row, 32 depths (8 groups of 4)
    {
      const int gm = m0 + tid;
      const double* a = bt.A + (size_t)gm * bt.lda + k0;
#pragma unroll
      for (int kg = 0; kg < LT_BK / 4; ++kg) {
        uint32_t h[4], l[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const double x = gm < M ? __ldg(a + 4 * kg + j) : 0.0;
          lt_split(x, h[j], l[j]);
        }
        const uint32_t o = lt_off(tid, kg);
        asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(sA + o), "r"(h[0]), "r"(h[1]), "r"(h[2]), "r"(h[3]));
        asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(sA + LT_TILE + o), "r"(l[0]), "r"(l[1]), "r"(l[2]),
                     "r"(l[3]));
      }
    }
    // slab tile, transposed to K-major: thread = one complex column (two real columns) x 16 depths
    {
      const int cp = tid & 63, kh = (tid >> 6) * 16;
      const int gn = n0 + 2 * cp;
      uint32_t hr[16], lr[16], hi_[16], li[16];
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int gk = k0 + kh + j;
        double2 v = make_double2(0.0, 0.0);
        if (gk < K && gn < N) {
          if (!PAIR) {
            v = __ldg(reinterpret_cast<const double2*>(bt.B0 + (size_t)gk * bt.ldb + gn));
          } else {
            const size_t off = (size_t)gk * (bt.ldb >> 1) + (gn >> 1);
            const cplx z = cmulc(__ldg(reinterpret_cast<const cplx*>(bt.B0) + off), __ldg(reinterpret_cast<const cplx*>(bt.B1) + off));
            v = make_double2(z.x, z.y);
          }
        }
        lt_split(v.x, hr[j], lr[j]);
        lt_split(v.y, hi_[j], li[j]);
      }
#pragma unroll
      for (int g = 0; g < 4; ++g) {
        const int kg = (kh >> 2) + g;
        const uint32_t o0 = lt_off(2 * cp, kg), o1 = lt_off(2 * cp + 1, kg);
        asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(sB + o0), "r"(hr[4 * g]), "r"(hr[4 * g + 1]),
                     "r"(hr[4 * g + 2]), "r"(hr[4 * g + 3]));
        asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(sB + LT_TILE + o0), "r"(lr[4 * g]), "r"(lr[4 * g + 1]),
                     "r"(lr[4 * g + 2]), "r"(lr[4 * g + 3]));
        asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(sB + o1), "r"(hi_[4 * g]), "r"(hi_[4 * g + 1]),
                     "r"(hi_[4 * g + 2]), "r"(hi_[4 * g + 3]));
        asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(sB + LT_TILE + o1), "r"(li[4 * g]), "r"(li[4 * g + 1]),
                     "r"(li[4 * g + 2]), "r"(li[4 * g + 3]));
      }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // generic-proxy stores -> tensor-core reads
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
      for (int s = 0; s < LT_BK / 8; ++s) {  // 8-deep MMA steps: two 16-byte core matrices each
        const uint64_t ah = lt_desc(sA + 256 * s), al = lt_desc(sA + LT_TILE + 256 * s);
        const uint64_t bh = lt_desc(sB + 256 * s), bl = lt_desc(sB + LT_TILE + 256 * s);
        lt_mma(tmem, ah, bh, (c | s) != 0);
        lt_mma(tmem, ah, bl, 1u);
        lt_mma(tmem, al, bh, 1u);
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
    }
    parity = (uint32_t)(c & 1);
    const bool got = lt_wait(bar, parity);
    ok = !__syncthreads_or(!got);
  }
  if (!ok) {
    if (tid == 0 && status) atomicOr(status, ST_TIMEOUT);
    // the MMAs may still be running: one more bounded wait on the same phase before the columns are freed
    lt_wait(bar, parity);
  } else {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // epilogue: warp w holds rows 32 w .. 32 w + 31 (TMEM lanes), 8 columns per load
    const int gm = m0 + 32 * warp + lane;
    double* crow = bt.C + (size_t)gm * bt.ldc;
#pragma unroll 1
    for (int cc = 0; cc < LT_BN / 8; ++cc) {
      uint32_t r[8];
      const uint32_t taddr = tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(8 * cc);
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (gm < M) {
#pragma unroll
        for (int j = 0; j < 8; j += 2) {
          const int gn = n0 + 8 * cc + j;
          if (gn < N)
            *reinterpret_cast<double2*>(crow + gn) =
                make_double2((double)__uint_as_float(r[j]), (double)__uint_as_float(r[j + 1]));
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(LT_TMEM_COLS));
  }
}

template <bool PAIR>
static void lt_launch(const LegGemmBatch* d_batches, int nbatch, int M, int K, int N, int* status, cudaStream_t st) {
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(legendre_tf32_kernel<PAIR>, cudaFuncAttributeMaxDynamicSharedMemorySize, LT_SMEM);
    attr = true;
  }
  dim3 grid((N + LT_BN - 1) / LT_BN, (M + LT_BM - 1) / LT_BM, nbatch);
  legendre_tf32_kernel<PAIR><<<grid, 128, LT_SMEM, st>>>(d_batches, M, K, N, status);
}

int launch_legendre_gemm_tf32(const LegGemmBatch* d_batches, int nbatch, int M, int K, int N, bool pair, int* status,
                              cudaStream_t st) {
  if (nbatch <= 0) return 0;
  if (N % 2) return (int)cudaErrorInvalidValue;  // slabs are complex: 16-byte pairs
  if (pair) lt_launch<true>(d_batches, nbatch, M, K, N, status, st);
  else lt_launch<false>(d_batches, nbatch, M, K, N, status, st);
  return (int)cudaGetLastError();
}

}  // namespace td1c
