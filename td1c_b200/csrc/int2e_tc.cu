// int2e_tc.cu -- the MO two-electron integrals of the mixed-precision RHS (mode 3)
// in split TF32 on the fifth-generation tensor cores (hprod_mkint2_sph.F90:2-100).
//
// int2e(i,j,k,l) = sum_x rho2_ij[x] v2sph_kl[x] over x in [0, K), K =
// Nr (lmax2 + 1), for the active pairs.  With the P stored active pairs
// (P <= 64) the products of every row pair with every column pair are one
// dense real GEMM per slice of K:
//   D(128 x N) = A B^T,  A rows 0..63 = Re rho2_p, rows 64..127 = Im rho2_p,
//                        B rows 0..NB-1 = Re v2sph_q, NB..2NB-1 = Im v2sph_q,
// so that sum_x rho2_p v2sph_q = (D(p,q) - D(64+p,NB+q)) + i (D(p,NB+q) +
// D(64+p,q)) and the conjugated column of a pair stored as (l, k) takes
// v2sph^* (two signs flip).  The m-selection rule is applied when the entries
// are formed; the tensor cores compute every product, which costs nothing
// next to the operand traffic.
//
// Every FP64 operand x is split into x_hi + x_lo (TF32) and A B^T =
// A_hi B_hi + A_hi B_lo + A_lo B_hi, three tcgen05.mma kind::tf32 per depth
// step of 8, accumulating FP32 in tensor memory.  To keep the FP32 sums short
// the K range is cut into 3 slices per CTA (about 260 depths each for Ne);
// after each slice the accumulator is read with tcgen05.ld and added into
// FP64 registers (two warps per TMEM lane quarter, each holding half of the
// columns), and the next slice starts a fresh accumulator.  Each CTA writes
// the partial sums of the plan's entries in FP64; int2e_sum_kernel adds the
// CTAs' partials in a fixed order, as for the FP64 kernels.
//
// Staging: all 256 threads copy the raw FP64 rows of a chunk of 16 complex
// depths with cp.async into a ring of raw slots (several chunks ahead), split
// the chunk into the hi/lo TF32 planes of one of two operand stages (canonical
// K-major layout), and one thread issues the chunk's MMAs and commits them to
// the stage's mbarrier; the stage is written again only after those MMAs have
// read it.  Every wait is bounded (1 s); a wait that runs out sets ST_TIMEOUT,
// and the decision to leave the loop is made by all threads together
// (__syncthreads_or), so no thread waits at a barrier the others left.  Before
// the tensor memory is freed every committed MMA has completed (the drain
// wait) and no cp.async is in flight.
#include "common.cuh"
#include "kernels.cuh"
#include "reductions.cuh"
#include "tc.cuh"

namespace td1c {

constexpr int I2T_KC = 16;          // complex depths per chunk
constexpr int I2T_NT = 256;         // threads
constexpr int I2T_SPC = 3;          // K slices per CTA
constexpr int I2T_RR = 3;           // raw slots (chunks in flight: I2T_RR - 1)
constexpr int I2T_PLANE_A = 128 * I2T_KC * 4;  // one A plane (hi or lo): 128 rows x 16 TF32 (8 KB)

size_t int2e_tc_smem(const I2tArgs& a) {
  const size_t raw = (size_t)2 * a.P * I2T_KC * sizeof(cplx);
  const size_t stage = 2 * (size_t)I2T_PLANE_A + 2 * (size_t)(2 * a.NB) * I2T_KC * 4;
  return (size_t)I2T_RR * raw + 2 * stage + 64;
}

__global__ void __launch_bounds__(I2T_NT, 1) int2e_tc_kernel(I2tArgs a) {
  extern __shared__ __align__(1024) unsigned char i2t_smem[];
  __shared__ unsigned long long opfree[2], done, drain;
  __shared__ uint32_t tmem_base;
  const int P = a.P, NB = a.NB, N = 2 * NB, RR = I2T_RR;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const size_t raw_bytes = (size_t)2 * P * I2T_KC * sizeof(cplx);
  const int plane_b = N * I2T_KC * 4;
  const int stage_bytes = 2 * I2T_PLANE_A + 2 * plane_b;
  unsigned char* s_stage = i2t_smem;                                  // 2 stages: A hi, A lo, B hi, B lo
  unsigned char* s_raw = i2t_smem + 2 * (size_t)stage_bytes;          // RR raw slots [2P rows][KC] complex
  const size_t K = a.K;
  const int nslice = gridDim.x * I2T_SPC;
  const size_t kper = ((K + nslice - 1) / nslice + I2T_KC - 1) / I2T_KC * I2T_KC;
  const int nch = (int)(kper / I2T_KC);  // chunks of a slice
  // chunk j of this CTA: slice j / nch, chunk j % nch (chunks past K read zeros)
  auto chunk_k0 = [&](int j) -> size_t { return (size_t)(blockIdx.x * I2T_SPC + j / nch) * kper + (size_t)(j % nch) * I2T_KC; };
  int my_slices = 0;  // the CTA's slices that start inside K (slices past K are left out)
  for (int q = 0; q < I2T_SPC; ++q)
    if ((size_t)(blockIdx.x * I2T_SPC + q) * kper < K) my_slices = q + 1;
  const int total = my_slices * nch;

  if (tid == 0) {
    mbar_init(&opfree[0], 1); mbar_init(&opfree[1], 1); mbar_init(&done, 1); mbar_init(&drain, 1);
    fence_mbar_init();
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(&tmem_base)), "r"(128u));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  // operand rows that hold no pair stay zero in both stages
  for (int e = tid; e < 2 * stage_bytes / 16; e += I2T_NT) reinterpret_cast<uint4*>(s_stage)[e] = make_uint4(0, 0, 0, 0);

  auto load = [&](int j) {
    if (j >= total) return;
    const size_t k0 = chunk_k0(j);
    unsigned char* dst = s_raw + (size_t)(j % RR) * raw_bytes;
    for (int e = tid; e < 2 * P * I2T_KC; e += I2T_NT) {
      const int row = e / I2T_KC, kk = e % I2T_KC;
      const int p = row < P ? row : row - P;
      const cplx* src = (row < P ? a.rho2 : a.v2sph) + (size_t)a.pair[p] * K;
      const bool in = k0 + kk < K;
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(su32(dst + (size_t)e * sizeof(cplx))),
                   "l"(src + (in ? k0 + kk : 0)), "r"(in ? 16u : 0u)
                   : "memory");
    }
  };
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base;
  fence_async_smem();  // the zeroed stages are seen by the tensor cores

  for (int s = 0; s < RR - 1; ++s) {
    load(s);
    asm volatile("cp.async.commit_group;" ::: "memory");
  }
  // FP64 sums of this thread's TMEM lane (32 (warp % 4) + lane) over half of the columns
  const int half = warp >> 2, nh = NB;  // N / 2 columns per half
  double acc[64];
#pragma unroll
  for (int q = 0; q < 64; ++q) acc[q] = 0.0;
  const uint32_t idesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
  const uint32_t sbo = (uint32_t)(I2T_KC * 32);
  bool failed = false;
  int nslice_done = 0;
  for (int j = 0; j < total; ++j) {
    const int s = j & 1;
    asm volatile("cp.async.wait_group %0;" ::"n"(I2T_RR - 2) : "memory");
    __syncthreads();  // raw chunk j has landed for every thread; chunk j - 1 is converted
    load(j + RR - 1);
    asm volatile("cp.async.commit_group;" ::: "memory");
    // stage s is free once the MMAs of chunk j - 2 have read it
    bool ok = j < 2 || mbar_wait(&opfree[s], ((j - 2) >> 1) & 1);
    if (__syncthreads_or(!ok)) { failed = true; break; }
    const unsigned char* raw = s_raw + (size_t)(j % RR) * raw_bytes;
    const uint32_t st = su32(s_stage + (size_t)s * stage_bytes);
    for (int e = tid; e < 2 * P * (I2T_KC / 4); e += I2T_NT) {
      const int row = e / (I2T_KC / 4), g = e % (I2T_KC / 4);
      const cplx* z = reinterpret_cast<const cplx*>(raw) + (size_t)row * I2T_KC + 4 * g;
      uint32_t rh[4], rl[4], ih[4], il[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const cplx v = z[u];
        tc_split(v.x, rh[u], rl[u]);
        tc_split(v.y, ih[u], il[u]);
      }
      // A (rho2): rows p and 64 + p; B (v2sph): rows q and NB + q
      const bool isa = row < P;
      const int p = isa ? row : row - P;
      const uint32_t hi_base = st + (isa ? 0u : 2u * I2T_PLANE_A);
      const uint32_t plane = isa ? (uint32_t)I2T_PLANE_A : (uint32_t)plane_b;
      const int r_re = p, r_im = isa ? 64 + p : NB + p;
      const uint32_t o_re = tc_off(r_re, 4 * g, I2T_KC), o_im = tc_off(r_im, 4 * g, I2T_KC);
      asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(hi_base + o_re), "r"(rh[0]), "r"(rh[1]), "r"(rh[2]), "r"(rh[3]));
      asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(hi_base + plane + o_re), "r"(rl[0]), "r"(rl[1]), "r"(rl[2]),
                   "r"(rl[3]));
      asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(hi_base + o_im), "r"(ih[0]), "r"(ih[1]), "r"(ih[2]), "r"(ih[3]));
      asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(hi_base + plane + o_im), "r"(il[0]), "r"(il[1]), "r"(il[2]),
                   "r"(il[3]));
    }
    fence_async_smem();  // generic-proxy stores -> tensor-core reads
    __syncthreads();
    const int c = j % nch;
    const bool slice_end = c == nch - 1;
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t ah = st, al = st + I2T_PLANE_A, bh = st + 2 * I2T_PLANE_A, bl = bh + plane_b;
#pragma unroll
      for (int ks = 0; ks < I2T_KC / 8; ++ks) {
        const uint32_t ko = (uint32_t)(ks * 256);
        const uint64_t dah = tc_desc(ah + ko, sbo), dal = tc_desc(al + ko, sbo);
        const uint64_t dbh = tc_desc(bh + ko, sbo), dbl = tc_desc(bl + ko, sbo);
        tc_mma(tmem, dah, dbh, idesc, (c | ks) != 0);
        tc_mma(tmem, dah, dbl, idesc, 1u);
        tc_mma(tmem, dal, dbh, idesc, 1u);
      }
      tc_commit(&opfree[s]);
      if (slice_end) tc_commit(&done);
    }
    if (slice_end) {
      // the slice's accumulator, added into FP64 registers
      const bool ok2 = mbar_wait(&done, nslice_done & 1);
      ++nslice_done;
      if (__syncthreads_or(!ok2)) { failed = true; break; }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
      for (int g = 0; g < 4; ++g) {
        if (16 * g < nh) {
          uint32_t r[16];
          const uint32_t taddr = tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(half * nh + 16 * g);
          asm volatile(
              "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
              "[%16];"
              : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
                "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
              : "r"(taddr));
          asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
          for (int q = 0; q < 16; ++q) acc[16 * g + q] += (double)__uint_as_float(r[q]);
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    }
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  // nothing may still write tensor memory when it is freed: every committed MMA has completed
  if (tid == 0 && total > 0) {
    tc_commit(&drain);
    if (!mbar_wait(&drain, 0)) atomicOr(a.status, ST_TIMEOUT);
  }
  if (failed && tid == 0) atomicOr(a.status, ST_TIMEOUT);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(128u));
  }
  if (failed) return;
  // the CTA's FP64 sums D(row, col) in shared memory (the ring is free), then its partial entries
  double* F = reinterpret_cast<double*>(i2t_smem);  // [128][N + 1]
  const int row = 32 * (warp & 3) + lane;
#pragma unroll
  for (int q = 0; q < 64; ++q)
    if (q < nh) F[(size_t)row * (N + 1) + half * nh + q] = acc[q];
  __syncthreads();
  cplx* out = a.partial + (size_t)blockIdx.x * a.nent;
  for (int e = tid; e < a.nent; e += I2T_NT) {
    const int4 en = a.ent[e];  // (row pair, column pair, conjugated column, -)
    const double rr = F[(size_t)en.x * (N + 1) + en.y], ri = F[(size_t)en.x * (N + 1) + NB + en.y];
    const double ir = F[(size_t)(64 + en.x) * (N + 1) + en.y], ii = F[(size_t)(64 + en.x) * (N + 1) + NB + en.y];
    out[e] = en.z ? mkc(rr + ii, ir - ri) : mkc(rr - ii, ri + ir);
  }
}

bool int2e_tc_fits(const I2tArgs& a) {
  return a.P >= 1 && a.P <= 64 && a.NB >= a.P && a.NB % 16 == 0 && 2 * a.NB <= 128 &&
         int2e_tc_smem(a) <= 224 * 1024 && (size_t)128 * (2 * a.NB + 1) * 8 <= int2e_tc_smem(a);
}

int launch_int2e_tc(const I2tArgs& t, const Int2eArgs& sum, int nsplit, cudaStream_t st) {
  const int n = sum.nact, n4 = n * n * n * n;
  if (n4 == 0) return 0;
  if (!int2e_tc_fits(t) || nsplit < 1) return (int)cudaErrorInvalidValue;
  cudaError_t e = cudaMemsetAsync(sum.int2e, 0, sizeof(cplx) * n4, st);
  if (e != cudaSuccess) return (int)e;
  // the dynamic shared memory this plan needs (the kernel's static barriers come on top)
  const size_t smem = int2e_tc_smem(t);
  static size_t attr[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64 || attr[dev] < smem) {
    e = cudaFuncSetAttribute(int2e_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return (int)e;
    if (dev >= 0 && dev < 64) attr[dev] = smem;
  }
  int2e_tc_kernel<<<nsplit, I2T_NT, smem, st>>>(t);
  e = cudaGetLastError();
  if (e != cudaSuccess) return (int)e;
  return launch_int2e_sum_fill(sum, nsplit, st);
}

}  // namespace td1c
