// legendre_gemm.cu -- batched FP64 "real table x complex slab" products.
//
// Every theta <-> l transform of the RHS has the form
//     C[b](M x 2Nr) = T[b](M x K) * B[b](K x 2Nr)
// with a real Legendre table T (selected by the batch's m) and a complex slab
// B viewed as K rows of 2*Nr reals (re, im interleaved, radial index fastest):
//   sph2ang1   orbg(r,th,i)   = sum_l  orb(r,l,i)    legf1(l,th,m_i)   bas_sph2ang1.F90:88-156
//   ang2sph2   rho2(r,l,j,i)  = sum_th rho(r,th,j,i) legb2(th,l,m_ji)  bas_ang2sph2.F90:330-482
//   sph2ang2   v2ang(r,th,j,i)= sum_l  v2sph(r,l,j,i) legf2(l,th,m_ji) bas_sph2ang2.F90:334-463
//   ang2sph1   gorb(r,l,i)    = sum_th gorbg(r,th,i) legb1(th,l,m_i)   bas_ang2sph1.F90:88-158
// For ang2sph2 the slab is the pair density conj(orbg_j) * orbg_i, formed in
// the tile loader so the (Nr x Ntheta x npair) pair field never touches HBM
// (hprod_mkrho2.F90:115-197 fused).
//
// FP64 tensor-core GEMM (mma.sync.m8n8k4.f64): 256 threads = 8 warps in a
// 2 (M) x 4 (N) grid, each warp MT m-tiles x 2 n-tiles of 8 x 8, CTA tile
// (16 MT) x 64 x 32.  The table chunk (stored [m][k]) and the slab chunk
// ([k][n]) go through registers into double-buffered shared memory with
// pitches of 4 mod 16 doubles, so every fragment load is conflict-free; the
// tables are padded copies whose rows are 16-byte aligned and whose depth is
// a multiple of 32 (zeros past K).  Rows of a table below |m| are zero,
// which reproduces the reference's l >= |m| loop bounds.
#include "common.cuh"
#include "kernels.cuh"

namespace td1c {

constexpr int LG_BN = 64, LG_BK = 32;
constexpr int LG_LDB = LG_BN + 4;  // pitch of a slab row in shared memory (doubles)
constexpr int LG_LDA = LG_BK + 4;  // pitch of a table row in shared memory (doubles)

__host__ __device__ constexpr size_t lg_smem_bytes(int mt) {
  return sizeof(double) * 2 * ((size_t)16 * mt * LG_LDA + (size_t)LG_BK * LG_LDB);
}

__device__ __forceinline__ void lg_dmma(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

template <int MT, bool PAIR>
__global__ void __launch_bounds__(256) legendre_gemm_kernel(const LegGemmBatch* __restrict__ batches, int M, int K, int N) {
  constexpr int BM = 16 * MT;
  constexpr int NA = BM * LG_BK / 2 / 256;  // double2 of the table chunk per thread
  constexpr int NB = LG_BK * LG_BN / 2 / 256;  // double2 of the slab chunk per thread (= complex elements)
  extern __shared__ __align__(16) double lg_smem[];
  double* As = lg_smem;                         // [2][BM][LDA]
  double* Bs = lg_smem + 2 * BM * LG_LDA;       // [2][BK][LDB]
  const LegGemmBatch bt = batches[blockIdx.z];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int gid = lane >> 2, tig = lane & 3;
  const int wm = warp >> 2, wn = warp & 3;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * LG_BN;

  double2 ra[NA], rb[NB];
  auto load = [&](int k0) {
#pragma unroll
    for (int q = 0; q < NA; ++q) {
      const int e = tid + 256 * q;  // double2 index in [0, BM * BK / 2)
      const int mm = e / (LG_BK / 2), kk = 2 * (e % (LG_BK / 2));
      const int gm = m0 + mm;
      ra[q] = gm < M ? __ldg(reinterpret_cast<const double2*>(bt.A + (size_t)gm * bt.lda + k0 + kk)) : make_double2(0, 0);
    }
#pragma unroll
    for (int q = 0; q < NB; ++q) {
      const int e = tid + 256 * q;  // double2 index in [0, BK * BN / 2)
      const int kk = e / (LG_BN / 2), nn = 2 * (e % (LG_BN / 2));
      const int gk = k0 + kk, gn = n0 + nn;
      double2 v = make_double2(0, 0);
      if (gk < K && gn < N) {
        if (!PAIR) {
          v = __ldg(reinterpret_cast<const double2*>(bt.B0 + (size_t)gk * bt.ldb + gn));
        } else {  // pair density: conj(Bj) * Bi at complex index gn / 2
          const size_t off = (size_t)gk * (bt.ldb >> 1) + (gn >> 1);
          const cplx bj = __ldg(reinterpret_cast<const cplx*>(bt.B0) + off);
          const cplx bi = __ldg(reinterpret_cast<const cplx*>(bt.B1) + off);
          const cplx z = cmulc(bj, bi);
          v = make_double2(z.x, z.y);
        }
      }
      rb[q] = v;
    }
  };
  auto store = [&](int s) {
    double* as = As + s * BM * LG_LDA;
    double* bs = Bs + s * LG_BK * LG_LDB;
#pragma unroll
    for (int q = 0; q < NA; ++q) {
      const int e = tid + 256 * q;
      *reinterpret_cast<double2*>(as + (e / (LG_BK / 2)) * LG_LDA + 2 * (e % (LG_BK / 2))) = ra[q];
    }
#pragma unroll
    for (int q = 0; q < NB; ++q) {
      const int e = tid + 256 * q;
      *reinterpret_cast<double2*>(bs + (e / (LG_BN / 2)) * LG_LDB + 2 * (e % (LG_BN / 2))) = rb[q];
    }
  };

  double acc[MT][2][2];
#pragma unroll
  for (int i = 0; i < MT; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
  const int nchunk = (K + LG_BK - 1) / LG_BK;
  load(0);
  store(0);
  if (nchunk > 1) load(LG_BK);
  __syncthreads();
  for (int c = 0; c < nchunk; ++c) {
    const double* as = As + (c & 1) * BM * LG_LDA + (wm * MT * 8 + gid) * LG_LDA + tig;
    const double* bs = Bs + (c & 1) * LG_BK * LG_LDB + tig * LG_LDB + wn * 16 + gid;
#pragma unroll
    for (int ks = 0; ks < LG_BK / 4; ++ks) {
      double a[MT], b[2];
#pragma unroll
      for (int i = 0; i < MT; ++i) a[i] = as[i * 8 * LG_LDA + 4 * ks];
#pragma unroll
      for (int j = 0; j < 2; ++j) b[j] = bs[4 * ks * LG_LDB + 8 * j];
#pragma unroll
      for (int i = 0; i < MT; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) lg_dmma(acc[i][j][0], acc[i][j][1], a[i], b[j]);
    }
    if (c + 1 < nchunk) {
      store((c + 1) & 1);  // the other buffer: last read in chunk c - 1, before the previous barrier
      if (c + 2 < nchunk) load((c + 2) * LG_BK);
    }
    __syncthreads();
  }
  // C(row gid, cols 2 tig, 2 tig + 1) of each tile
#pragma unroll
  for (int i = 0; i < MT; ++i) {
    const int gm = m0 + wm * MT * 8 + i * 8 + gid;
    if (gm >= M) continue;
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const int gn = n0 + wn * 16 + j * 8 + 2 * tig;
      if (gn < N) *reinterpret_cast<double2*>(bt.C + (size_t)gm * bt.ldc + gn) = make_double2(acc[i][j][0], acc[i][j][1]);
    }
  }
}

template <int MT, bool PAIR>
static void lg_launch(const LegGemmBatch* d_batches, int nbatch, int M, int K, int N, cudaStream_t st) {
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(legendre_gemm_kernel<MT, PAIR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lg_smem_bytes(MT));
    attr = true;
  }
  dim3 grid((N + LG_BN - 1) / LG_BN, (M + 16 * MT - 1) / (16 * MT), nbatch);
  legendre_gemm_kernel<MT, PAIR><<<grid, 256, lg_smem_bytes(MT), st>>>(d_batches, M, K, N);
}

int launch_legendre_gemm(const LegGemmBatch* d_batches, int nbatch, int M, int K, int N, bool pair,
                         cudaStream_t st) {
  return launch_legendre_gemm_mt(d_batches, nbatch, M, K, N, pair, 0, st);
}

// mt: the CTA's m-tiles (3: 48 rows, 6: 96 rows); 0 chooses by M
int launch_legendre_gemm_mt(const LegGemmBatch* d_batches, int nbatch, int M, int K, int N, bool pair, int mt,
                            cudaStream_t st) {
  if (nbatch <= 0) return 0;
  if (N % 2) return (int)cudaErrorInvalidValue;  // slabs are complex: 16-byte pairs
  if (mt == 3 || (mt != 6 && M <= 48)) {
    if (pair) lg_launch<3, true>(d_batches, nbatch, M, K, N, st);
    else lg_launch<3, false>(d_batches, nbatch, M, K, N, st);
  } else {
    if (pair) lg_launch<6, true>(d_batches, nbatch, M, K, N, st);
    else lg_launch<6, false>(d_batches, nbatch, M, K, N, st);
  }
  return (int)cudaGetLastError();
}

}  // namespace td1c
