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
// Register-tiled FP64 FFMA GEMM: B200's FP64 rate is the same on the CUDA
// cores as through DMMA, and tcgen05 has no f64 kind.  256 threads, thread
// micro-tile TM x 4, CTA tile (16 TM) x 64 x 16, smem double-buffered via
// register prefetch.  Rows of the table below |m| are zero, which reproduces
// the reference's l >= |m| loop bounds.
#include "common.cuh"
#include "kernels.cuh"

namespace td1c {

template <int TM, bool PAIR>
__global__ void __launch_bounds__(256)
legendre_gemm_kernel(const LegGemmBatch* __restrict__ batches, int M, int K, int N) {
  constexpr int BM = 16 * TM, BN = 64, BK = 16;
  __shared__ double As[BK][BM + 1];
  __shared__ double Bs[BK][BN];
  const LegGemmBatch bt = batches[blockIdx.z];
  const double* __restrict__ A = bt.A;
  double* __restrict__ C = bt.C;
  const int tid = threadIdx.x;
  // warp-friendly thread grid: each warp covers 4 (ty) x 8 (tx)
  const int warp = tid >> 5, lane = tid & 31;
  const int ty = (warp >> 1) * 4 + (lane >> 3);
  const int tx = (warp & 1) * 8 + (lane & 7);
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;

  double acc[TM][4];
#pragma unroll
  for (int i = 0; i < TM; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;

  // global -> register staging
  constexpr int A_PER = BM * BK / 256;  // = TM
  double ra[A_PER];
  double rb[4];
  auto load_tiles = [&](int k0) {
#pragma unroll
    for (int q = 0; q < A_PER; ++q) {
      int e = tid + 256 * q;        // e in [0, BM*BK)
      int mm = e / BK, kk = e % BK;
      int gm = m0 + mm, gk = k0 + kk;
      ra[q] = (gm < M && gk < K) ? __ldg(A + (size_t)gm * K + gk) : 0.0;
    }
    if (!PAIR) {
      const double* __restrict__ B = bt.B0;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        int e = tid + 256 * q;      // e in [0, BK*BN)
        int kk = e / BN, nn = e % BN;
        int gk = k0 + kk, gn = n0 + nn;
        rb[q] = (gk < K && gn < N) ? __ldg(B + (size_t)gk * bt.ldb + gn) : 0.0;
      }
    } else {
      // pair density: element (k, n) of conj(Bj) * Bi, complex index n/2
      const cplx* __restrict__ Bj = reinterpret_cast<const cplx*>(bt.B0);
      const cplx* __restrict__ Bi = reinterpret_cast<const cplx*>(bt.B1);
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        int e = tid + 256 * q;      // complex element in [0, BK*BN/2)
        int kk = e / (BN / 2), cc = e % (BN / 2);
        int gk = k0 + kk, gc = (n0 >> 1) + cc;
        cplx z = mkc(0.0, 0.0);
        if (gk < K && 2 * gc < N) {
          size_t off = (size_t)gk * (bt.ldb >> 1) + gc;
          cplx bj = __ldg(Bj + off), bi = __ldg(Bi + off);
          z = cmulc(bj, bi);
        }
        rb[2 * q] = z.x; rb[2 * q + 1] = z.y;
      }
    }
  };
  auto store_tiles = [&]() {
#pragma unroll
    for (int q = 0; q < A_PER; ++q) {
      int e = tid + 256 * q;
      As[e % BK][e / BK] = ra[q];
    }
    if (!PAIR) {
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        int e = tid + 256 * q;
        Bs[e / BN][e % BN] = rb[q];
      }
    } else {
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        int e = tid + 256 * q;
        int kk = e / (BN / 2), cc = e % (BN / 2);
        Bs[kk][2 * cc] = rb[2 * q];
        Bs[kk][2 * cc + 1] = rb[2 * q + 1];
      }
    }
  };

  load_tiles(0);
  for (int k0 = 0; k0 < K; k0 += BK) {
    store_tiles();
    __syncthreads();
    if (k0 + BK < K) load_tiles(k0 + BK);
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      double a[TM], b[4];
#pragma unroll
      for (int i = 0; i < TM; ++i) a[i] = As[kk][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < TM; ++i) {
    int gm = m0 + ty + 16 * i;
    if (gm >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      int gn = n0 + tx + 16 * j;
      if (gn < N) C[(size_t)gm * bt.ldc + gn] = acc[i][j];
    }
  }
}

int launch_legendre_gemm(const LegGemmBatch* d_batches, int nbatch, int M, int K, int N, bool pair,
                         cudaStream_t st) {
  if (nbatch <= 0) return 0;
  dim3 block(256);
  if (M <= 48) {
    dim3 grid((N + 63) / 64, (M + 47) / 48, nbatch);
    if (pair) legendre_gemm_kernel<3, true><<<grid, block, 0, st>>>(d_batches, M, K, N);
    else legendre_gemm_kernel<3, false><<<grid, block, 0, st>>>(d_batches, M, K, N);
  } else {
    dim3 grid((N + 63) / 64, (M + 95) / 96, nbatch);
    if (pair) legendre_gemm_kernel<6, true><<<grid, block, 0, st>>>(d_batches, M, K, N);
    else legendre_gemm_kernel<6, false><<<grid, block, 0, st>>>(d_batches, M, K, N);
  }
  return (int)cudaGetLastError();
}

}  // namespace td1c
