// int2e_dmma.cu -- MO two-electron integrals (hprod_mkint2_sph.F90:2-100)
// on the FP64 tensor cores.
//
// int2e(i,j,k,l) = sum_x rho2_ij[x] v2sph_kl[x] over x in [0, K), K =
// Nr (lmax2 + 1), for i >= j and m_i + m_k = m_j + m_l.  For every Delta =
// m_i - m_j the rows ij and the columns kl form a dense complex product
// C = A B^T, computed with four real products per complex depth step:
//   Re C += Re A Re B + Im A (-Im B),   Im C += Re A Im B + Im A Re B
// on mma.sync.m8n8k4.f64 tiles of 8 rows x 8 columns x 4 complex depths,
// each of the four products in its own accumulator (independent chains).
// Lane (g, t) of a fragment handles depth x = 4 s + t, so one 128-bit
// shared-memory load gives it both parts of its A (row g) or B (column g)
// element; a conjugated column flips the sign of Im B in the same lane.
//
// One CTA owns a slice of K and every block: the slice of each A row (rho2
// of the block rows) and each B row (v2sph of the block columns) is staged
// in shared memory by cp.async in a 4-stage ring (each thread's copy
// addresses computed once); the 16 warps run the groups (m-tile x up to 3
// n-tiles) the host assigned to them.  Each CTA writes its partial sums;
// int2e_sum_kernel adds them in a fixed order.
#include "common.cuh"
#include "kernels.cuh"
#include "reductions.cuh"

namespace td1c {

constexpr int I2D_KC = 16;                 // complex depth per stage
constexpr int I2D_PITCH = 2 * I2D_KC + 8;  // doubles per staged row: rows 2g, 2g+1 fall in opposite bank halves
constexpr int I2D_NS = 4;                  // stages
constexpr int I2D_LMAX = 8;                // staged 16-byte copies per thread and stage (nrows KC <= 8 NW 32)

__device__ __forceinline__ void dmma_8x8x4(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}
__device__ __forceinline__ void cp_async_16(unsigned dst, const void* src, unsigned src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

size_t int2e_dmma_smem(const I2dArgs& a) {
  return sizeof(double) * (size_t)I2D_NS * (a.nra + a.nrb) * I2D_PITCH;
}
bool int2e_dmma_fits(const I2dArgs& a) {
  return int2e_dmma_smem(a) <= 227 * 1024 && (size_t)(a.nra + a.nrb) * I2D_KC <= (size_t)I2D_LMAX * I2D_NW * 32;
}

__global__ void __launch_bounds__(I2D_NW * 32, 1) int2e_dmma_kernel(I2dArgs a) {
  extern __shared__ __align__(16) double i2d_smem[];
  const int nrows = a.nra + a.nrb;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int gid = lane >> 2, tig = lane & 3;
  const size_t K = a.K;
  const size_t kper = ((K + gridDim.x - 1) / gridDim.x + I2D_KC - 1) / I2D_KC * I2D_KC;
  const size_t k0 = (size_t)blockIdx.x * kper, k1 = min(K, k0 + kper);
  const int nchunk = k1 > k0 ? (int)((k1 - k0 + I2D_KC - 1) / I2D_KC) : 0;
  const unsigned stage_bytes = (unsigned)(sizeof(double) * nrows * I2D_PITCH);
  const unsigned smem0 = (unsigned)__cvta_generic_to_shared(i2d_smem);

  // padding rows hold zeros in every stage and are never loaded
  for (int row = warp; row < nrows; row += I2D_NW) {
    const int pr = row < a.nra ? a.a_pair[row] : a.b_pair[row - a.nra].x;
    if (pr < 0)
      for (int e = lane; e < I2D_NS * I2D_PITCH; e += 32)
        i2d_smem[(size_t)(e / I2D_PITCH) * nrows * I2D_PITCH + (size_t)row * I2D_PITCH + e % I2D_PITCH] = 0.0;
  }
  // this thread's copies: element e = tid + i blockDim (row e / KC, depth e % KC)
  const cplx* src[I2D_LMAX];
  unsigned dst[I2D_LMAX];
  int kofs[I2D_LMAX];
#pragma unroll
  for (int i = 0; i < I2D_LMAX; ++i) {
    const int e = tid + i * blockDim.x;
    src[i] = nullptr; dst[i] = 0; kofs[i] = 0;
    if (e < nrows * I2D_KC) {
      const int row = e / I2D_KC, kk = e % I2D_KC;
      const int pr = row < a.nra ? a.a_pair[row] : a.b_pair[row - a.nra].x;
      if (pr >= 0) {
        src[i] = (row < a.nra ? a.rho2 : a.v2sph) + (size_t)pr * K + k0 + kk;
        dst[i] = smem0 + (unsigned)(sizeof(double) * ((size_t)row * I2D_PITCH + 2 * kk));
        kofs[i] = kk;
      }
    }
  }
  auto load = [&](int chunk) {
    if (chunk >= nchunk) return;
    const size_t kb = (size_t)chunk * I2D_KC;
    const unsigned so = (unsigned)(chunk % I2D_NS) * stage_bytes;
    const bool tail = k0 + kb + I2D_KC > k1;
#pragma unroll
    for (int i = 0; i < I2D_LMAX; ++i) {
      if (!src[i]) continue;
      if (!tail) {
        cp_async_16(dst[i] + so, src[i] + kb, 16u);
      } else {  // past k1: zero fill, reading nothing, from the slice's first (valid) element
        const bool in = k0 + kb + kofs[i] < k1;
        cp_async_16(dst[i] + so, in ? src[i] + kb : src[i] - kofs[i], in ? 16u : 0u);
      }
    }
  };

  // this warp's groups with the lane's fragment offsets (in double2 units)
  int nnt[I2D_MAXG], aoff[I2D_MAXG], boff[I2D_MAXG][I2D_NTMAX];
  unsigned bcj[I2D_MAXG];  // bit t: n-tile t of the lane's column is conjugated
  // [g][t][chain][c0|c1]: Re A Re B, Im A (-Im B), Re A Im B, Im A Re B as
  // four independent accumulator chains, added at the end
  double acc[I2D_MAXG][I2D_NTMAX][4][2];
  const int* wg = a.warp_group + ((size_t)blockIdx.y * I2D_NW + warp) * I2D_MAXG;
#pragma unroll
  for (int g = 0; g < I2D_MAXG; ++g) {
    const int gi = wg[g];
    const I2dGroup G = gi >= 0 ? a.groups[gi] : I2dGroup{0, 0, 0, 0};
    nnt[g] = G.nnt;
    aoff[g] = (G.arow0 + gid) * (I2D_PITCH / 2) + tig;
    bcj[g] = 0;
#pragma unroll
    for (int t = 0; t < I2D_NTMAX; ++t) {
      const int brow = G.brow0 + 8 * t + gid;
      boff[g][t] = (a.nra + brow) * (I2D_PITCH / 2) + tig;
      if (t < G.nnt && a.b_pair[brow].y) bcj[g] |= 1u << t;
#pragma unroll
      for (int h = 0; h < 4; ++h) acc[g][t][h][0] = acc[g][t][h][1] = 0.0;
    }
  }

#pragma unroll
  for (int s = 0; s < I2D_NS - 1; ++s) { load(s); cp_async_commit(); }
  for (int chunk = 0; chunk < nchunk; ++chunk) {
    cp_async_wait<I2D_NS - 2>();
    __syncthreads();  // stage chunk % NS complete for every thread; stage (chunk - 1) % NS free
    load(chunk + I2D_NS - 1);
    cp_async_commit();
    const double2* sm = reinterpret_cast<const double2*>(i2d_smem + (size_t)(chunk % I2D_NS) * nrows * I2D_PITCH);
#pragma unroll
    for (int g = 0; g < I2D_MAXG; ++g) {
      if (nnt[g] == 0) continue;
#pragma unroll
      for (int s = 0; s < I2D_KC / 4; ++s) {
        const double2 av = sm[aoff[g] + 4 * s];
#pragma unroll
        for (int t = 0; t < I2D_NTMAX; ++t) {
          if (t < nnt[g]) {
            const double2 bv = sm[boff[g][t] + 4 * s];
            const double bi = ((bcj[g] >> t) & 1) ? -bv.y : bv.y;
            dmma_8x8x4(acc[g][t][0][0], acc[g][t][0][1], av.x, bv.x);
            dmma_8x8x4(acc[g][t][1][0], acc[g][t][1][1], av.y, -bi);
            dmma_8x8x4(acc[g][t][2][0], acc[g][t][2][1], av.x, bi);
            dmma_8x8x4(acc[g][t][3][0], acc[g][t][3][1], av.y, bv.x);
          }
        }
      }
    }
  }
  cp_async_wait<0>();
  // partial sums: C(row gid, col 2 tig + i) of each tile
  double2* out = reinterpret_cast<double2*>(a.partial) + (size_t)blockIdx.x * a.nblkent;
#pragma unroll
  for (int g = 0; g < I2D_MAXG; ++g) {
    if (nnt[g] == 0) continue;
    const I2dGroup G = a.groups[wg[g]];
    const int ae = a.a_ent[G.arow0 + gid];
#pragma unroll
    for (int t = 0; t < I2D_NTMAX; ++t) {
      if (t >= nnt[g]) continue;
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int bc = a.b_col[G.brow0 + 8 * t + 2 * tig + i];
        if (ae >= 0 && bc >= 0)
          out[ae + bc] = make_double2(acc[g][t][0][i] + acc[g][t][1][i], acc[g][t][2][i] + acc[g][t][3][i]);
      }
    }
  }
}

int launch_int2e_dmma(const I2dArgs& d, const Int2eArgs& sum, int nsplit, cudaStream_t st) {
  const int n = sum.nact, n4 = n * n * n * n;
  if (n4 == 0) return 0;
  cudaError_t e = cudaMemsetAsync(sum.int2e, 0, sizeof(cplx) * n4, st);
  if (e != cudaSuccess) return (int)e;
  if (d.ngroups > 0) {
    if (!int2e_dmma_fits(d)) return (int)cudaErrorInvalidValue;
    const size_t smem = int2e_dmma_smem(d);
    static bool attr = false;
    if (!attr) {
      cudaFuncSetAttribute(int2e_dmma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
      attr = true;
    }
    dim3 grid(nsplit, d.nsets);
    int2e_dmma_kernel<<<grid, I2D_NW * 32, smem, st>>>(d);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
      fprintf(stderr, "td1c_b200: int2e DMMA kernel (grid %d x %d, smem %zu): %s\n", nsplit, d.nsets, smem,
              cudaGetErrorString(e));
      return (int)e;
    }
  }
  return launch_int2e_sum_fill(sum, nsplit, st);
}

}  // namespace td1c
