// reductions.cu -- orbital matrix elements and MO integrals of the RHS.
//
// orbdots: for every (j, i) with m_j = m_i, i dynamic, over the nbas basis
//   A(j,i) = <phi_j | (g + h1 + h0) phi_i>          hprod_mkint1_sph.F90:2-103
//   B(j,i) = <phi_j | v2 phi_i>                      (A + B = <phi_j|F phi_i>,
//                                                    hprod_htot_mkxmat.F90 _cc/_ca/_aa1)
//   C(j,i) = <(h0 + h1) phi_j | phi_i>, j frozen     hprod_htot_mkxmat.F90:2-77
//   E(i)   = <phi_i | (h0 + h1) phi_i>, i dynamic core   hprod_ene_dcore.F90
//   GV(j,i) = <phi_j | (g + v2) phi_i>, j frozen     hprod_htot_mkxmat.F90:2-77
// as deterministic two-pass reductions (per-chunk partials, then a fixed-
// order sum), the race-free pattern of the reference's per-thread partial
// arrays.
//
// int2e (hprod_mkint2_sph.F90:2-100): int2e(i,j,k,l) = sum_{r,L} rho2_ij v2sph_kl
// for i >= j active and m_i + m_k = m_j + m_l.  The m rule splits the
// (ij) x (kl) matrix into dense blocks by delta = m_i - m_j; each block is a
// complex GEMM over K = Nr (lmax2 + 1) split across CTAs, with A/B chunks
// staged in shared memory; partials are summed in a fixed order and the
// i < j half is filled by int2e(i,j,k,l) = conj(int2e(j,i,l,k)).
#include "common.cuh"
#include "kernels.cuh"
#include "reductions.cuh"

namespace td1c {

constexpr int OD_CHUNK = 128;

__global__ void __launch_bounds__(256) orbdots_kernel(OrbdotsArgs a) {
  extern __shared__ cplx sm[];
  const int nfun = a.nfun, C = OD_CHUNK;
  cplx* so = sm;                       // [nfun][C] orb
  cplx* sf = so + (size_t)nfun * C;    // [nfun][C] g + h1 + h0
  cplx* sv = sf + (size_t)nfun * C;    // [nfun][C] v2
  cplx* sh = sv + (size_t)nfun * C;    // [nfun][C] h0 + h1
  cplx* sgv = sh + (size_t)nfun * C;   // [nfun][C] g + v2
  const size_t base = (size_t)blockIdx.x * C;
  for (int e = threadIdx.x; e < nfun * C; e += blockDim.x) {
    int f = e / C, k = e % C;
    size_t g = base + k;
    cplx o = mkc(0, 0), fv = mkc(0, 0), v = mkc(0, 0), h = mkc(0, 0), gv = mkc(0, 0);
    if (g < (size_t)a.nbas) {
      size_t idx = (size_t)f * a.nbas + g;
      o = a.orb[idx];
      cplx h0 = a.h0orb[idx], h1 = a.h1orb[idx], gg = a.gorb[idx];
      fv = cadd(cadd(gg, h1), h0);
      v = a.v2orb[idx];
      h = cadd(h0, h1);
      gv = cadd(gg, v);
    }
    so[e] = o; sf[e] = fv; sv[e] = v; sh[e] = h; sgv[e] = gv;
  }
  __syncthreads();
  cplx* out = a.partial + (size_t)blockIdx.x * a.nent;
  // one warp per entry, lanes over the chunk (conflict-free), fixed-order
  // shuffle reduction
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int t = wid; t < a.nent; t += nw) {
    const int4 en = a.ent[t];  // (kind, j, i, 0)
    const int kind = en.x, j = en.y, i = en.z;
    const cplx* x; const cplx* y;
    if (kind == 0) { x = so + j * C; y = sf + i * C; }        // A
    else if (kind == 1) { x = so + j * C; y = sv + i * C; }   // B
    else if (kind == 2) { x = sh + j * C; y = so + i * C; }   // C
    else if (kind == 3) { x = so + i * C; y = sh + i * C; }   // E
    else { x = so + j * C; y = sgv + i * C; }                 // <phi_j|(g+v2) phi_i>
    cplx s = mkc(0, 0);
    for (int k = lane; k < C; k += 32) {
      cplx xv = x[k], yv = y[k];
      s.x = fma(xv.x, yv.x, fma(xv.y, yv.y, s.x));
      s.y = fma(xv.x, yv.y, fma(-xv.y, yv.x, s.y));
    }
    for (int o = 16; o > 0; o >>= 1) { s.x += __shfl_xor_sync(0xffffffff, s.x, o); s.y += __shfl_xor_sync(0xffffffff, s.y, o); }
    if (lane == 0) out[t] = s;
  }
}

// fixed-order sum of the per-chunk partials: one warp per entry, lane l adds
// chunks l, l + 32, ... in order, then a fixed xor tree combines the lanes
__global__ void sum_partials_kernel(const cplx* __restrict__ partial, int nchunk, int nent, cplx* __restrict__ out) {
  const int t = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (t >= nent) return;
  cplx s = mkc(0, 0);
  for (int c = lane; c < nchunk; c += 32) s = cadd(s, partial[(size_t)c * nent + t]);
  for (int o = 16; o > 0; o >>= 1) { s.x += __shfl_xor_sync(0xffffffffu, s.x, o); s.y += __shfl_xor_sync(0xffffffffu, s.y, o); }
  if (lane == 0) out[t] = s;
}

int orbdots_nchunk(size_t nbas) { return (int)((nbas + OD_CHUNK - 1) / OD_CHUNK); }

int launch_orbdots(const OrbdotsArgs& a, cudaStream_t st) {
  const int nchunk = orbdots_nchunk((size_t)a.nbas);
  size_t smem = sizeof(cplx) * 5 * (size_t)a.nfun * OD_CHUNK;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(orbdots_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    attr = true;
  }
  orbdots_kernel<<<nchunk, 256, smem, st>>>(a);
  sum_partials_kernel<<<(a.nent + 7) / 8, 256, 0, st>>>(a.partial, nchunk, a.nent, a.result);
  return (int)cudaGetLastError();
}

// ---------------------------------------------------------------------------
// int2e block GEMM: C(ij, kl) = sum_x A_ij[x] B_kl[x] over x in [0, K)
// CTA = (K split, block); 192 threads = 2 K slices x (8 row groups x 12
// column groups), each thread a 3 x 3 complex register tile; K chunks of 32
// staged in shared memory with a one-chunk register prefetch.
// ---------------------------------------------------------------------------
constexpr int I2_KC = 32, I2_R = 24, I2_C = 36, I2_NT = 192;

__global__ void __launch_bounds__(I2_NT) int2e_block_kernel(Int2eArgs a) {
  __shared__ cplx sA[I2_R][I2_KC + 1];
  __shared__ cplx sB[I2_C][I2_KC + 1];
  cplx (*sred)[9] = reinterpret_cast<cplx (*)[9]>(&sB[0][0]);  // reuses sB after the K loop
  const Int2eBlock blk = a.blocks[blockIdx.y];
  const int nr = blk.nrow, nc = blk.ncol;
  const int t = threadIdx.x;
  const int slice = t / 96, tt = t % 96;
  // compact 3 x 3 tiles over the block's actual shape: only ceil(nr/3) x
  // ceil(nc/3) threads of a slice compute, so small blocks occupy few warps
  const int ncg = (nc + 2) / 3, nrg = (nr + 2) / 3;
  const bool act = tt < nrg * ncg;
  const int rg = act ? tt / ncg : 0, cg = act ? tt % ncg : 0;
  const size_t K = a.K;
  const size_t kper = ((K + gridDim.x - 1) / gridDim.x + I2_KC - 1) / I2_KC * I2_KC;
  const size_t k0 = (size_t)blockIdx.x * kper, k1 = min(K, k0 + kper);
  cplx acc[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) acc[i][j] = mkc(0, 0);
  // each thread stages up to 4 A and 6 B elements per chunk
  constexpr int NA = (I2_R * I2_KC + I2_NT - 1) / I2_NT, NB = (I2_C * I2_KC + I2_NT - 1) / I2_NT;
  cplx ra[NA], rb[NB];
  auto load = [&](size_t kc) {
#pragma unroll
    for (int u = 0; u < NA; ++u) {
      int e = t + u * I2_NT;
      int rr = e / I2_KC, kk = e % I2_KC;
      cplx v = mkc(0, 0);
      if (rr < nr && kc + kk < k1) v = __ldg(a.rho2 + (size_t)a.row_pair[blk.row0 + rr] * K + kc + kk);
      ra[u] = v;
    }
#pragma unroll
    for (int u = 0; u < NB; ++u) {
      int e = t + u * I2_NT;
      int cc = e / I2_KC, kk = e % I2_KC;
      cplx v = mkc(0, 0);
      if (cc < nc && kc + kk < k1) {
        int2 pc = a.col_pair[blk.col0 + cc];
        v = __ldg(a.v2sph + (size_t)pc.x * K + kc + kk);
        if (pc.y) v = cconj(v);
      }
      rb[u] = v;
    }
  };
  if (k0 < k1) load(k0);
  for (size_t kc = k0; kc < k1; kc += I2_KC) {
#pragma unroll
    for (int u = 0; u < NA; ++u) { int e = t + u * I2_NT; if (e < I2_R * I2_KC) sA[e / I2_KC][e % I2_KC] = ra[u]; }
#pragma unroll
    for (int u = 0; u < NB; ++u) { int e = t + u * I2_NT; if (e < I2_C * I2_KC) sB[e / I2_KC][e % I2_KC] = rb[u]; }
    __syncthreads();
    if (kc + I2_KC < k1) load(kc + I2_KC);
#pragma unroll 4
    for (int kk = slice; act && kk < I2_KC; kk += 2) {
      cplx av[3], bv[3];
#pragma unroll
      for (int i = 0; i < 3; ++i) av[i] = sA[rg * 3 + i][kk];
#pragma unroll
      for (int j = 0; j < 3; ++j) bv[j] = sB[cg * 3 + j][kk];
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) cfma(acc[i][j], av[i], bv[j]);
    }
    __syncthreads();
  }
  if (slice == 1 && act) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) sred[tt][i * 3 + j] = acc[i][j];
  }
  __syncthreads();
  if (slice == 0 && act) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        int r = rg * 3 + i, c = cg * 3 + j;
        if (r < nr && c < nc)
          a.partial[((size_t)blockIdx.x * a.nblkent) + blk.ent0 + r * nc + c] = cadd(acc[i][j], sred[tt][i * 3 + j]);
      }
  }
}

// one warp per entry: lane l adds splits l, l + 32, ... in order, then a
// fixed xor tree combines the lanes (deterministic)
__global__ void int2e_sum_kernel(Int2eArgs a, int nsplit) {
  const int t = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (t >= a.nblkent) return;
  cplx s = mkc(0, 0);
  for (int c = lane; c < nsplit; c += 32) s = cadd(s, a.partial[(size_t)c * a.nblkent + t]);
  for (int o = 16; o > 0; o >>= 1) { s.x += __shfl_xor_sync(0xffffffffu, s.x, o); s.y += __shfl_xor_sync(0xffffffffu, s.y, o); }
  if (lane) return;
  int4 d = a.ent_dst[t];  // (i, j, k, l) active indices
  const int n = a.nact;
  a.int2e[d.x + n * (d.y + n * (d.z + n * d.w))] = s;
}

__global__ void int2e_fill_kernel(Int2eArgs a) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = a.nact;
  if (t >= n * n * n * n) return;
  int i = t % n, j = (t / n) % n, k = (t / (n * n)) % n, l = t / (n * n * n);
  if (i < j) a.int2e[t] = cconj(a.int2e[j + n * (i + n * (l + n * k))]);
}

// fixed-order sum of nsplit partial blocks into int2e, then the i < j half
int launch_int2e_sum_fill(const Int2eArgs& a, int nsplit, cudaStream_t st) {
  const int n = a.nact, n4 = n * n * n * n;
  if (a.nblkent > 0) int2e_sum_kernel<<<(a.nblkent + 7) / 8, 256, 0, st>>>(a, nsplit);
  int2e_fill_kernel<<<(n4 + 127) / 128, 128, 0, st>>>(a);
  return (int)cudaGetLastError();
}

int launch_int2e(const Int2eArgs& a, int nsplit, cudaStream_t st) {
  const int n = a.nact, n4 = n * n * n * n;
  if (n4 == 0) return 0;
  cudaError_t e = cudaMemsetAsync(a.int2e, 0, sizeof(cplx) * n4, st);
  if (e != cudaSuccess) { fprintf(stderr, "td1c_b200: int2e memset: %s\n", cudaGetErrorString(e)); return (int)e; }
  if (a.nblocks > 0) {
    dim3 grid(nsplit, a.nblocks);
    int2e_block_kernel<<<grid, I2_NT, 0, st>>>(a);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
      fprintf(stderr, "td1c_b200: int2e block kernel (grid %d x %d): %s\n", nsplit, a.nblocks, cudaGetErrorString(e));
      return (int)e;
    }
    int2e_sum_kernel<<<(a.nblkent + 7) / 8, 256, 0, st>>>(a, nsplit);
    e = cudaGetLastError();
    if (e != cudaSuccess) { fprintf(stderr, "td1c_b200: int2e sum: %s\n", cudaGetErrorString(e)); return (int)e; }
  }
  int2e_fill_kernel<<<(n4 + 127) / 128, 128, 0, st>>>(a);
  return (int)cudaGetLastError();
}

}  // namespace td1c
