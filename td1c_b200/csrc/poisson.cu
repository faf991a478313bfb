// poisson.cu -- multipole radial Poisson solve (hprod_mkv2mf.F90:118-182).
//
// For every stored orbital pair p and multipole l >= |m_p| the reference
// splits rho2(:, l, p) into real and imaginary parts, forms
//     t   = sum_r rho(r) r^l / (2 pi) / r_max^(2l+1)
//     rhs = rho(r) (2l+1) / (2 pi r sqrt(w_r))
// solves  L_l L_l^T x = rhs  with the dpbtrf factor of
// [l(l+1)/r^2 + 2 T] (band nd) by dpbtrs, and returns
//     v2sph = (x + t r^(l+1) sqrt(w_r)) 4 pi / ((2l+1) r sqrt(w_r)).
//
// Layout of the work: one warp per (l, group of 16 pairs); lane 2P+c solves
// the real (c = 0) or imaginary (c = 1) part of pair P.  The substitutions
// run row by row in the order of dtbsv (forward: band terms oldest first,
// backward: farthest first), with the last nd solution values in registers
// and the older band terms summed into four partial sums so only the newest
// term sits on the recurrence.  Everything a row needs from the matrix side
// -- the nd band values, the reciprocal diagonal and the two per-row scaling
// factors -- is one row of a per-l table (tabf for the forward sweep, tabb
// for the backward one), so a row costs a handful of 128-bit broadcast loads
// from shared memory.  Blocks of nd rows move between HBM and shared memory
// by the TMA: per block one bulk copy of the table rows and one tensor copy
// of the 16 pairs' nd complex values (a 4-d box over (re|im, pair, row, l)
// that lands as [row][pair][re|im], so every lane reads one contiguous line
// per row; rows past Nr zero-filled) land in a 4-stage ring tracked by
// mbarriers, and the
// forward result y and the final v2sph leave through one tensor store per
// block (clipped at Nr).  y is parked in the v2sph buffer between the
// sweeps.  Every mbarrier wait is bounded; a wait that runs out sets
// ST_TIMEOUT in the status word and the warp drains and returns.
#include <algorithm>

#include "common.cuh"
#include "kernels.cuh"
#include "tma.cuh"

namespace td1c {

namespace {

constexpr int PS_PAIRS = 16;      // pairs per warp
constexpr int PS_STAGES = 4;      // depth of the load ring

// byte offset of the staged-block ring: 128 bytes of mbarriers, the table
// stages, rounded up to the 128-byte alignment of a TMA box
__host__ __device__ constexpr size_t poisson_rbuf_offset(int nd, int w) {
  return (128 + (size_t)PS_STAGES * nd * w * 8 + 127) / 128 * 128;
}

}  // namespace

// Row tables of width W = ND + 4 rounded up to even (16-byte rows):
//   tabf[l][j] = { L(j, j-ND) .. L(j, j-1), 1/L(j,j), invr(j), rpl0(j), 0.. }
//   tabb[l][j] = { L(j+ND, j) .. L(j+1, j), 1/L(j,j), rpl1(j), fac2(j), 0.. }
// for j < Np (Nr rounded up to a multiple of ND); rows j >= Nr are identity
// rows (band 0, reciprocal diagonal 1, factors 0), band entries that fall
// outside 0..Nr-1 are 0.
__global__ void poisson_tables_kernel(PoissonArgs a, double* __restrict__ tabf, double* __restrict__ tabb) {
  const int ND = a.nd, LD = ND + 1, W = poisson_row_width(ND), Nr = a.Nr;
  const int Np = (Nr + ND - 1) / ND * ND;
  const size_t n = (size_t)a.L2 * Np;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const int l = (int)(e / Np), j = (int)(e % Np);
    const double* gL = a.d2ll + (size_t)l * Nr * LD;
    double* f = tabf + e * W;
    double* b = tabb + e * W;
    for (int i = 0; i < W; ++i) { f[i] = 0.0; b[i] = 0.0; }
    if (j >= Nr) { f[ND] = 1.0; b[ND] = 1.0; continue; }
    const size_t lr = (size_t)l * Nr + j;
    for (int i = 0; i < ND; ++i) {
      const int k = ND - i;
      if (j - k >= 0) f[i] = gL[(size_t)(j - k) * LD + k];
      if (j + k < Nr) b[i] = gL[(size_t)j * LD + k];
    }
    f[ND] = a.d2rinv[lr]; f[ND + 1] = a.invr[lr]; f[ND + 2] = a.rpl0[lr];
    b[ND] = a.d2rinv[lr]; b[ND + 1] = a.rpl1[lr]; b[ND + 2] = a.fac2[lr];
  }
}

template <int ND>
__global__ void __launch_bounds__(32, 1) poisson_kernel(const __grid_constant__ PoissonArgs a) {
  constexpr int W = (ND + 5) / 2 * 2;  // table row width (doubles)
  constexpr int BOX = 2 * ND;          // doubles per pair in a staged block
  extern __shared__ __align__(128) unsigned char ps_smem[];
  unsigned long long* bar = reinterpret_cast<unsigned long long*>(ps_smem);  // [PS_STAGES]
  double* fbuf = reinterpret_cast<double*>(ps_smem + 128);                   // [S][ND][W]
  double* rbuf = reinterpret_cast<double*>(ps_smem + poisson_rbuf_offset(ND, W));  // [S][16][BOX]
  double* ybuf = rbuf + PS_STAGES * PS_PAIRS * BOX;                                 // [2][16][BOX]

  const int l = blockIdx.x;
  const int lane = threadIdx.x;
  const int Nr = a.Nr;
  const int nb = (Nr + ND - 1) / ND, Np = nb * ND;
  const int p0 = blockIdx.y * PS_PAIRS;
  const int np = min(PS_PAIRS, a.npair - p0);
  const int P = lane >> 1;
  bool active = P < np;
  if (active) {
    const int m = a.pair_m[p0 + P];
    active = l >= (m < 0 ? -m : m);
  }
  const double* tabf_l = a.tabf + (size_t)l * Np * W;
  const double* tabb_l = a.tabb + (size_t)l * Np * W;
  // box bytes: rows past Nr and pairs past npair arrive zero-filled and count
  const unsigned tx_bytes = (unsigned)(ND * W * 8) + (unsigned)(BOX * a.boxp * 8);
  // a staged block is [row][pair][re|im] (boxp pairs), so lane 2P+c reads
  // row u at u * rstride + lane: one contiguous line per row
  const int rstride = 2 * a.boxp;
  const bool owner = P < a.boxp;  // lanes past the box must not write: their slots belong to the next row
  if (!owner) active = false;

  if (lane == 0) {
    for (int s = 0; s < PS_STAGES; ++s) mbar_init(&bar[s], 1);
    fence_mbar_init();
  }
  __syncwarp();

  // issue the loads of task q (forward block q, or backward block 2 nb - 1 - q)
  auto issue = [&](int q) {
    if (lane == 0) {
      const bool fwd = q < nb;
      const int b = fwd ? q : 2 * nb - 1 - q;
      const int s = q % PS_STAGES;
      mbar_expect_tx(&bar[s], tx_bytes);
      bulk_load(fbuf + (size_t)s * ND * W, (fwd ? tabf_l : tabb_l) + (size_t)b * ND * W, ND * W * 8, &bar[s]);
      tensor_load_4d(rbuf + (size_t)s * PS_PAIRS * BOX, fwd ? &a.tm_rho : &a.tm_v2, 0, p0, b * ND, l, &bar[s]);
    }
  };
  // store ybuf half h to the rows of block b (rows past Nr and pairs past
  // npair are clipped by the tensor map)
  auto store = [&](int h, int b) {
    fence_async_smem();
    __syncwarp();
    if (lane == 0) {
      tensor_store_4d(&a.tm_v2, 0, p0, b * ND, l, ybuf + (size_t)h * PS_PAIRS * BOX);
      bulk_commit();
    }
  };
  auto wait_task = [&](int q) -> bool {  // warp-uniform result
    const bool r = mbar_wait(&bar[q % PS_STAGES], (unsigned)((q / PS_STAGES) & 1));
    return __all_sync(0xffffffffu, r);
  };

  bool ok = true;
  int issued = 0, consumed = 0;  // tasks issued / consumed
  double win[ND];
  double t = 0.0;

  // ---- forward substitution  L y = rhs
  for (; issued < min(PS_STAGES, nb); ++issued) issue(issued);
#pragma unroll
  for (int k = 0; k < ND; ++k) win[k] = 0.0;
  for (int b = 0; b < nb; ++b) {
    if (!wait_task(b)) { ok = false; break; }
    consumed = b + 1;
    if (lane == 0) bulk_wait_read_1();  // ybuf half (b & 1) no longer read by the store of block b - 2
    __syncwarp();
    const int s = b % PS_STAGES, h = b & 1;
    const double* __restrict__ fb = fbuf + (size_t)s * ND * W;
    const double* __restrict__ rb = rbuf + (size_t)s * PS_PAIRS * BOX + lane;  // row u at rb[u * rstride]
    double* __restrict__ yb = ybuf + (size_t)h * PS_PAIRS * BOX + lane;
    // the block's inputs first and its results after it, so no shared-memory
    // store sits between the rows and the loads of later rows can be hoisted
    double in[ND];
#pragma unroll
    for (int u = 0; u < ND; ++u) in[u] = active ? rb[u * rstride] : 0.0;
#pragma unroll
    for (int u = 0; u < ND; ++u) {
      double fr[W];
#pragma unroll
      for (int i = 0; i < W / 2; ++i) {
        const double2 v = reinterpret_cast<const double2*>(fb + u * W)[i];
        fr[2 * i] = v.x; fr[2 * i + 1] = v.y;
      }
      const double rho = in[u];
      t = fma(rho, fr[ND + 2], t);
      // L(j, j-k) = fr[ND - k]; y_{j-k} in win[(u - k) mod ND]
      double pa = rho * fr[ND + 1], pb = 0.0, pc = 0.0, pd = 0.0;
#pragma unroll
      for (int k = ND; k >= 2; --k) {
        const double term = fr[ND - k] * win[(u - k + ND) % ND];
        const int g = (ND - k) & 3;
        if (g == 0) pa -= term; else if (g == 1) pb -= term; else if (g == 2) pc -= term; else pd -= term;
      }
      const double sacc = fma(-fr[ND - 1], win[(u - 1 + ND) % ND], (pa + pb) + (pc + pd));
      win[u] = sacc * fr[ND];
    }
#pragma unroll
    for (int u = 0; u < ND; ++u)
      if (owner) yb[u * rstride] = win[u];
    store(h, b);
    if (issued < nb) issue(issued++);
  }
  // all y stores complete and visible before the backward sweep reads them back
  if (lane == 0) bulk_wait_all();
  fence_async_global();
  __syncwarp();

  // ---- back substitution  L^T x = y, fused with the boundary term and scaling
  //      v2sph = (x + t fac1 r^(l+1) sqrt(w)) 4 pi / ((2l+1) r sqrt(w))
  if (ok) {
    t *= a.fac1[l];
#pragma unroll
    for (int k = 0; k < ND; ++k) win[k] = 0.0;
    for (; issued < min(nb + PS_STAGES, 2 * nb); ++issued) issue(issued);
    for (int i = 0; i < nb; ++i) {
      const int q = nb + i, b = nb - 1 - i;
      if (!wait_task(q)) { ok = false; break; }
      consumed = q + 1;
      if (lane == 0) bulk_wait_read_1();
      __syncwarp();
      const int s = q % PS_STAGES, h = q & 1;
      const double* __restrict__ fb = fbuf + (size_t)s * ND * W;
      const double* __restrict__ rb = rbuf + (size_t)s * PS_PAIRS * BOX + lane;
      double* __restrict__ yb = ybuf + (size_t)h * PS_PAIRS * BOX + lane;
      double in[ND];
#pragma unroll
      for (int u = 0; u < ND; ++u) in[u] = active ? rb[u * rstride] : 0.0;
#pragma unroll
      for (int u = ND - 1; u >= 0; --u) {
        double fr[W];
#pragma unroll
        for (int k2 = 0; k2 < W / 2; ++k2) {
          const double2 v = reinterpret_cast<const double2*>(fb + u * W)[k2];
          fr[2 * k2] = v.x; fr[2 * k2 + 1] = v.y;
        }
        const double yv = in[u];
        // L(j+k, j) = fr[ND - k]; x_{j+k} in win[(u + k) mod ND]; farthest first
        double pa = yv, pb = 0.0, pc = 0.0, pd = 0.0;
#pragma unroll
        for (int k = ND; k >= 2; --k) {
          const double term = fr[ND - k] * win[(u + k) % ND];
          const int g = (ND - k) & 3;
          if (g == 0) pa -= term; else if (g == 1) pb -= term; else if (g == 2) pc -= term; else pd -= term;
        }
        const double sacc = fma(-fr[ND - 1], win[(u + 1) % ND], (pa + pb) + (pc + pd));
        win[u] = sacc * fr[ND];
      }
#pragma unroll
      for (int u = 0; u < ND; ++u) {
        if (owner) yb[u * rstride] = fma(t, fb[u * W + ND + 1], win[u]) * fb[u * W + ND + 2];
      }
      store(h, b);
      if (issued < 2 * nb) issue(issued++);
    }
  }
  if (!ok) {
    if (lane == 0) atomicOr(a.status, ST_TIMEOUT);
    // let the loads still in flight land before the shared memory is released
    for (int q = consumed; q < issued; ++q) (void)wait_task(q);
  }
  if (lane == 0) bulk_wait_all();
}

template <int ND>
static int launch_nd(const PoissonArgs& a, cudaStream_t st) {
  constexpr int W = (ND + 5) / 2 * 2, BOX = 2 * ND;
  const size_t smem = poisson_rbuf_offset(ND, W) + sizeof(double) * (size_t)(PS_STAGES + 2) * PS_PAIRS * BOX;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(poisson_kernel<ND>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    attr = true;
  }
  if (a.npair <= 0) return 0;
  if (a.boxp != std::min(PS_PAIRS, a.npair)) return (int)cudaErrorInvalidValue;  // maps not encoded
  dim3 grid(a.L2, (a.npair + PS_PAIRS - 1) / PS_PAIRS);
  poisson_kernel<ND><<<grid, 32, smem, st>>>(a);
  return (int)cudaGetLastError();
}

// 3-d views [npair][L2][2 Nr] of rho2 and v2sph with a box of one block of
// nd complex rows x one l x up to 16 pairs
int poisson_encode_maps(PoissonArgs& a) {
  if (a.npair <= 0) { a.boxp = 0; return 0; }
  a.boxp = std::min(PS_PAIRS, a.npair);
  // 4-d view (re|im, pair, row, l) of [pair][l][row] complex: the box
  // (2, boxp, nd, 1) lands in shared memory as [row][pair][re|im]
  const cuuint64_t dims[4] = {2u, (cuuint64_t)a.npair, (cuuint64_t)a.Nr, (cuuint64_t)a.L2};
  const cuuint64_t strides[3] = {(cuuint64_t)a.L2 * a.Nr * 16, 16u, (cuuint64_t)a.Nr * 16};
  const cuuint32_t box[4] = {2u, (cuuint32_t)a.boxp, (cuuint32_t)a.nd, 1u};
  int rc = encode_f64_map(&a.tm_rho, a.rho2, 4, dims, strides, box, "Poisson rho2");
  if (!rc) rc = encode_f64_map(&a.tm_v2, a.v2sph, 4, dims, strides, box, "Poisson v2sph");
  return rc;
}

int launch_poisson_tables(const PoissonArgs& a, double* tabf, double* tabb, cudaStream_t st) {
  const int Np = (a.Nr + a.nd - 1) / a.nd * a.nd;
  const size_t n = (size_t)a.L2 * Np;
  poisson_tables_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(a, tabf, tabb);
  return (int)cudaGetLastError();
}

int launch_poisson(const PoissonArgs& a, cudaStream_t st) {
  switch (a.nd) {
    case 4: return launch_nd<4>(a, st);
    case 6: return launch_nd<6>(a, st);
    case 7: return launch_nd<7>(a, st);
    case 8: return launch_nd<8>(a, st);
    case 10: return launch_nd<10>(a, st);
    case 12: return launch_nd<12>(a, st);
    case 16: return launch_nd<16>(a, st);
    case 20: return launch_nd<20>(a, st);
    default: return (int)cudaErrorInvalidValue;
  }
}

}  // namespace td1c
