// poisson.cu -- multipole radial Poisson solve (hprod_mkv2mf.F90:118-182).
//
// For every stored orbital pair p and multipole l >= |m_p| the reference
// splits rho2(:, l, p) into real and imaginary parts, forms
//     t   = sum_r rho(r) r^l / (2 pi) / r_max^(2l+1)
//     rhs = rho(r) (2l+1) / (2 pi r sqrt(w_r))
// solves  L_l L_l^T x = rhs  with the dpbtrf factor of
// [l(l+1)/r^2 + 2 T] (band nd) by dpbtrs, and returns
//     v2sph = (x + t r^(l+1) sqrt(w_r)) 4 pi / ((2l+1) r sqrt(w_r)).
// One CTA owns one l; every thread runs the forward and back substitution of
// one (pair, re|im) right-hand side.  The substitution is sequential in r and
// the SM holds only a few warps, so the loop is written to be branch-free:
// shared memory holds the l's band factor (diagonal replaced by its
// reciprocal) framed by nd zero rows on each side and identity rows that
// round Nr up to a multiple of nd, so no step needs a bounds test; the last
// nd solution values live in registers (nd is a template parameter); the
// band terms of older values are summed (oldest first, as dtbsv) into four
// independent partial sums so only the newest value's FMA and the
// reciprocal multiply sit on the recurrence; inputs and the final scaling
// columns are loaded one block of nd rows ahead.  The homogeneous boundary
// term and the final scaling are fused into the back substitution.
#include "common.cuh"
#include "kernels.cuh"

namespace td1c {

template <int ND>
__global__ void __launch_bounds__(128) poisson_kernel(PoissonArgs a) {
  extern __shared__ double sm[];
  const int l = blockIdx.x;
  const int Nr = a.Nr;
  const int nb = (Nr + ND - 1) / ND;
  const int Np = nb * ND;                          // padded rows
  constexpr int LD = ND + 1;
  double* sL = sm + (size_t)ND * LD;               // row j at sL + LD j, rows -ND .. Np+ND-1
  double* s0 = sm + (size_t)(Np + 2 * ND) * LD;    // [Np] r^l / (2 pi)
  double* sI = s0 + Np;                            // [Np] (2l+1) / (2 pi r sqrt w)
  const double* __restrict__ gL = a.d2ll + (size_t)l * Nr * LD;
  for (int e = threadIdx.x; e < (Np + 2 * ND) * LD; e += blockDim.x) {
    const int row = e / LD - ND, k = e % LD;
    double v = 0.0;
    if (row >= 0 && row < Nr) v = (k == 0) ? a.d2rinv[(size_t)l * Nr + row] : gL[(size_t)row * LD + k];
    else if (row >= Nr && row < Np && k == 0) v = 1.0;  // identity padding rows
    sm[e] = v;
  }
  for (int j = threadIdx.x; j < Np; j += blockDim.x) {
    s0[j] = j < Nr ? a.rpl0[(size_t)l * Nr + j] : 0.0;
    sI[j] = j < Nr ? a.invr[(size_t)l * Nr + j] : 0.0;
  }
  __syncthreads();
  const int nsys = 2 * a.npair;
  const double fac1 = a.fac1[l];
  const double* __restrict__ rpl1 = a.rpl1 + (size_t)l * Nr;
  const double* __restrict__ fac2 = a.fac2 + (size_t)l * Nr;
  for (int s = threadIdx.x + blockIdx.y * blockDim.x; s < nsys; s += blockDim.x * gridDim.y) {
    const int p = s >> 1, c = s & 1;
    const int m = a.pair_m[p];
    const int am = m < 0 ? -m : m;
    double* __restrict__ out = reinterpret_cast<double*>(a.v2sph + ((size_t)p * a.L2 + l) * Nr) + c;
    if (l < am) {
      for (int r = 0; r < Nr; ++r) out[2 * r] = 0.0;
      continue;
    }
    const double* __restrict__ in = reinterpret_cast<const double*>(a.rho2 + ((size_t)p * a.L2 + l) * Nr) + c;
    double t = 0.0;
    double win[ND], cur[ND], nxt[ND];
#pragma unroll
    for (int k = 0; k < ND; ++k) { win[k] = 0.0; cur[k] = __ldg(in + 2 * min(k, Nr - 1)); }
    // ---- forward substitution  L y = rhs  (y kept in out for the back pass)
    for (int b = 0; b < nb; ++b) {
      const int jb = b * ND;
#pragma unroll
      for (int u = 0; u < ND; ++u) nxt[u] = __ldg(in + 2 * min(jb + ND + u, Nr - 1));
#pragma unroll
      for (int u = 0; u < ND; ++u) {
        const int j = jb + u;
        const double rho = cur[u];
        t = fma(rho, s0[j], t);
        const double* Lr = sL + (size_t)LD * j;
        // L(j, j-k) = ab[k + LD (j-k)] = Lr[-ND k]; y_{j-k} in win[(u-k) mod ND]
        double pa = rho * sI[j], pb = 0.0, pc = 0.0, pd = 0.0;
#pragma unroll
        for (int k = ND; k >= 2; --k) {
          const double term = Lr[-ND * k] * win[(u - k + ND) % ND];
          const int g = (ND - k) & 3;
          if (g == 0) pa -= term; else if (g == 1) pb -= term; else if (g == 2) pc -= term; else pd -= term;
        }
        const double sacc = fma(-Lr[-ND], win[(u - 1 + ND) % ND], (pa + pb) + (pc + pd));
        const double y = sacc * Lr[0];
        win[u] = y;
        if (j < Nr) out[2 * j] = y;
      }
#pragma unroll
      for (int u = 0; u < ND; ++u) cur[u] = nxt[u];
    }
    // ---- back substitution  L^T x = y  fused with the boundary term and scaling
    //      v2sph = (x + t fac1 r^(l+1) sqrt(w)) 4 pi / ((2l+1) r sqrt(w))
    t *= fac1;
    double c1[ND], c2[ND], n1[ND], n2[ND];
#pragma unroll
    for (int k = 0; k < ND; ++k) win[k] = 0.0;
    {
      const int jb = (nb - 1) * ND;
#pragma unroll
      for (int u = 0; u < ND; ++u) {
        const int jj = min(jb + u, Nr - 1);
        cur[u] = (jb + u < Nr) ? out[2 * jj] : 0.0;
        c1[u] = __ldg(rpl1 + jj); c2[u] = __ldg(fac2 + jj);
      }
    }
    for (int b = nb - 1; b >= 0; --b) {
      const int jb = b * ND;
      if (b > 0) {
#pragma unroll
        for (int u = 0; u < ND; ++u) {
          const int jj = jb - ND + u;
          nxt[u] = out[2 * jj]; n1[u] = __ldg(rpl1 + jj); n2[u] = __ldg(fac2 + jj);
        }
      }
#pragma unroll
      for (int u = ND - 1; u >= 0; --u) {
        const int j = jb + u;
        const double* Lc = sL + (size_t)LD * j;
        // L(j+k, j) = ab[k + LD j] = Lc[k]; x_{j+k} in win[(u+k) mod ND]; farthest first
        double pa = cur[u], pb = 0.0, pc = 0.0, pd = 0.0;
#pragma unroll
        for (int k = ND; k >= 2; --k) {
          const double term = Lc[k] * win[(u + k) % ND];
          const int g = (ND - k) & 3;
          if (g == 0) pa -= term; else if (g == 1) pb -= term; else if (g == 2) pc -= term; else pd -= term;
        }
        const double sacc = fma(-Lc[1], win[(u + 1) % ND], (pa + pb) + (pc + pd));
        const double x = sacc * Lc[0];
        win[u] = x;
        if (j < Nr) out[2 * j] = fma(t, c1[u], x) * c2[u];
      }
      if (b > 0) {
#pragma unroll
        for (int u = 0; u < ND; ++u) { cur[u] = nxt[u]; c1[u] = n1[u]; c2[u] = n2[u]; }
      }
    }
  }
}

template <int ND>
static int launch_nd(const PoissonArgs& a, cudaStream_t st) {
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(poisson_kernel<ND>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    attr = true;
  }
  const int Np = (a.Nr + ND - 1) / ND * ND;
  const size_t smem = sizeof(double) * ((size_t)(Np + 2 * ND) * (ND + 1) + 2 * (size_t)Np);
  if (smem > 227 * 1024) return (int)cudaErrorInvalidValue;
  int nsys = 2 * a.npair;
  int ysplit = (nsys + 127) / 128;
  dim3 grid(a.L2, ysplit);
  poisson_kernel<ND><<<grid, 128, smem, st>>>(a);
  return (int)cudaGetLastError();
}

int launch_poisson(const PoissonArgs& a, size_t, cudaStream_t st) {
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
