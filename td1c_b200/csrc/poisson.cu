// poisson.cu -- multipole radial Poisson solve (hprod_mkv2mf.F90:118-182).
//
// For every stored orbital pair p and multipole l >= |m_p| the reference
// splits rho2(:, l, p) into real and imaginary parts, forms
//     t   = sum_r rho(r) r^l / (2 pi) / r_max^(2l+1)
//     rhs = rho(r) (2l+1) / (2 pi r sqrt(w_r))
// solves  L_l L_l^T x = rhs  with the dpbtrf factor of
// [l(l+1)/r^2 + 2 T] (band nd) by dpbtrs, and returns
//     v2sph = (x + t r^(l+1) sqrt(w_r)) 4 pi / ((2l+1) r sqrt(w_r)).
// Here one CTA owns one l: the band factor of that l is staged in shared
// memory (Nr x (nd+1) doubles, 201 KB for Ne) and every thread runs the
// forward and back substitution of one (pair, re|im) right-hand side, with
// the last nd solution values held in registers (nd is a template
// parameter) so each step is nd FMAs from smem broadcasts.  The diagonal is
// applied as a multiply by its reciprocal.
#include "common.cuh"
#include "kernels.cuh"

namespace td1c {

template <int ND>
__global__ void __launch_bounds__(128) poisson_kernel(PoissonArgs a) {
  extern __shared__ double sL[];  // [Nr][ND+1]
  const int l = blockIdx.x;
  const int Nr = a.Nr;
  const double* __restrict__ gL = a.d2ll + (size_t)l * Nr * (ND + 1);
  for (int e = threadIdx.x; e < Nr * (ND + 1); e += blockDim.x) sL[e] = gL[e];
  __syncthreads();
  const int nsys = 2 * a.npair;
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
    const double* __restrict__ rpl0 = a.rpl0 + (size_t)l * Nr;
    const double* __restrict__ invr = a.invr + (size_t)l * Nr;
    const double* __restrict__ rinv = a.d2rinv + (size_t)l * Nr;
    double t = 0.0;
    double win[ND];
#pragma unroll
    for (int k = 0; k < ND; ++k) win[k] = 0.0;
    // forward substitution  L y = rhs  (y stored into out)
    for (int jb = 0; jb < Nr; jb += ND) {
#pragma unroll
      for (int u = 0; u < ND; ++u) {
        const int j = jb + u;
        if (j < Nr) {
          double rho = in[2 * j];
          t = fma(rho, __ldg(rpl0 + j), t);
          double sacc = rho * __ldg(invr + j);
#pragma unroll
          for (int k = ND; k >= 1; --k) {  // oldest first, as dtbsv's column sweep
            // L(j, j-k) = ab[k + (ND+1)(j-k)], y_{j-k} in win[(u-k) mod ND]
            if (j - k >= 0) sacc = fma(-sL[k + (ND + 1) * (j - k)], win[(u - k + ND) % ND], sacc);
          }
          double y = sacc * __ldg(rinv + j);
          win[u] = y;
          out[2 * j] = y;
        }
      }
    }
    // back substitution  L^T x = y
#pragma unroll
    for (int k = 0; k < ND; ++k) win[k] = 0.0;
    const int nb = (Nr + ND - 1) / ND;
    for (int b = nb - 1; b >= 0; --b) {
#pragma unroll
      for (int u = ND - 1; u >= 0; --u) {
        const int j = b * ND + u;
        if (j < Nr) {
          double sacc = out[2 * j];
#pragma unroll
          for (int k = ND; k >= 1; --k) {  // farthest first, as dtbsv('T')
            // L(j+k, j) = ab[k + (ND+1) j], x_{j+k} in win[(u+k) mod ND]
            if (j + k < Nr) sacc = fma(-sL[k + (ND + 1) * j], win[(u + k) % ND], sacc);
          }
          double x = sacc * __ldg(rinv + j);
          win[u] = x;
          out[2 * j] = x;
        }
      }
    }
    // homogeneous boundary term and scaling
    t *= a.fac1[l];
    const double* __restrict__ rpl1 = a.rpl1 + (size_t)l * Nr;
    const double* __restrict__ fac2 = a.fac2 + (size_t)l * Nr;
    for (int r = 0; r < Nr; ++r) out[2 * r] = fma(t, __ldg(rpl1 + r), out[2 * r]) * __ldg(fac2 + r);
  }
}

template <int ND>
static int launch_nd(const PoissonArgs& a, size_t smem, cudaStream_t st) {
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(poisson_kernel<ND>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    attr = true;
  }
  int nsys = 2 * a.npair;
  int ysplit = (nsys + 127) / 128;
  dim3 grid(a.L2, ysplit);
  poisson_kernel<ND><<<grid, 128, smem, st>>>(a);
  return (int)cudaGetLastError();
}

int launch_poisson(const PoissonArgs& a, size_t smem, cudaStream_t st) {
  switch (a.nd) {
    case 4: return launch_nd<4>(a, smem, st);
    case 6: return launch_nd<6>(a, smem, st);
    case 7: return launch_nd<7>(a, smem, st);
    case 8: return launch_nd<8>(a, smem, st);
    case 10: return launch_nd<10>(a, smem, st);
    case 12: return launch_nd<12>(a, smem, st);
    case 16: return launch_nd<16>(a, smem, st);
    case 20: return launch_nd<20>(a, smem, st);
    case 22: return launch_nd<22>(a, smem, st);
    default: return (int)cudaErrorInvalidValue;
  }
}

}  // namespace td1c
