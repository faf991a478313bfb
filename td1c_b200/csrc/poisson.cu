// poisson.cu -- multipole radial Poisson solve (hprod_mkv2mf.F90:118-182).
//
// For every stored orbital pair p and multipole l >= |m_p| the reference
// splits rho2(:, l, p) into real and imaginary parts, forms
//     t   = sum_r rho(r) r^l / (2 pi) / r_max^(2l+1)
//     rhs = rho(r) (2l+1) / (2 pi r sqrt(w_r))
// solves  L_l L_l^T x = rhs  with the dpbtrf factor of
// [l(l+1)/r^2 + 2 T] (band nd) by dpbtrs, and returns
//     v2sph = (x + t r^(l+1) sqrt(w_r)) 4 pi / ((2l+1) r sqrt(w_r)).
// One CTA owns one l.  Shared memory holds that l's band factor with the
// diagonal replaced by its reciprocal (Nr x (nd+1) doubles, 201 KB for Ne)
// plus the r^l/(2 pi) and (2l+1)/(2 pi r sqrt w) columns; every thread runs
// the forward and back substitution of one (pair, re|im) right-hand side.
// The substitution is sequential in r, so the kernel is latency-bound: the
// last nd solution values live in registers (nd is a template parameter),
// the terms are summed oldest-first as dtbsv does so only the newest value
// sits on the critical path, and each block of nd inputs is loaded one block
// ahead (register double buffer) so no global access waits inside the chain.
#include "common.cuh"
#include "kernels.cuh"

namespace td1c {

template <int ND>
__global__ void __launch_bounds__(128) poisson_kernel(PoissonArgs a) {
  extern __shared__ double sm[];
  const int l = blockIdx.x;
  const int Nr = a.Nr;
  double* sL = sm;                          // [Nr][ND+1], sL[(ND+1) j] = 1 / L(j,j)
  double* s0 = sm + (size_t)Nr * (ND + 1);  // [Nr] r^l / (2 pi)
  double* sI = s0 + Nr;                     // [Nr] (2l+1) / (2 pi r sqrt w)
  const double* __restrict__ gL = a.d2ll + (size_t)l * Nr * (ND + 1);
  for (int e = threadIdx.x; e < Nr * (ND + 1); e += blockDim.x) sL[e] = gL[e];
  __syncthreads();
  for (int j = threadIdx.x; j < Nr; j += blockDim.x) {
    sL[(size_t)(ND + 1) * j] = a.d2rinv[(size_t)l * Nr + j];
    s0[j] = a.rpl0[(size_t)l * Nr + j];
    sI[j] = a.invr[(size_t)l * Nr + j];
  }
  __syncthreads();
  const int nsys = 2 * a.npair;
  const int nb = (Nr + ND - 1) / ND;
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
    for (int k = 0; k < ND; ++k) { win[k] = 0.0; cur[k] = (k < Nr) ? __ldg(in + 2 * k) : 0.0; }
    // forward substitution  L y = rhs  (y stored into out)
    for (int b = 0; b < nb; ++b) {
      const int jb = b * ND;
#pragma unroll
      for (int u = 0; u < ND; ++u) { const int jn = jb + ND + u; nxt[u] = (jn < Nr) ? __ldg(in + 2 * jn) : 0.0; }
#pragma unroll
      for (int u = 0; u < ND; ++u) {
        const int j = jb + u;
        if (j < Nr) {
          const double rho = cur[u];
          t = fma(rho, s0[j], t);
          double sacc = rho * sI[j];
          const double* Lr = sL + (size_t)(ND + 1) * j;
#pragma unroll
          for (int k = ND; k >= 1; --k) {  // oldest first, as dtbsv's column sweep
            // L(j, j-k) = ab[k + (ND+1)(j-k)] = Lr[k - (ND+1) k] ; y_{j-k} in win[(u-k) mod ND]
            if (j - k >= 0) sacc = fma(-Lr[k - (ND + 1) * k], win[(u - k + ND) % ND], sacc);
          }
          const double y = sacc * Lr[0];
          win[u] = y;
          out[2 * j] = y;
        }
      }
#pragma unroll
      for (int u = 0; u < ND; ++u) cur[u] = nxt[u];
    }
    // back substitution  L^T x = y  (reads back the thread's own forward values)
#pragma unroll
    for (int k = 0; k < ND; ++k) win[k] = 0.0;
    {
      const int jb = (nb - 1) * ND;
#pragma unroll
      for (int u = 0; u < ND; ++u) cur[u] = (jb + u < Nr) ? out[2 * (jb + u)] : 0.0;
    }
    for (int b = nb - 1; b >= 0; --b) {
      const int jb = b * ND;
      if (b > 0) {
#pragma unroll
        for (int u = 0; u < ND; ++u) nxt[u] = out[2 * (jb - ND + u)];
      }
#pragma unroll
      for (int u = ND - 1; u >= 0; --u) {
        const int j = jb + u;
        if (j < Nr) {
          double sacc = cur[u];
          const double* Lc = sL + (size_t)(ND + 1) * j;
#pragma unroll
          for (int k = ND; k >= 1; --k) {  // farthest first, as dtbsv('T')
            // L(j+k, j) = ab[k + (ND+1) j] = Lc[k] ; x_{j+k} in win[(u+k) mod ND]
            if (j + k < Nr) sacc = fma(-Lc[k], win[(u + k) % ND], sacc);
          }
          const double x = sacc * Lc[0];
          win[u] = x;
          out[2 * j] = x;
        }
      }
      if (b > 0) {
#pragma unroll
        for (int u = 0; u < ND; ++u) cur[u] = nxt[u];
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
static int launch_nd(const PoissonArgs& a, cudaStream_t st) {
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(poisson_kernel<ND>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    attr = true;
  }
  const size_t smem = sizeof(double) * ((size_t)a.Nr * (ND + 1) + 2 * (size_t)a.Nr);
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
