// observables.cu -- state-level operations outside the RHS: the length-form
// dipole and the orthonormalisation used by imaginary-time relaxation.
//
// Dipole <z> of the state (hprod_dipole.F90:2-70,
// dip(1) = Re hprod_trace1(den1, orb, z orb); dip(2) = 0 for the length form).
//
//   (z phi_j)(r, l) = x_r [alpha(l-1, m) phi_j(r, l-1) + alpha(l, m) phi_j(r, l+1)]
//                     (hprod_zprod with unit field, hprod_zprod.F90:108-135)
//   <z> = Re [ 2 sum_{core f} <phi_f|z phi_f> + sum_{ia, ja, m_i = m_j} <phi_i|z phi_j> den1(ja, ia) ]
//                     (hprod_trace1.F90:2-88)
// The matrix elements are accumulated per radial chunk (fixed order) and
// combined with the 1-RDM in one finishing thread block, so the value does
// not depend on scheduling.
#include "common.cuh"
#include "kernels.cuh"

namespace td1c {

constexpr int DIP_CHUNK = 64;  // radial points per CTA

// partial[chunk][e] = sum over the chunk's r and all l of conj(phi_i) (P phi_j), with P
// z (mode 0: hprod_zprod), the acceleration operator (mode 1: hprod_azprod,
// hprod_azprod.F90:100-135, the same l +- 1 coupling with bas_azfac = -alph Z / r^2
// in place of r alph, bas_gen_azfac.F90:68-72) or P phi given (mode 2)
__global__ void __launch_bounds__(256) dipole_partial_kernel(DipoleArgs a) {
  const int r0 = blockIdx.x * DIP_CHUNK;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int e = warp; e < a.nent; e += nw) {
    const int2 ij = a.ent[e];
    const int i = ij.x, j = ij.y, m = a.mval[j];
    const int am = m < 0 ? -m : m;
    const double* al = a.alph + (size_t)(m + a.mmax1) * a.L1;
    const cplx* pi = a.wfn + (size_t)i * a.L1 * a.Nr;
    const cplx* pj = a.wfn + (size_t)j * a.L1 * a.Nr;
    const cplx* vj = a.pv ? a.pv + (size_t)j * a.L1 * a.Nr : nullptr;
    cplx s = mkc(0, 0);
    for (int q = lane; q < DIP_CHUNK * a.L1; q += 32) {
      const int l = q / DIP_CHUNK, r = r0 + q % DIP_CHUNK;
      if (r >= a.Nr || l < am) continue;
      cplx zp = mkc(0, 0);
      if (a.mode == 2) {
        zp = vj[(size_t)l * a.Nr + r];
      } else {
        const double x = a.xrad[r + 1];
        const double g = a.mode == 1 ? -a.znuc / (x * x) : x;
        if (l - 1 >= am) { const cplx w = pj[(size_t)(l - 1) * a.Nr + r]; const double t = g * al[l - 1]; zp.x = fma(w.x, t, zp.x); zp.y = fma(w.y, t, zp.y); }
        if (l + 1 < a.L1) { const cplx w = pj[(size_t)(l + 1) * a.Nr + r]; const double t = g * al[l]; zp.x = fma(w.x, t, zp.x); zp.y = fma(w.y, t, zp.y); }
      }
      s = cadd(s, cmulc(pi[(size_t)l * a.Nr + r], zp));
    }
    for (int o = 16; o > 0; o >>= 1) { s.x += __shfl_xor_sync(0xffffffffu, s.x, o); s.y += __shfl_xor_sync(0xffffffffu, s.y, o); }
    if (lane == 0) a.partial[(size_t)blockIdx.x * a.nent + e] = s;
  }
}

// sum the chunks of every entry in order, weight them and add
__global__ void dipole_finish_kernel(DipoleArgs a, int nchunk) {
  __shared__ double red[256];
  double part = 0.0;
  for (int e = threadIdx.x; e < a.nent; e += blockDim.x) {
    cplx s = mkc(0, 0);
    for (int c = 0; c < nchunk; ++c) s = cadd(s, a.partial[(size_t)c * a.nent + e]);
    const int2 ij = a.ent[e];
    if (ij.x < a.ncore) {
      part += 2.0 * s.x;  // core orbital, doubly occupied (i == j)
    } else {
      const int ia = ij.x - a.ncore, ja = ij.y - a.ncore;
      part += cmul(s, a.den1[ja + a.nact * ia]).x;  // den1(ja, ia)
    }
  }
  red[threadIdx.x] = part;
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st) red[threadIdx.x] += red[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0) a.out[0] = red[0];
}

int launch_dipole(const DipoleArgs& a, cudaStream_t st) {
  const int nchunk = (a.Nr + DIP_CHUNK - 1) / DIP_CHUNK;
  if (a.nent <= 0) return (int)cudaMemsetAsync(a.out, 0, sizeof(double), st);
  dipole_partial_kernel<<<nchunk, 256, 0, st>>>(a);
  dipole_finish_kernel<<<1, 256, 0, st>>>(a, nchunk);
  return (int)cudaGetLastError();
}

int dipole_partial_size(int Nr, int nent) { return ((Nr + DIP_CHUNK - 1) / DIP_CHUNK) * nent; }

// ---------------------------------------------------------------------------
// wfn_orth_cic + wfn_orth_orb (wfn_orth.F90:2-29, 31-110; fedvr_normalized,
// ecs_flag = 0): normalise the CI vector; then modified Gram-Schmidt of every
// non-frozen orbital against all earlier orbitals of equal m (each overlap
// with the already projected orbital), then normalisation, over l >= |m|.
// One CTA; every sum is a fixed-order block reduction.
// ---------------------------------------------------------------------------
constexpr int ORTH_NT = 1024;

__device__ cplx orth_block_sum(cplx v, cplx* red) {
  const int tid = threadIdx.x;
  red[tid] = v;
  __syncthreads();
  for (int st = ORTH_NT / 2; st > 0; st >>= 1) {
    if (tid < st) red[tid] = cadd(red[tid], red[tid + st]);
    __syncthreads();
  }
  const cplx r = red[0];
  __syncthreads();
  return r;
}

__global__ void __launch_bounds__(ORTH_NT) orth_kernel(int Nr, int L1, int nfun, int nfcore, int lcic,
                                                       const int* __restrict__ mval, cplx* wfn, cplx* cic) {
  __shared__ cplx red[ORTH_NT];
  const int tid = threadIdx.x;
  cplx s = mkc(0, 0);
  for (int d = tid; d < lcic; d += ORTH_NT) s.x += cabs2(cic[d]);
  const double cn = 1.0 / sqrt(orth_block_sum(s, red).x);
  for (int d = tid; d < lcic; d += ORTH_NT) cic[d] = cscale(cic[d], cn);
  for (int i = nfcore; i < nfun; ++i) {
    const int mi = mval[i], l0 = mi < 0 ? -mi : mi;
    cplx* pi = wfn + (size_t)i * L1 * Nr;
    const int n = (L1 - l0) * Nr;  // the l >= |m| rows are contiguous
    for (int j = 0; j < i; ++j) {
      if (mval[j] != mi) continue;
      const cplx* pj = wfn + (size_t)j * L1 * Nr;
      cplx ov = mkc(0, 0);
      for (int e = tid; e < n; e += ORTH_NT) ov = cadd(ov, cmulc(pj[(size_t)l0 * Nr + e], pi[(size_t)l0 * Nr + e]));
      ov = orth_block_sum(ov, red);
      for (int e = tid; e < n; e += ORTH_NT) pi[(size_t)l0 * Nr + e] = csub(pi[(size_t)l0 * Nr + e], cmul(pj[(size_t)l0 * Nr + e], ov));
      __syncthreads();
    }
    cplx nr = mkc(0, 0);
    for (int e = tid; e < n; e += ORTH_NT) nr.x += cabs2(pi[(size_t)l0 * Nr + e]);
    const double inv = 1.0 / sqrt(orth_block_sum(nr, red).x);
    for (int e = tid; e < n; e += ORTH_NT) pi[(size_t)l0 * Nr + e] = cscale(pi[(size_t)l0 * Nr + e], inv);
    __syncthreads();
  }
}

int launch_orth(int Nr, int L1, int nfun, int nfcore, int lcic, const int* mval, cplx* wfn, cplx* cic, cudaStream_t st) {
  orth_kernel<<<1, ORTH_NT, 0, st>>>(Nr, L1, nfun, nfcore, lcic, mval, wfn, cic);
  return (int)cudaGetLastError();
}

}  // namespace td1c
