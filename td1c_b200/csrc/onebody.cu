// onebody.cu -- one-body part of the orbital RHS on the FEDVR x (l, m) basis.
//
//   h0orb(r,l,i) = sum_{r'} T_l(r,r') orb(r',l,i)           hprod_tprod.F90:152-235
//   h1orb        = length gauge  E r alpha_lm coupling      hprod_zprod.F90:108-135
//                  velocity gauge A (-i alpha)(d/dr, (l+1)/r) hprod_pzprod.F90:114-213
//   frozen core in velocity gauge also gets E r alpha_lm    hprod_htot.F90:120-122
//
// One CTA per (orbital, 32-point radial tile, chunk of 12 l channels): the
// tile of the chunk's channels and of one halo channel on each side, with a
// +-nd radial halo, is staged in shared memory by cp.async (all copies in
// flight at once), the banded kinetic (tmat) and derivative (pmat) stencils
// are applied from smem, the derivative is kept in smem, and the l <-> l+-1
// laser coupling is formed from smem -- orbitals are read from HBM once (plus
// the halos) and h0/h1 written once.  About 56 KB of smem per CTA for 21-point
// elements: four CTAs per SM.
// The band coefficients come from the (2nd+1) x nrad radk/radk0/radp tables
// (the tile's rows staged in smem with an odd pitch, so that neither the
// staging stores nor the stencil's loads conflict) plus a per-(l, r) diagonal,
// instead of the reference's (2nd+1) x Nr x L1 tmat (19 MB for Ne).  Summation
// runs over r' in ascending order like zdotu.
#include "common.cuh"
#include "kernels.cuh"

namespace td1c {

constexpr int OB_TILE = 32;          // radial points per CTA
constexpr int OB_TP = OB_TILE + 1;   // smem pitch of a band row (odd)
constexpr int OB_LC = 12;            // own l channels per CTA

__device__ __forceinline__ void ob_cp16(void* dst, const void* src, bool ok) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src),
               "r"(ok ? 16u : 0u)
               : "memory");
}
__device__ __forceinline__ void ob_cp8(void* dst, const void* src, bool ok) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src),
               "r"(ok ? 8u : 0u)
               : "memory");
}

__global__ void __launch_bounds__(256) onebody_kernel(OneBodyArgs a) {
  extern __shared__ __align__(16) double smem_d[];
  const int Nr = a.Nr, L1 = a.L1, nd = a.nd, bw = 2 * nd + 1;
  const int W = OB_TILE + 2 * nd;
  const int f = blockIdx.y;
  const int r0 = blockIdx.x * OB_TILE;
  const int l0 = blockIdx.z * OB_LC;                                      // first own channel
  const int lb = l0 > 0 ? l0 - 1 : 0, le = l0 + OB_LC + 1 < L1 ? l0 + OB_LC + 1 : L1;  // staged [lb, le)
  const int ns = le - lb;
  cplx* so = reinterpret_cast<cplx*>(smem_d);                             // [ns][W]
  cplx* sdw = so + (size_t)(OB_LC + 2) * W;                               // [ns][OB_TILE]
  double* sb = reinterpret_cast<double*>(sdw + (size_t)(OB_LC + 2) * OB_TILE);  // [3][bw][OB_TP] radk, radk0, radp
  for (int e = threadIdx.x; e < OB_TILE * bw; e += blockDim.x) {
    const int q = e / bw, jb = e % bw;
    const int ir = r0 + q + 1;
    const bool ok = ir <= Nr;
    const size_t o = ok ? (size_t)bw * ir + jb : 0;
    const int d = jb * OB_TP + q;
    ob_cp8(sb + d, a.radk + o, ok);
    ob_cp8(sb + OB_TP * bw + d, a.radk0 + o, ok);
    ob_cp8(sb + 2 * OB_TP * bw + d, a.radp + o, ok);
  }
  const int m = a.mval[f];
  const int am = m < 0 ? -m : m;
  const cplx* __restrict__ orb = a.orb + (size_t)f * L1 * Nr;
  for (int e = threadIdx.x; e < ns * W; e += blockDim.x) {
    const int ls = e / W, q = e % W;
    const int r = r0 - nd + q;
    const bool ok = r >= 0 && r < Nr;
    ob_cp16(so + e, orb + (ok ? (size_t)(lb + ls) * Nr + r : 0), ok);
  }
  asm volatile("cp.async.commit_group;" ::: "memory");
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  __syncthreads();
  const double zf = a.lfield[2];
  const double ef = a.lfield[5];
  const bool vel = a.igauge == 1;
  const bool fc = f < a.nfcore;
  cplx* __restrict__ h0 = a.h0orb + (size_t)f * L1 * Nr;
  cplx* __restrict__ h1 = a.h1orb + (size_t)f * L1 * Nr;
  // h0 of the own channels; the radial derivative of every staged channel (velocity gauge)
  for (int e = threadIdx.x; e < ns * OB_TILE; e += blockDim.x) {
    const int ls = e / OB_TILE, q = e % OB_TILE, l = lb + ls;
    const int r = r0 + q;
    if (r >= Nr) continue;
    const bool own = l >= l0 && l < l0 + OB_LC;
    if (!own && !vel) continue;
    const int ir = r + 1;  // Fortran irad
    int jll, jul;
    fedvr_row_span(ir, nd, Nr, jll, jul);  // the band is zero outside the row's element(s)
    cplx hs = mkc(0.0, 0.0), ds = mkc(0.0, 0.0);
    if (l >= am) {
      const double* rk = sb + (l == 0 ? 0 : OB_TP * bw) + q;
      const double* rp = sb + 2 * OB_TP * bw + q;
      const double td = own ? a.tdiag[(size_t)l * Nr + r] : 0.0;
      const cplx* srow = so + (size_t)ls * W + (nd + q);  // srow[k] = orb(r + k)
      for (int jr = jll; jr <= jul; ++jr) {
        int jb = nd + jr - ir;
        cplx w = srow[jr - ir];
        if (own) {
          double t = (jr == ir) ? td : rk[jb * OB_TP];
          hs.x = fma(w.x, t, hs.x); hs.y = fma(w.y, t, hs.y);
        }
        if (vel) { double p = rp[jb * OB_TP]; ds.x = fma(w.x, p, ds.x); ds.y = fma(w.y, p, ds.y); }
      }
    }
    if (own) h0[(size_t)l * Nr + r] = hs;
    sdw[(size_t)ls * OB_TILE + q] = ds;
  }
  __syncthreads();
  // laser coupling of the own channels
  for (int e = threadIdx.x; e < OB_LC * OB_TILE; e += blockDim.x) {
    const int l = l0 + e / OB_TILE, q = e % OB_TILE;
    const int r = r0 + q;
    if (r >= Nr || l >= L1) continue;
    const int ls = l - lb;
    const double x = a.xrad[r + 1];
    const double* __restrict__ al = a.alph + (size_t)(m + a.mmax1) * L1;
    const cplx* sc = so + nd + q;  // sc[ls * W] = orb(r, lb + ls)
    cplx h = mkc(0.0, 0.0);
    if (vel) {
      // iteration l-1 (as upper channel), then iteration l (as lower channel)
      if (l - 1 >= am) {
        double alp = al[l - 1];
        double t1 = -zf * alp;                         // zfield * (-i alpha): (0, t1)
        double t2 = zf * ((-alp * (double)l) / x);     // zfield * (-i alpha l / r): (0, t2)
        cplx dwv = sdw[(size_t)(ls - 1) * OB_TILE + q], wv = sc[(size_t)(ls - 1) * W];
        h.x = h.x - dwv.y * t1; h.y = h.y + dwv.x * t1;
        h.x = h.x + wv.y * t2;  h.y = h.y - wv.x * t2;
      }
      if (l >= am && l <= L1 - 2) {
        double alp = al[l];
        double t1 = -zf * alp;
        double t2 = zf * ((-alp * (double)(l + 1)) / x);
        cplx dwv = sdw[(size_t)(ls + 1) * OB_TILE + q], wv = sc[(size_t)(ls + 1) * W];
        h.x = h.x - dwv.y * t1; h.y = h.y + dwv.x * t1;
        h.x = h.x - wv.y * t2;  h.y = h.y + wv.x * t2;
      }
    }
    // length-gauge coupling: zfield for all orbitals in the length gauge,
    // efield on the frozen core in the velocity gauge
    double zz = vel ? (fc ? ef : 0.0) : zf;
    if (zz != 0.0 || !vel) {
      if (l - 1 >= am) {
        double t = zz * (x * al[l - 1]);
        cplx wv = sc[(size_t)(ls - 1) * W];
        h.x = fma(wv.x, t, h.x); h.y = fma(wv.y, t, h.y);
      }
      if (l >= am && l <= L1 - 2) {
        double t = zz * (x * al[l]);
        cplx wv = sc[(size_t)(ls + 1) * W];
        h.x = fma(wv.x, t, h.x); h.y = fma(wv.y, t, h.y);
      }
    }
    h1[(size_t)l * Nr + r] = h;
  }
}

size_t onebody_smem(int nd) {
  const int W = OB_TILE + 2 * nd;
  return sizeof(cplx) * ((size_t)(OB_LC + 2) * W + (size_t)(OB_LC + 2) * OB_TILE) +
         sizeof(double) * 3 * (size_t)OB_TP * (2 * nd + 1);
}

int launch_onebody(const OneBodyArgs& a, cudaStream_t st) {
  const size_t smem = onebody_smem(a.nd);
  if (smem > 200 * 1024) return (int)cudaErrorInvalidValue;
  static bool attr[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64 || !attr[dev]) {
    cudaError_t e = cudaFuncSetAttribute(onebody_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    if (e != cudaSuccess) return (int)e;
    if (dev >= 0 && dev < 64) attr[dev] = true;
  }
  dim3 grid((a.Nr + OB_TILE - 1) / OB_TILE, a.nfun, (a.L1 + OB_LC - 1) / OB_LC);
  onebody_kernel<<<grid, 256, smem, st>>>(a);
  return (int)cudaGetLastError();
}

}  // namespace td1c
