// onebody.cu -- one-body part of the orbital RHS on the FEDVR x (l, m) basis.
//
//   h0orb(r,l,i) = sum_{r'} T_l(r,r') orb(r',l,i)           hprod_tprod.F90:152-235
//   h1orb        = length gauge  E r alpha_lm coupling      hprod_zprod.F90:108-135
//                  velocity gauge A (-i alpha)(d/dr, (l+1)/r) hprod_pzprod.F90:114-213
//   frozen core in velocity gauge also gets E r alpha_lm    hprod_htot.F90:120-122
//
// One CTA per (orbital, 32-point radial tile): the tile of every l channel
// plus a +-nd halo is staged in shared memory once, the banded kinetic
// (tmat) and derivative (pmat) stencils are applied to all l channels from
// smem, the derivative is kept in smem, and the l <-> l+-1 laser coupling is
// formed from smem -- orbitals are read from HBM once and h0/h1 written once.
// The band coefficients come from the (2nd+1) x nrad radk/radk0/radp tables
// (the tile's rows staged in smem) plus a per-(l, r) diagonal, instead of the
// reference's (2nd+1) x Nr x L1 tmat (19 MB for Ne).  Summation runs over r'
// in ascending order like zdotu.
#include "common.cuh"
#include "kernels.cuh"

namespace td1c {

constexpr int OB_TILE = 32;

__global__ void __launch_bounds__(256) onebody_kernel(OneBodyArgs a) {
  extern __shared__ double smem_d[];
  const int Nr = a.Nr, L1 = a.L1, nd = a.nd, bw = 2 * nd + 1;
  const int W = OB_TILE + 2 * nd;
  cplx* so = reinterpret_cast<cplx*>(smem_d);  // [L1][W]
  cplx* sdw = so + (size_t)L1 * W;             // [L1][OB_TILE]
  double* sb = reinterpret_cast<double*>(sdw + (size_t)L1 * OB_TILE);  // [3][bw][OB_TILE] radk, radk0, radp rows
  const int f = blockIdx.y;
  const int r0 = blockIdx.x * OB_TILE;
  for (int e = threadIdx.x; e < OB_TILE * bw; e += blockDim.x) {
    const int q = e / bw, jb = e % bw;
    const int ir = r0 + q + 1;
    double k0 = 0.0, k1 = 0.0, pp = 0.0;
    if (ir <= Nr) {
      const size_t o = (size_t)bw * ir + jb;
      k0 = a.radk[o]; k1 = a.radk0[o]; pp = a.radp[o];
    }
    const int d = jb * OB_TILE + q;  // band index major: lanes (q) hit consecutive banks
    sb[d] = k0; sb[OB_TILE * bw + d] = k1; sb[2 * OB_TILE * bw + d] = pp;
  }
  const int m = a.mval[f];
  const int am = m < 0 ? -m : m;
  const cplx* __restrict__ orb = a.orb + (size_t)f * L1 * Nr;
  // stage
  for (int e = threadIdx.x; e < L1 * W; e += blockDim.x) {
    int l = e / W, q = e % W;
    int r = r0 - nd + q;
    so[e] = (r >= 0 && r < Nr) ? orb[(size_t)l * Nr + r] : mkc(0.0, 0.0);
  }
  __syncthreads();
  const double zf = a.lfield[2];
  const double ef = a.lfield[5];
  const bool vel = a.igauge == 1;
  const bool fc = f < a.nfcore;
  cplx* __restrict__ h0 = a.h0orb + (size_t)f * L1 * Nr;
  cplx* __restrict__ h1 = a.h1orb + (size_t)f * L1 * Nr;
  // h0 and radial derivative
  for (int e = threadIdx.x; e < L1 * OB_TILE; e += blockDim.x) {
    int l = e / OB_TILE, q = e % OB_TILE;
    int r = r0 + q;
    if (r >= Nr) continue;
    const int ir = r + 1;  // Fortran irad
    int jll, jul;
    fedvr_row_span(ir, nd, Nr, jll, jul);  // the band is zero outside the row's element(s)
    cplx hs = mkc(0.0, 0.0), ds = mkc(0.0, 0.0);
    if (l >= am) {
      const double* rk = sb + (l == 0 ? 0 : OB_TILE * bw) + q;
      const double* rp = sb + 2 * OB_TILE * bw + q;
      const double td = a.tdiag[(size_t)l * Nr + r];
      const cplx* srow = so + (size_t)l * W + (nd + q);  // srow[k] = orb(r + k)
      for (int jr = jll; jr <= jul; ++jr) {
        int jb = nd + jr - ir;
        cplx w = srow[jr - ir];
        double t = (jr == ir) ? td : rk[jb * OB_TILE];
        hs.x = fma(w.x, t, hs.x); hs.y = fma(w.y, t, hs.y);
        if (vel) { double p = rp[jb * OB_TILE]; ds.x = fma(w.x, p, ds.x); ds.y = fma(w.y, p, ds.y); }
      }
    }
    h0[(size_t)l * Nr + r] = hs;
    sdw[(size_t)l * OB_TILE + q] = ds;
  }
  __syncthreads();
  // laser coupling
  for (int e = threadIdx.x; e < L1 * OB_TILE; e += blockDim.x) {
    int l = e / OB_TILE, q = e % OB_TILE;
    int r = r0 + q;
    if (r >= Nr) continue;
    const double x = a.xrad[r + 1];
    const double* __restrict__ al = a.alph + (size_t)(m + a.mmax1) * L1;
    const cplx* sc = so + nd + q;  // sc[l * W] = orb(r, l)
    cplx h = mkc(0.0, 0.0);
    if (vel) {
      // iteration l-1 (as upper channel), then iteration l (as lower channel)
      if (l - 1 >= am) {
        double alp = al[l - 1];
        double t1 = -zf * alp;                         // zfield * (-i alpha): (0, t1)
        double t2 = zf * ((-alp * (double)l) / x);     // zfield * (-i alpha l / r): (0, t2)
        cplx dwv = sdw[(size_t)(l - 1) * OB_TILE + q], wv = sc[(size_t)(l - 1) * W];
        h.x = h.x - dwv.y * t1; h.y = h.y + dwv.x * t1;
        h.x = h.x + wv.y * t2;  h.y = h.y - wv.x * t2;
      }
      if (l >= am && l <= L1 - 2) {
        double alp = al[l];
        double t1 = -zf * alp;
        double t2 = zf * ((-alp * (double)(l + 1)) / x);
        cplx dwv = sdw[(size_t)(l + 1) * OB_TILE + q], wv = sc[(size_t)(l + 1) * W];
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
        cplx wv = sc[(size_t)(l - 1) * W];
        h.x = fma(wv.x, t, h.x); h.y = fma(wv.y, t, h.y);
      }
      if (l >= am && l <= L1 - 2) {
        double t = zz * (x * al[l]);
        cplx wv = sc[(size_t)(l + 1) * W];
        h.x = fma(wv.x, t, h.x); h.y = fma(wv.y, t, h.y);
      }
    }
    h1[(size_t)l * Nr + r] = h;
  }
}

int launch_onebody(const OneBodyArgs& a, cudaStream_t st) {
  const int W = OB_TILE + 2 * a.nd;
  size_t smem = sizeof(cplx) * ((size_t)a.L1 * W + (size_t)a.L1 * OB_TILE) + sizeof(double) * 3 * OB_TILE * (2 * a.nd + 1);
  static bool attr_set = false;
  if (!attr_set) {
    cudaFuncSetAttribute(onebody_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    attr_set = true;
  }
  dim3 grid((a.Nr + OB_TILE - 1) / OB_TILE, a.nfun);
  onebody_kernel<<<grid, 256, smem, st>>>(a);
  return (int)cudaGetLastError();
}

}  // namespace td1c
