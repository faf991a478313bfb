// mfprod.cu -- two-electron mean-field action on the (r, theta) grid
// (hprod_mfprod2.F90:2-34 and its callees, dofc = false):
//   fcx1  gorbg_i  -= W(fc,i) orbg_fc                        (158-200)
//   dcj   gorbg_i  += [sum_{j in dc} 2 W(j,j)] orbg_i        (242-306)
//   dcx   gorbg_i  -= W(j,i) orbg_j, j in dc                 (308-366)
//   actj  v2orbg_c += [sum_{jk act} W(j,k) den1(k,j)] orbg_c  (368-437)
//   actx  v2orbg_c += sum_j wd1_j W(j,c),
//         wd1_j = -1/2 sum_{k, m_k = m_j} den1(k,j) orbg_k   (439-514)
//   act2  d2v_ij = sum_{kl} den2(j,i,l,k) W(k,l)   (i >= j, m rule, |den2| > 1e-15)
//         twfn_i += orbg_j d2v_ij,  twfn_j += orbg_i conj(d2v_ij)
//         v2orbg_k += sum_{i, m_i = m_k} rden(i,k) twfn_i     (619-694)
// W(a,b) is the stored pair (a,b) or the conjugate of the stored (b,a).
//
// act2 is organised as dense blocks: the m rule m_i + m_k = m_j + m_l pairs
// the rows ij (i >= j, m_i - m_j = d) with the columns kl (m_l - m_k = d), so
// for each d the contraction is a dense complex product over the block.  One
// thread per grid point keeps the block's d2v accumulators in registers and
// reads every W(k,l) once; the coefficients (den2, thresholded) are broadcast
// from shared memory; twfn and the orbitals of the CTA's points live in
// shared memory.
#include "common.cuh"
#include "kernels.cuh"

namespace td1c {

constexpr int MF_MAXF = 16;
constexpr int MF_NIJ = 24;   // rows of one act2 block chunk
constexpr int MF_TQ = 128;   // grid points per CTA

// coef[b.coff + kl * nij + ij] = den2(j,i,l,k), or 0 when |den2| <= thrwfn
__global__ void act2_fill_kernel(int n, const Act2Coef* __restrict__ map, const cplx* __restrict__ den2, cplx* __restrict__ coef) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  cplx d = den2[map[e].d2idx];
  bool keep = sqrt(cabs2(d)) > 1.0e-15;  // thrwfn (mod_const.F90:32)
  coef[map[e].dst] = keep ? d : mkc(0.0, 0.0);
}

__device__ __forceinline__ cplx ldW(const cplx* __restrict__ W, int p, int cj, size_t ngrid, size_t q) {
  cplx w = __ldg(W + (size_t)p * ngrid + q);
  return cj ? cconj(w) : w;
}

__global__ void __launch_bounds__(MF_TQ) mfprod_kernel(MfprodArgs a) {
  extern __shared__ double smd[];
  const int nact = a.nact, ncore = a.ncore, nfcore = a.nfcore, nfun = a.nfun;
  const int ncoef = a.ncoef;
  cplx* scoef = reinterpret_cast<cplx*>(smd);                // [ncoef]
  cplx* sphi = scoef + ncoef;                                  // [nfun][TQ]
  cplx* stw = sphi + (size_t)nfun * MF_TQ;                     // [nact][TQ]
  __shared__ cplx srden[MF_MAXF * MF_MAXF];
  __shared__ cplx sden1[MF_MAXF * MF_MAXF];
  __shared__ Act2Block sblk[32];
  __shared__ int2 srow[256];   // (ia, ja) of block rows
  __shared__ int2 scol[512];   // (pair, conj) of block columns
  const bool do_act2 = a.nelact >= 2 && nact > 0 && a.nblk > 0;
  for (int e = threadIdx.x; e < ncoef; e += blockDim.x) scoef[e] = a.coef[e];
  for (int e = threadIdx.x; e < nact * nact; e += blockDim.x) { srden[e] = a.rden[e]; sden1[e] = a.den1[e]; }
  for (int e = threadIdx.x; e < a.nblk; e += blockDim.x) sblk[e] = a.blk[e];
  for (int e = threadIdx.x; e < a.nrow; e += blockDim.x) srow[e] = a.rows[e];
  for (int e = threadIdx.x; e < a.ncol; e += blockDim.x) scol[e] = a.cols[e];
  const size_t ng = a.ngrid;
  const size_t q0 = (size_t)blockIdx.x * MF_TQ;
  const int tq = threadIdx.x;
  const size_t q = q0 + tq;
  const bool live = q < ng;
  for (int f = 0; f < nfun; ++f) sphi[(size_t)f * MF_TQ + tq] = live ? __ldg(a.orbg + (size_t)f * ng + q) : mkc(0, 0);
  for (int i = 0; i < nact; ++i) stw[(size_t)i * MF_TQ + tq] = mkc(0, 0);
  __syncthreads();
  if (!live) return;
  const cplx* __restrict__ W = a.W;
  auto PO = [&](int x, int y) { return a.pair_of[x * nfun + y]; };
  auto PC = [&](int x, int y) { return a.pair_cj[x * nfun + y]; };
  auto PHI = [&](int f) { return sphi[(size_t)f * MF_TQ + tq]; };
  const int ndcore = ncore - nfcore;
  // ---- core terms into gorbg for every dynamic orbital
  cplx dcsum = mkc(0.0, 0.0);
  for (int j = nfcore; j < ncore; ++j) { cplx w = ldW(W, PO(j, j), PC(j, j), ng, q); dcsum.x += w.x * 2.0; dcsum.y += w.y * 2.0; }
  for (int i = nfcore; i < nfun; ++i) {
    cplx g = mkc(0, 0);
    for (int j = 0; j < nfcore; ++j) {  // fcx1
      cplx w = ldW(W, PO(j, i), PC(j, i), ng, q);
      g = csub(g, cmul(w, PHI(j)));
    }
    if (ndcore > 0) {
      g = cadd(g, cmul(dcsum, PHI(i)));  // dcj
      for (int j = nfcore; j < ncore; ++j) {  // dcx
        cplx w = ldW(W, PO(j, i), PC(j, i), ng, q);
        g = csub(g, cmul(w, PHI(j)));
      }
    }
    a.gorbg[(size_t)i * ng + q] = g;
  }
  // ---- active terms into v2orbg of the dynamic cores
  for (int i = nfcore; i < ncore; ++i) a.v2orbg[(size_t)i * ng + q] = mkc(0, 0);
  if (ndcore > 0 && nact > 0) {
    cplx d2v = mkc(0.0, 0.0);
    for (int ja = 0; ja < nact; ++ja)
      for (int ka = 0; ka < nact; ++ka) {
        cplx w = ldW(W, PO(ncore + ja, ncore + ka), PC(ncore + ja, ncore + ka), ng, q);
        cfma(d2v, w, sden1[ka + nact * ja]);
      }
    for (int i = nfcore; i < ncore; ++i) {
      cplx v = a.v2orbg[(size_t)i * ng + q];
      v = cadd(v, cmul(d2v, PHI(i)));
      a.v2orbg[(size_t)i * ng + q] = v;
    }
    for (int ja = 0; ja < nact; ++ja) {
      const int jf = ncore + ja;
      cplx wd1 = mkc(0.0, 0.0);
      for (int ka = 0; ka < nact; ++ka) {
        const int kf = ncore + ka;
        if (a.mval[jf] != a.mval[kf]) continue;
        cplx dens = cscale(sden1[ka + nact * ja], -0.5);
        wd1 = cadd(wd1, cmul(PHI(kf), dens));
      }
      for (int i = nfcore; i < ncore; ++i) {
        cplx w = ldW(W, PO(jf, i), PC(jf, i), ng, q);
        cplx v = a.v2orbg[(size_t)i * ng + q];
        v = cadd(v, cmul(wd1, w));
        a.v2orbg[(size_t)i * ng + q] = v;
      }
    }
  }
  // ---- act2: dense blocks of the 2-RDM contraction
  if (do_act2) {
    cplx* tw = stw + tq;  // tw[i * TQ]
    for (int b = 0; b < a.nblk; ++b) {
      const Act2Block B = sblk[b];
      cplx acc[MF_NIJ];
#pragma unroll
      for (int r = 0; r < MF_NIJ; ++r) acc[r] = mkc(0, 0);
      for (int kl = 0; kl < B.ncol; ++kl) {
        const int2 pc = scol[B.col0 + kl];
        const cplx w = ldW(W, pc.x, pc.y, ng, q);
        const cplx* cf = scoef + B.coff + (size_t)kl * B.nrow;
#pragma unroll
        for (int r = 0; r < MF_NIJ; ++r)
          if (r < B.nrow) cfma(acc[r], cf[r], w);
      }
#pragma unroll
      for (int r = 0; r < MF_NIJ; ++r) {
        if (r < B.nrow) {
          const int2 ij = srow[B.row0 + r];
          const int ia = ij.x, ja = ij.y;
          const cplx oj = PHI(ncore + ja), oi = PHI(ncore + ia);
          tw[(size_t)ia * MF_TQ] = cadd(tw[(size_t)ia * MF_TQ], cmul(oj, acc[r]));
          if (ia > ja) tw[(size_t)ja * MF_TQ] = cadd(tw[(size_t)ja * MF_TQ], cmul(oi, cconj(acc[r])));
        }
      }
    }
    for (int ka = 0; ka < nact; ++ka) {
      const int kf = ncore + ka;
      cplx v = mkc(0, 0);
      for (int x = 0; x < nact; ++x)
        if (a.mval[ncore + x] == a.mval[kf]) v = cadd(v, cmul(srden[x + nact * ka], tw[(size_t)x * MF_TQ]));
      a.v2orbg[(size_t)kf * ng + q] = v;
    }
  } else {
    for (int ka = 0; ka < nact; ++ka) a.v2orbg[(size_t)(ncore + ka) * ng + q] = mkc(0, 0);
  }
}

int launch_mfprod(const MfprodArgs& a, cudaStream_t st) {
  if (a.nfun > MF_MAXF || a.nblk > 32 || a.nrow > 256 || a.ncol > 512) return (int)cudaErrorInvalidValue;
  const bool do_act2 = a.nelact >= 2 && a.nact > 0 && a.nblk > 0;
  if (do_act2) act2_fill_kernel<<<(a.ncoef + 127) / 128, 128, 0, st>>>(a.ncoef, a.coef_map, a.den2, a.coef);
  size_t smem = sizeof(cplx) * ((size_t)a.ncoef + (size_t)a.nfun * MF_TQ + (size_t)a.nact * MF_TQ);
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(mfprod_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024);
    attr = true;
  }
  if (smem > 160 * 1024) return (int)cudaErrorInvalidValue;
  mfprod_kernel<<<(unsigned)((a.ngrid + MF_TQ - 1) / MF_TQ), MF_TQ, smem, st>>>(a);
  return (int)cudaGetLastError();
}

}  // namespace td1c
