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
// One thread per grid point; the 2-RDM coefficients are compacted once per
// RHS into a (ij, kl, coef) list (m rule and threshold applied) that every
// CTA stages in shared memory.
#include "common.cuh"
#include "kernels.cuh"

namespace td1c {

// fill the 2-RDM coefficients of the host-built m-allowed entry list:
// coef = den2(j,i,l,k), or 0 when |den2| <= thrwfn (mod_const.F90:32)
__global__ void act2_fill_kernel(int n, const cplx* __restrict__ den2, Act2Entry* __restrict__ list) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  cplx d = den2[list[e].d2idx];
  bool keep = sqrt(cabs2(d)) > 1.0e-15;
  list[e].cre = keep ? d.x : 0.0;
  list[e].cim = keep ? d.y : 0.0;
}

__device__ __forceinline__ cplx ldW(const cplx* __restrict__ W, int p, int cj, size_t ngrid, int q) {
  cplx w = __ldg(W + (size_t)p * ngrid + q);
  return cj ? cconj(w) : w;
}

constexpr int MF_MAXF = 16;

__global__ void __launch_bounds__(128) mfprod_kernel(MfprodArgs a) {
  extern __shared__ Act2Entry slist[];
  __shared__ cplx srden[MF_MAXF * MF_MAXF];
  __shared__ cplx sden1[MF_MAXF * MF_MAXF];
  const int nact = a.nact, ncore = a.ncore, nfcore = a.nfcore, nfun = a.nfun;
  const Act2Entry* __restrict__ glist = a.act2_list;
  const int nlist = (a.nelact >= 2 && nact > 0) ? a.nact2 : 0;
  for (int e = threadIdx.x; e < nlist; e += blockDim.x) slist[e] = glist[e];
  for (int e = threadIdx.x; e < nact * nact; e += blockDim.x) { srden[e] = a.rden[e]; sden1[e] = a.den1[e]; }
  __syncthreads();
  const size_t ng = a.ngrid;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= a.ngrid) return;
  const cplx* __restrict__ W = a.W;
  const cplx* __restrict__ og = a.orbg;
  auto PO = [&](int x, int y) { return a.pair_of[x * nfun + y]; };
  auto PC = [&](int x, int y) { return a.pair_cj[x * nfun + y]; };
  const int ndcore = ncore - nfcore;
  // ---- core terms into gorbg for every dynamic orbital
  cplx dcsum = mkc(0.0, 0.0);
  for (int j = nfcore; j < ncore; ++j) { cplx w = ldW(W, PO(j, j), PC(j, j), ng, q); dcsum.x += w.x * 2.0; dcsum.y += w.y * 2.0; }
  for (int i = nfcore; i < nfun; ++i) {
    cplx g = a.gorbg[(size_t)i * ng + q];
    for (int j = 0; j < nfcore; ++j) {  // fcx1
      cplx w = ldW(W, PO(j, i), PC(j, i), ng, q);
      g = csub(g, cmul(w, __ldg(og + (size_t)j * ng + q)));
    }
    if (ndcore > 0) {
      g = cadd(g, cmul(dcsum, __ldg(og + (size_t)i * ng + q)));  // dcj
      for (int j = nfcore; j < ncore; ++j) {  // dcx
        cplx w = ldW(W, PO(j, i), PC(j, i), ng, q);
        g = csub(g, cmul(w, __ldg(og + (size_t)j * ng + q)));
      }
    }
    a.gorbg[(size_t)i * ng + q] = g;
  }
  // ---- active terms into v2orbg of the dynamic cores
  if (ndcore > 0 && nact > 0) {
    cplx d2v = mkc(0.0, 0.0);
    for (int ja = 0; ja < nact; ++ja)
      for (int ka = 0; ka < nact; ++ka) {
        cplx w = ldW(W, PO(ncore + ja, ncore + ka), PC(ncore + ja, ncore + ka), ng, q);
        cfma(d2v, w, sden1[ka + nact * ja]);
      }
    for (int i = nfcore; i < ncore; ++i) {
      cplx v = a.v2orbg[(size_t)i * ng + q];
      v = cadd(v, cmul(d2v, __ldg(og + (size_t)i * ng + q)));
      a.v2orbg[(size_t)i * ng + q] = v;
    }
    for (int ja = 0; ja < nact; ++ja) {
      const int jf = ncore + ja;
      cplx wd1 = mkc(0.0, 0.0);
      for (int ka = 0; ka < nact; ++ka) {
        const int kf = ncore + ka;
        if (a.mval[jf] != a.mval[kf]) continue;
        cplx dens = cscale(sden1[ka + nact * ja], -0.5);
        wd1 = cadd(wd1, cmul(__ldg(og + (size_t)kf * ng + q), dens));
      }
      for (int i = nfcore; i < ncore; ++i) {
        cplx w = ldW(W, PO(jf, i), PC(jf, i), ng, q);
        cplx v = a.v2orbg[(size_t)i * ng + q];
        v = cadd(v, cmul(wd1, w));
        a.v2orbg[(size_t)i * ng + q] = v;
      }
    }
  }
  // ---- act2: 2-RDM contraction
  if (nlist > 0) {
    cplx tw[MF_MAXF];
#pragma unroll
    for (int i = 0; i < MF_MAXF; ++i) tw[i] = mkc(0.0, 0.0);
    int e = 0, ij = 0;
    for (int ia = 0; ia < nact; ++ia)
      for (int ja = 0; ja <= ia; ++ja, ++ij) {
        cplx d2v = mkc(0.0, 0.0);
        while (e < nlist && slist[e].ij == ij) {
          const Act2Entry& en = slist[e];
          cplx w = ldW(W, en.pair, en.conj, ng, q);
          cfma(d2v, mkc(en.cre, en.cim), w);
          ++e;
        }
        cplx oj = __ldg(og + (size_t)(ncore + ja) * ng + q);
        cplx oi = __ldg(og + (size_t)(ncore + ia) * ng + q);
        // tw[ia] += oj * d2v ; tw[ja] += oi * conj(d2v)  (register-indexed through a small switch)
#pragma unroll
        for (int x = 0; x < MF_MAXF; ++x) {
          if (x == ia) tw[x] = cadd(tw[x], cmul(oj, d2v));
          if (x == ja && ia > ja) tw[x] = cadd(tw[x], cmul(oi, cconj(d2v)));
        }
      }
    for (int ka = 0; ka < nact; ++ka) {
      const int kf = ncore + ka;
      cplx v = a.v2orbg[(size_t)kf * ng + q];
#pragma unroll
      for (int x = 0; x < MF_MAXF; ++x) {
        if (x < nact && a.mval[ncore + x] == a.mval[kf]) v = cadd(v, cmul(srden[x + nact * ka], tw[x]));
      }
      a.v2orbg[(size_t)kf * ng + q] = v;
    }
  }
}

int launch_mfprod(const MfprodArgs& a, cudaStream_t st) {
  if (a.nfun > MF_MAXF) return (int)cudaErrorInvalidValue;
  const int nlist = (a.nelact >= 2 && a.nact > 0) ? a.nact2 : 0;
  if (nlist > 0) act2_fill_kernel<<<(nlist + 127) / 128, 128, 0, st>>>(nlist, a.den2, a.act2_list);
  size_t smem = sizeof(Act2Entry) * (size_t)nlist;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(mfprod_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024);
    attr = true;
  }
  if (smem > 160 * 1024) return (int)cudaErrorInvalidValue;
  mfprod_kernel<<<(a.ngrid + 127) / 128, 128, smem, st>>>(a);
  return (int)cudaGetLastError();
}

}  // namespace td1c
