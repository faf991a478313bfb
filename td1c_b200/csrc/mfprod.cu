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
#include <algorithm>

#include "common.cuh"
#include "kernels.cuh"

namespace td1c {

static int launch_mfprod_scalar(const MfprodArgs& a, cudaStream_t st);

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

// ---------------------------------------------------------------------------
// act2 on the FP64 tensor cores.  Persistent CTAs of 4 warps (2 per SM)
// load the padded coefficients and the plan tables once, then loop over
// tiles of MFD_TQ grid points:
//   1. cp.async stages the tile's slice of every stored pair's W (rows of
//      MFD_TQ points, pitch MFD_WP) and the orbitals in shared memory; row
//      npair of the W slice is zero.
//   2. core terms (fcx1, dcj, dcx into gorbg; actj, actx into v2orbg of the
//      dynamic cores) over (point, orbital) items.
//   3. D2V[ij][pt] = sum_kl C[ij][kl] W(kl)[pt] per block as
//      mma.sync.m8n8k4.f64 tiles (rows ij, columns points, depth kl) with
//      four real products per complex step, stored to shared memory.
//   4. twfn_x[pt] from the target's D2V rows (in row order, as the
//      reference's loop), then v2orbg_k = sum_x rden(x, k) twfn_x.
// ---------------------------------------------------------------------------
constexpr int MFD_TQ = 16;              // points per CTA (2 n-tiles): 3 CTAs per SM
constexpr int MFD_WP = MFD_TQ + 2;      // double2 pitch of a W row: rows 8 banks apart
// double2 pitch of a D2V row: odd, so the 8 rows x 4 column pairs of one
// fragment store fall on 8 different 16-byte bank groups (4 wavefronts, the
// minimum for 512 bytes; a pitch of MFD_TQ put all 8 rows on one group)
constexpr int MFD_DP = MFD_TQ + 1;
constexpr int MFD_NT = 128;             // threads
constexpr int MFD_MAXB = 16, MFD_MAXCOL = 256, MFD_MAXROW = 128, MFD_MAXE = 512;

__device__ __forceinline__ void mfd_dmma(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}
__device__ __forceinline__ void mfd_cp16(void* dst, const void* src, unsigned bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src),
               "r"(bytes)
               : "memory");
}

static size_t mfd_smem_bytes(const MfprodArgs& a) {
  return sizeof(cplx) * ((size_t)(a.npair + 1) * MFD_WP + (size_t)a.ncoef_d + 2 * (size_t)a.nfun * MFD_TQ +
                         (size_t)a.nrow * MFD_DP + (size_t)a.nact * MFD_TQ);
}
static bool mfd_fits(const MfprodArgs& a) {
  return a.dmma && a.nfun <= MF_MAXF && a.nblk_d <= MFD_MAXB && a.ndcol <= MFD_MAXCOL && a.nrow <= MFD_MAXROW &&
         a.nelist <= MFD_MAXE && mfd_smem_bytes(a) <= 200 * 1024;
}

__global__ void __launch_bounds__(MFD_NT) mfprod_dmma_kernel(MfprodArgs a) {
  extern __shared__ __align__(16) cplx mfd_smem[];
  const int nact = a.nact, ncore = a.ncore, nfcore = a.nfcore, nfun = a.nfun, npair = a.npair;
  cplx* sW = mfd_smem;                                   // [npair + 1][WP]
  cplx* sC = sW + (size_t)(npair + 1) * MFD_WP;          // [ncoef_d]
  cplx* sPhi2 = sC + a.ncoef_d;                          // 2 x [nfun][TQ]: this tile's and the next
  cplx* sD = sPhi2 + 2 * (size_t)nfun * MFD_TQ;          // [nrow][DP]
  cplx* sTw = sD + (size_t)a.nrow * MFD_DP;              // [nact][TQ]
  __shared__ MfdBlock sblk[MFD_MAXB];
  __shared__ int2 scol[MFD_MAXCOL];
  __shared__ int2 sel[MFD_MAXE];
  __shared__ int seoff[MF_MAXF + 1];
  __shared__ cplx srden[MF_MAXF * MF_MAXF], sden1[MF_MAXF * MF_MAXF];
  __shared__ int spo[MF_MAXF * MF_MAXF], spc[MF_MAXF * MF_MAXF], smv[MF_MAXF];
  const int tid = threadIdx.x;
  const size_t ng = a.ngrid;
  const bool do_act2 = a.nelact >= 2 && nact > 0 && a.nblk_d > 0;
  const int ntile = (int)((ng + MFD_TQ - 1) / MFD_TQ);

  // ---- once per CTA: coefficients and tables
  if (do_act2)
    for (int e = tid; e < a.ncoef_d; e += MFD_NT) mfd_cp16(sC + e, a.dcoef + e, 16u);
  asm volatile("cp.async.commit_group;" ::: "memory");
  for (int e = tid; e < MFD_WP; e += MFD_NT) sW[(size_t)npair * MFD_WP + e] = mkc(0, 0);
  for (int e = tid; e < a.nblk_d; e += MFD_NT) sblk[e] = a.dblk[e];
  for (int e = tid; e < a.ndcol; e += MFD_NT) scol[e] = a.dcol[e];
  for (int e = tid; e < a.nelist; e += MFD_NT) sel[e] = a.elist[e];
  for (int e = tid; e <= nact; e += MFD_NT) seoff[e] = a.eoff[e];
  for (int e = tid; e < nact * nact; e += MFD_NT) { srden[e] = a.rden[e]; sden1[e] = a.den1[e]; }
  for (int e = tid; e < nfun * nfun; e += MFD_NT) { spo[e] = a.pair_of[e]; spc[e] = a.pair_cj[e]; }
  for (int e = tid; e < nfun; e += MFD_NT) smv[e] = a.mval[e];

  // a tile's W rows and orbitals; row npair of the W slice is zero.  The
  // copies of tile k + 1 are issued once tile k's DMMA phase has read sW, so
  // they land while tile k's twfn and v2orbg phase runs (the orbitals are
  // double-buffered: that phase still reads tile k's).
  auto stage = [&](int tile, int buf) {
    if (tile < ntile) {
      const size_t q0 = (size_t)tile * MFD_TQ;
      for (int e = tid; e < npair * MFD_TQ; e += MFD_NT) {
        const int p = e / MFD_TQ, t = e % MFD_TQ;
        const bool in = q0 + t < ng;
        mfd_cp16(sW + (size_t)p * MFD_WP + t, a.W + (size_t)p * ng + (in ? q0 + t : 0), in ? 16u : 0u);
      }
      cplx* ph = sPhi2 + (size_t)buf * nfun * MFD_TQ;
      for (int e = tid; e < nfun * MFD_TQ; e += MFD_NT) {
        const int f = e / MFD_TQ, t = e % MFD_TQ;
        const bool in = q0 + t < ng;
        mfd_cp16(ph + e, a.orbg + (size_t)f * ng + (in ? q0 + t : 0), in ? 16u : 0u);
      }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  stage(blockIdx.x, 0);
  int buf = 0;
  for (int tile = blockIdx.x; tile < ntile; tile += gridDim.x, buf ^= 1) {
  const size_t q0 = (size_t)tile * MFD_TQ;
  // ---- 1. this tile's W rows and orbitals (staged during the previous tile)
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  __syncthreads();
  const cplx* sPhi = sPhi2 + (size_t)buf * nfun * MFD_TQ;

  auto PHI = [&](int f, int t) { return sPhi[(size_t)f * MFD_TQ + t]; };
  auto WXY = [&](int x, int y, int t) {  // W(x, y) at point t from the stored pair
    const int e = x * nfun + y;
    const cplx w = sW[(size_t)spo[e] * MFD_WP + t];
    return spc[e] ? cconj(w) : w;
  };
  const int ndcore = ncore - nfcore;
  // ---- 2. core terms (same sums and order as mfprod_kernel)
  for (int e = tid; e < (nfun - nfcore) * MFD_TQ; e += MFD_NT) {
    const int i = nfcore + e / MFD_TQ, t = e % MFD_TQ;
    if (q0 + t >= ng) continue;
    cplx g = mkc(0, 0);
    for (int j = 0; j < nfcore; ++j) g = csub(g, cmul(WXY(j, i, t), PHI(j, t)));  // fcx1
    if (ndcore > 0) {
      cplx dcsum = mkc(0.0, 0.0);
      for (int j = nfcore; j < ncore; ++j) { cplx w = WXY(j, j, t); dcsum.x += w.x * 2.0; dcsum.y += w.y * 2.0; }
      g = cadd(g, cmul(dcsum, PHI(i, t)));                                        // dcj
      for (int j = nfcore; j < ncore; ++j) g = csub(g, cmul(WXY(j, i, t), PHI(j, t)));  // dcx
    }
    a.gorbg[(size_t)i * ng + q0 + t] = g;
  }
  for (int e = tid; e < ndcore * MFD_TQ; e += MFD_NT) {
    const int i = nfcore + e / MFD_TQ, t = e % MFD_TQ;
    if (q0 + t >= ng) continue;
    cplx v = mkc(0, 0);
    if (nact > 0) {
      cplx d2v = mkc(0.0, 0.0);
      for (int ja = 0; ja < nact; ++ja)
        for (int ka = 0; ka < nact; ++ka) cfma(d2v, WXY(ncore + ja, ncore + ka, t), sden1[ka + nact * ja]);
      v = cadd(v, cmul(d2v, PHI(i, t)));
      for (int ja = 0; ja < nact; ++ja) {
        const int jf = ncore + ja;
        cplx wd1 = mkc(0.0, 0.0);
        for (int ka = 0; ka < nact; ++ka) {
          const int kf = ncore + ka;
          if (smv[jf] != smv[kf]) continue;
          wd1 = cadd(wd1, cmul(PHI(kf, t), cscale(sden1[ka + nact * ja], -0.5)));
        }
        v = cadd(v, cmul(wd1, WXY(jf, i, t)));
      }
    }
    a.v2orbg[(size_t)i * ng + q0 + t] = v;
  }
  if (!do_act2) {
    for (int e = tid; e < nact * MFD_TQ; e += MFD_NT) {
      const int t = e % MFD_TQ;
      if (q0 + t < ng) a.v2orbg[(size_t)(ncore + e / MFD_TQ) * ng + q0 + t] = mkc(0, 0);
    }
    __syncthreads();  // phase 2's reads of sW are done
    stage(tile + gridDim.x, buf ^ 1);
    continue;
  }
  // ---- 3. D2V tiles on the tensor cores: each warp runs its (block,
  //      m-tile) items over all MFD_TQ / 8 n-tiles at once, the four real
  //      products of each tile in separate accumulators
  const int lane = tid & 31, warp = tid >> 5, gid = lane >> 2, tig = lane & 3;
  constexpr int NT = MFD_TQ / 8;
  for (int it = 0; it < 8; ++it) {
    const int2 wi = a.witem[warp][it];
    if (wi.x < 0) break;
    const MfdBlock B = sblk[wi.x];
    const int mt = wi.y;
    double acc[NT][4][2];
#pragma unroll
    for (int t = 0; t < NT; ++t)
#pragma unroll
      for (int h = 0; h < 4; ++h) acc[t][h][0] = acc[t][h][1] = 0.0;
    const cplx* arow = sC + B.coff + (size_t)(mt * 8 + gid) * B.pa + tig;
    for (int ks = 0; ks < B.kpad / 4; ++ks) {
      const cplx av = arow[4 * ks];
      const int2 pc = scol[B.col0 + 4 * ks + tig];
      const cplx* wrow = sW + (size_t)pc.x * MFD_WP + gid;
#pragma unroll
      for (int t = 0; t < NT; ++t) {
        const cplx bv = wrow[8 * t];
        const double bi = pc.y ? -bv.y : bv.y;
        mfd_dmma(acc[t][0][0], acc[t][0][1], av.x, bv.x);
        mfd_dmma(acc[t][1][0], acc[t][1][1], av.y, -bi);
        mfd_dmma(acc[t][2][0], acc[t][2][1], av.x, bi);
        mfd_dmma(acc[t][3][0], acc[t][3][1], av.y, bv.x);
      }
    }
    const int r = mt * 8 + gid;
    if (r < B.nr) {
#pragma unroll
      for (int t = 0; t < NT; ++t) {
        cplx* drow = sD + (size_t)(B.drow0 + r) * MFD_DP + t * 8 + 2 * tig;
        drow[0] = mkc(acc[t][0][0] + acc[t][1][0], acc[t][2][0] + acc[t][3][0]);
        drow[1] = mkc(acc[t][0][1] + acc[t][1][1], acc[t][2][1] + acc[t][3][1]);
      }
    }
  }
  __syncthreads();  // also: phases 2 and 3 have read sW
  stage(tile + gridDim.x, buf ^ 1);
  // ---- 4. twfn, then v2orbg of the active orbitals
  for (int e = tid; e < nact * MFD_TQ; e += MFD_NT) {
    const int x = e / MFD_TQ, t = e % MFD_TQ;
    cplx tw = mkc(0, 0);
    for (int k = seoff[x]; k < seoff[x + 1]; ++k) {
      const int2 en = sel[k];
      const cplx d = sD[(size_t)en.x * MFD_DP + t];
      const cplx o = PHI(ncore + (en.y & 0xffff), t);
      tw = cadd(tw, cmul(o, (en.y >> 16) ? cconj(d) : d));
    }
    sTw[(size_t)x * MFD_TQ + t] = tw;
  }
  __syncthreads();
  for (int e = tid; e < nact * MFD_TQ; e += MFD_NT) {
    const int ka = e / MFD_TQ, t = e % MFD_TQ;
    if (q0 + t >= ng) continue;
    const int kf = ncore + ka;
    cplx v = mkc(0, 0);
    for (int x = 0; x < nact; ++x)
      if (smv[ncore + x] == smv[kf]) v = cadd(v, cmul(srden[x + nact * ka], sTw[(size_t)x * MFD_TQ + t]));
    a.v2orbg[(size_t)kf * ng + q0 + t] = v;
  }
  }  // tile loop
}

int launch_mfprod(const MfprodArgs& a, cudaStream_t st) {
  if (mfd_fits(a)) {
    const bool do_act2 = a.nelact >= 2 && a.nact > 0 && a.nblk_d > 0;
    if (do_act2) act2_fill_kernel<<<(a.ncoef + 127) / 128, 128, 0, st>>>(a.ncoef, a.dmap, a.den2, a.dcoef);
    const size_t smem = mfd_smem_bytes(a);
    static bool attr = false;
    if (!attr) {
      cudaFuncSetAttribute(mfprod_dmma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
      attr = true;
    }
    // persistent: as many CTAs as are resident at once (shared memory decides; at
    // least 2 per SM), sized once per shared-memory footprint
    static int nsm = 0, cps = 0;
    static size_t cps_smem = 0;
    if (!nsm) {
      int dev = 0;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    }
    if (cps_smem != smem) {
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&cps, mfprod_dmma_kernel, MFD_NT, smem) != cudaSuccess) cps = 2;
      cps = std::max(cps, 2);
      cps_smem = smem;
    }
    const int ntile = (int)((a.ngrid + MFD_TQ - 1) / MFD_TQ);
    int grid = std::min(ntile, cps * nsm);
    if (a.max_cta > 0) grid = std::min(grid, a.max_cta);
    mfprod_dmma_kernel<<<(unsigned)grid, MFD_NT, smem, st>>>(a);
    return (int)cudaGetLastError();
  }
  return launch_mfprod_scalar(a, st);
}

static int launch_mfprod_scalar(const MfprodArgs& a, cudaStream_t st) {
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
