// poisson_cond.cu -- the radial Poisson solve of the mean field
// (hprod_mkv2mf_poissonp, hprod_mkv2mf.F90:118-182) by static condensation.
//
// Per pair and l the reference solves A_l x = b with A_l = l(l+1)/r^2 + 2 T
// (the d2ll band, factored by dpbtrf) and b = rho (2l+1)/(2 pi r sqrt(w)),
// then v = (x + t r^(l+1) sqrt(w)) 4 pi / ((2l+1) r sqrt(w)) with the
// boundary term t = sum_r rho r^l / (2 pi) / rmax^(2l+1).  The banded
// substitution is sequential over the nrad - 1 rows.  Here A_l is inverted
// the way h1prop.cu inverts 1 + c T: A_l couples only the points of one
// finite element, so
//   1. each element's share of the bridge right-hand sides and of t (three
//      dot products over its points: A symmetric makes
//      A(bridge, I_e) A_e^-1 b(I_e) = GL . b(I_e));
//   2. per (pair, l) the tridiagonal bridge system (symmetric positive
//      definite, LU without interchanges) gives x(B), and t is summed;
//   3. x(I_e) = A_e^-1 b(I_e) - GL_e x(left) - GR_e x(right), then v,
//      element by element, the interior products on the FP64 tensor cores.
// Passes 1 and 3 are parallel over pairs, multipoles and elements; the only
// sequential part is the 59-point bridge solve.  The set-up inverts each
// interior block by Gauss-Jordan elimination with partial pivoting and folds
// the pointwise factors (b = rho invr, v = (x + t rpl1) fac2) into
// per-(l, element) records, so a tile stages one record per multipole.
#include <algorithm>

#include "common.cuh"
#include "kernels.cuh"
#include "tc.cuh"

namespace td1c {

// A_l(i, j) for 1-based radial indices, |i - j| <= nd
struct PsMat {
  const double* xrad;
  const double* radk;
  int nd, l;
  __device__ double operator()(int i, int j) const {
    double v = 2.0 * radk[(size_t)(2 * nd + 1) * i + nd + j - i];
    if (i == j) {
      const double ak = 1.0 / xrad[i];
      v += ak * ak * (double)l * (double)(l + 1);
    }
    return v;
  }
};

// pointwise Poisson factors: [L2][Nr] tables over radial points ip = 1 .. Nr
struct PsPoint {
  const double *invr, *rpl0, *rpl1, *fac2;
};

constexpr int PSC_NT = 64;

// per (element, l): the interior inverse by Gauss-Jordan elimination, GL/GR,
// the bridge couplings, and the two records
__global__ void __launch_bounds__(PSC_NT) ps_cond_elem_kernel(PsCond f, const double* __restrict__ xrad,
                                                              const double* __restrict__ radk, PsPoint pp,
                                                              int* status) {
  extern __shared__ double sa[];  // [ni][2 ni] augmented [A | I]
  __shared__ int piv_row;
  __shared__ double glk[24], grk[24];
  const int e = blockIdx.x, l = blockIdx.y, ni = f.ni, nd = f.nd, w = 2 * ni, tid = threadIdx.x;
  const PsMat A{xrad, radk, nd, l};
  const int i0 = nd * e;
  for (int q = tid; q < ni * w; q += PSC_NT) {
    const int r = q / w, c = q % w;
    sa[q] = c < ni ? A(i0 + r + 1, i0 + c + 1) : (c - ni == r ? 1.0 : 0.0);
  }
  __syncthreads();
  bool singular = false;
  for (int p = 0; p < ni; ++p) {
    if (tid == 0) {
      int best = p;
      double bv = -1.0;
      for (int r = p; r < ni; ++r)
        if (fabs(sa[r * w + p]) > bv) { bv = fabs(sa[r * w + p]); best = r; }
      piv_row = best;
    }
    __syncthreads();
    const int pr = piv_row;
    if (pr != p)
      for (int c = tid; c < w; c += PSC_NT) { const double t = sa[p * w + c]; sa[p * w + c] = sa[pr * w + c]; sa[pr * w + c] = t; }
    __syncthreads();
    const double pv = sa[p * w + p];
    if (pv == 0.0) { singular = true; break; }
    const double rp = 1.0 / pv;
    __syncthreads();
    for (int c = tid; c < w; c += PSC_NT) sa[p * w + c] *= rp;
    __syncthreads();
    for (int q = tid; q < ni * w; q += PSC_NT) {
      const int r = q / w, c = q % w;
      if (r == p || c == p) continue;
      sa[q] -= sa[r * w + p] * sa[p * w + c];
    }
    __syncthreads();
    for (int r = tid; r < ni; r += PSC_NT)
      if (r != p) sa[r * w + p] = 0.0;
    __syncthreads();
  }
  if (singular) {
    if (tid == 0) atomicOr(status, ST_CHOLESKY);
    return;
  }
  const size_t base = ((size_t)l * f.nfe + e) * ni;
  const bool hasl = e >= 1, hasr = e + 1 < f.nfe;
  for (int k = tid; k < ni; k += PSC_NT) {
    double gl = 0.0, gr = 0.0;
    for (int j = 0; j < ni; ++j) {
      const double a = sa[k * w + ni + j];
      if (hasl) gl = fma(a, A(i0 + j + 1, i0), gl);
      if (hasr) gr = fma(a, A(i0 + j + 1, i0 + nd), gr);
    }
    f.gl[base + k] = gl;
    f.gr[base + k] = gr;
    glk[k] = gl;
    grk[k] = gr;
    f.vl[base + k] = hasl ? A(i0, i0 + k + 1) : 0.0;
    f.vr[base + k] = hasr ? A(i0 + nd, i0 + k + 1) : 0.0;
  }
  __syncthreads();
  const size_t lr = (size_t)l * f.Nr;
  auto at = [&](const double* tab, int ip) { return ip >= 1 ? tab[lr + ip - 1] : 0.0; };
  // element record: W(j, k) = fac2(k) Ainv(k, j) invr(j) as [j][k] (k the interior point
  // i0 + k + 1), fac2 GL, fac2 GR, fac2 rpl1, then (fac2, fac2 rpl1) at the left bridge i0
  double* er = f.erec + ((size_t)l * f.nfe + e) * f.er;
  for (int q = tid; q < ni * ni; q += PSC_NT) {
    const int j = q / ni, k = q % ni;
    er[q] = at(pp.fac2, i0 + k + 1) * sa[k * w + ni + j] * at(pp.invr, i0 + j + 1);
  }
  for (int k = tid; k < ni; k += PSC_NT) {
    const double f2 = at(pp.fac2, i0 + k + 1);
    er[ni * ni + k] = f2 * glk[k];
    er[ni * ni + ni + k] = f2 * grk[k];
    er[ni * ni + 2 * ni + k] = f2 * at(pp.rpl1, i0 + k + 1);
  }
  if (tid == 0) {
    const double f2 = hasl ? at(pp.fac2, i0) : 0.0;
    er[ni * ni + 3 * ni] = f2;
    er[ni * ni + 3 * ni + 1] = hasl ? f2 * at(pp.rpl1, i0) : 0.0;
    for (int q = ni * ni + 3 * ni + 2; q < f.er; ++q) er[q] = 0.0;
  }
  // share record: rows (t, left share, right share) over the owned points pt = 0 .. nd - 1
  // (radial point i0 + pt): rpl0; invr at the bridge and -GL invr inside; -GR invr inside
  double* sr = f.srec + ((size_t)l * f.nfe + e) * f.sr;
  for (int pt = tid; pt < nd; pt += PSC_NT) {
    const double iv = at(pp.invr, i0 + pt);
    sr[pt] = at(pp.rpl0, i0 + pt);
    sr[nd + pt] = !hasl ? 0.0 : (pt == 0 ? iv : -glk[pt - 1] * iv);
    sr[2 * nd + pt] = (!hasr || pt == 0) ? 0.0 : -grk[pt - 1] * iv;
  }
  if (tid == 0)
    for (int q = 3 * nd; q < f.sr; ++q) sr[q] = 0.0;
}

// per l: the bridge Schur complement and its LU without interchanges (it is
// symmetric positive definite)
__global__ void ps_cond_bridge_kernel(PsCond f, const double* __restrict__ xrad, const double* __restrict__ radk,
                                      int* status) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= f.L2) return;
  const int nb = f.nb, ni = f.ni, nd = f.nd;
  if (nb <= 0) return;
  const PsMat A{xrad, radk, nd, l};
  const size_t eb = (size_t)l * f.nfe * ni;
  auto dot = [&](const double* a, const double* b) {
    double s = 0.0;
    for (int k = 0; k < ni; ++k) s = fma(a[k], b[k], s);
    return s;
  };
  double* tm = f.tm + (size_t)l * nb;
  double* tw = f.tw + (size_t)l * nb;
  double* tu = f.tu + (size_t)l * nb;
  double wprev = 0.0, uprev = 0.0;
  for (int b = 0; b < nb; ++b) {
    const int ib = nd * (b + 1);
    double d = A(ib, ib) - dot(f.vr + eb + (size_t)b * ni, f.gr + eb + (size_t)b * ni) -
               dot(f.vl + eb + (size_t)(b + 1) * ni, f.gl + eb + (size_t)(b + 1) * ni);
    if (b > 0) {
      const int ia = nd * b;  // previous bridge
      const double sub = A(ib, ia) - dot(f.vr + eb + (size_t)b * ni, f.gl + eb + (size_t)b * ni);
      const double m = sub / wprev;
      tm[b] = m;
      d -= m * uprev;
    } else {
      tm[b] = 0.0;
    }
    if (!(d > 0.0)) { atomicOr(status, ST_CHOLESKY); return; }
    tw[b] = 1.0 / d;
    const double up = b + 1 < nb ? A(ib, ib + nd) - dot(f.vl + eb + (size_t)(b + 1) * ni, f.gr + eb + (size_t)(b + 1) * ni) : 0.0;
    tu[b] = up;
    wprev = d;
    uprev = up;
  }
}

int launch_ps_cond_setup(PsCond& f, const double* xrad, const double* radk, const double* invr, const double* rpl0,
                         const double* rpl1, const double* fac2, int* status, cudaStream_t st) {
  const size_t smem = sizeof(double) * (size_t)f.ni * 2 * f.ni;
  if (f.ni > 24 || smem > 48 * 1024) return ST_CONFIG;
  ps_cond_elem_kernel<<<dim3(f.nfe, f.L2), PSC_NT, smem, st>>>(f, xrad, radk, PsPoint{invr, rpl0, rpl1, fac2}, status);
  ps_cond_bridge_kernel<<<(f.L2 + 31) / 32, 32, 0, st>>>(f, xrad, radk, status);
  return (int)cudaGetLastError();
}

// ---------------------------------------------------------------------------
// per-RHS passes
// ---------------------------------------------------------------------------
// A tile is one element e, multipoles l0 .. l0 + LC - 1 and pairs
// p0 .. p0 + PC - 1, one CTA that stages the tile's rho rows, its records
// and (pass 3) the bridge values with cp.async (zero-filled outside the
// grid, the multipole range and the pair range), then computes from shared
// memory.
constexpr int PSE_LC = 4;    // multipoles per tile
constexpr int PSE_PC = 32;   // pairs per tile
constexpr int PSE_NT = 256;  // threads per tile

__device__ __forceinline__ void psc_cp16(void* dst, const void* src, bool ok) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src),
               "r"(ok ? 16u : 0u)
               : "memory");
}
__device__ __forceinline__ void psc_cp8(void* dst, const void* src, bool ok) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src),
               "r"(ok ? 8u : 0u)
               : "memory");
}
__device__ __forceinline__ void psc_cp4(void* dst, const void* src, bool ok) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src),
               "r"(ok ? 4u : 0u)
               : "memory");
}
__device__ __forceinline__ void psc_wait_all() {
  asm volatile("cp.async.commit_group;" ::: "memory");
  asm volatile("cp.async.wait_group 0;" ::: "memory");
}

// 1. the element's shares: the three rows of its share record (t, left,
// right) times its rho over the owned points (the left bridge and the
// interior; point 0 of the first element lies outside the grid and reads as
// zero).  The staged rows have a pair stride odd in 16-byte units, so the
// eight lanes of a quarter-warp (consecutive pairs) hit distinct banks.
__host__ __device__ inline int ps_share_stride(int nd) { return PSE_LC * nd + 1; }
size_t ps_share_smem(int nd, int sr) {
  return sizeof(cplx) * (size_t)PSE_PC * ps_share_stride(nd) + sizeof(double) * (size_t)PSE_LC * sr + sizeof(int) * PSE_PC;
}

template <int NDT>
__global__ void __launch_bounds__(PSE_NT) ps_share_kernel(PsCondArgs a) {
  extern __shared__ __align__(16) unsigned char ps_sm[];
  const PsCond& F = a.f;
  const int nd = NDT > 0 ? NDT : F.nd, sr = F.sr;
  const int nfe = F.nfe, Nr = a.Nr, L2 = a.L2, npair = a.npair, tid = threadIdx.x;
  const int e = blockIdx.x, l0 = blockIdx.y * PSE_LC, p0 = blockIdx.z * PSE_PC, ir0 = nd * e;
  const int S = ps_share_stride(nd);
  cplx* RHO = reinterpret_cast<cplx*>(ps_sm);                           // [PC][S]: [LC][nd] per pair
  double* REC = reinterpret_cast<double*>(RHO + (size_t)PSE_PC * S);   // [LC][sr]
  int* PM = reinterpret_cast<int*>(REC + (size_t)PSE_LC * sr);         // [PC]
  for (int q = tid; q < PSE_PC * PSE_LC * nd; q += PSE_NT) {
    const int pc = q / (PSE_LC * nd), lc = (q / nd) % PSE_LC, pt = q % nd;
    const int p = p0 + pc, l = l0 + lc, ip = ir0 + pt;
    const bool ok = p < npair && l < L2 && ip >= 1 && ip <= Nr;
    psc_cp16(RHO + pc * S + lc * nd + pt, a.rho2 + (ok ? ((size_t)p * L2 + l) * Nr + ip - 1 : 0), ok);
  }
  {
    const int lc = tid / (PSE_NT / PSE_LC), l = l0 + lc;  // PSE_NT / LC threads per record
    const bool ok = l < L2;
    const double* src = F.srec + (ok ? ((size_t)l * nfe + e) * sr : 0);
    for (int c = tid % (PSE_NT / PSE_LC); c < sr / 2; c += PSE_NT / PSE_LC)
      psc_cp16(REC + lc * sr + 2 * c, src + (ok ? 2 * c : 0), ok);
  }
  for (int q = tid; q < PSE_PC; q += PSE_NT) psc_cp4(PM + q, a.pair_m + (p0 + q < npair ? p0 + q : 0), p0 + q < npair);
  psc_wait_all();
  __syncthreads();
  // s = 0: t and the left share; s = 1: the right share
  for (int it = tid; it < 2 * PSE_PC * PSE_LC; it += PSE_NT) {
    const int s = it / (PSE_PC * PSE_LC), pc = it % PSE_PC, lc = (it / PSE_PC) % PSE_LC;
    const int p = p0 + pc, l = l0 + lc;
    if (p >= npair || l >= L2) continue;
    const int m = PM[pc];
    if (l < (m < 0 ? -m : m)) continue;
    const cplx* rho = RHO + pc * S + lc * nd;
    const double* rec = REC + lc * sr;
    const size_t le = (size_t)l * nfe + e;
    if (s == 0) {
      cplx t = mkc(0, 0), c = mkc(0, 0);
#pragma unroll 4
      for (int pt = 0; pt < nd; ++pt) {
        const cplx r = rho[pt];
        const double c0 = rec[pt], c1 = rec[nd + pt];
        t.x = fma(c0, r.x, t.x); t.y = fma(c0, r.y, t.y);
        c.x = fma(c1, r.x, c.x); c.y = fma(c1, r.y, c.y);
      }
      a.tpart[le * npair + p] = t;
      if (e >= 1) a.cb[(le * 2) * npair + p] = c;
    } else if (e + 1 < nfe) {
      cplx c = mkc(0, 0);
#pragma unroll 4
      for (int pt = 1; pt < nd; ++pt) {
        const cplx r = rho[pt];
        const double c2 = rec[2 * nd + pt];
        c.x = fma(c2, r.x, c.x); c.y = fma(c2, r.y, c.y);
      }
      a.cb[(le * 2 + 1) * npair + p] = c;
    }
  }
}

// 2. per (l, pair chunk): bridge right-hand sides, tridiagonal solve, t.
// One thread per pair; everything the recurrence reads is staged first, by
// all PSB_STAGE threads of the CTA.
constexpr int PSB_NT = 32;      // pairs per CTA (threads of the recurrence)
constexpr int PSB_STAGE = 128;  // threads of the CTA

size_t ps_bridge_smem(int nfe, int nb) {
  return sizeof(cplx) * (size_t)PSB_NT * nfe * 3 + sizeof(double) * 3 * (size_t)nb;
}

__global__ void __launch_bounds__(PSB_STAGE) ps_bridge_kernel(PsCondArgs a) {
  extern __shared__ cplx psb_sm[];
  const PsCond& F = a.f;
  const int l = blockIdx.x, p0 = blockIdx.y * PSB_NT, nb = F.nb, nfe = F.nfe, npair = a.npair, tid = threadIdx.x;
  cplx* CB = psb_sm;                         // [nfe][2][NT]
  cplx* TP = CB + (size_t)PSB_NT * nfe * 2;  // [nfe][NT]
  double* tm = reinterpret_cast<double*>(TP + (size_t)PSB_NT * nfe);
  double* tw = tm + nb;
  double* tu = tw + nb;
  for (int q = tid; q < PSB_NT * nfe * 2; q += PSB_STAGE) {
    const int r = q / PSB_NT, pc = q % PSB_NT, p = p0 + pc;
    const bool ok = p < npair && ((r & 1) ? r < 2 * nfe - 1 : r >= 2);  // shares that exist
    psc_cp16(CB + q, a.cb + (ok ? ((size_t)l * nfe * 2 + r) * npair + p : 0), ok);
  }
  for (int q = tid; q < PSB_NT * nfe; q += PSB_STAGE) {
    const int r = q / PSB_NT, pc = q % PSB_NT, p = p0 + pc;
    const bool ok = p < npair;
    psc_cp16(TP + q, a.tpart + (ok ? ((size_t)l * nfe + r) * npair + p : 0), ok);
  }
  for (int q = tid; q < nb; q += PSB_STAGE) {
    const size_t o = (size_t)l * nb + q;
    psc_cp8(tm + q, F.tm + o, true);
    psc_cp8(tw + q, F.tw + o, true);
    psc_cp8(tu + q, F.tu + o, true);
  }
  psc_wait_all();
  __syncthreads();
  const int p = p0 + tid;
  if (tid >= PSB_NT || p >= npair) return;
  const int m = a.pair_m[p];
  if (l < (m < 0 ? -m : m)) return;
  cplx* xb = a.xb + (size_t)l * nb * npair + p;  // xb[b * npair]
  // forward: y_b = g_b - m_b y_(b-1); y_b is parked in the consumed share slot 2b + 1
  cplx y = mkc(0, 0);
  for (int b = 0; b < nb; ++b) {
    cplx g = cadd(CB[(2 * b + 1) * PSB_NT + tid], CB[(2 * b + 2) * PSB_NT + tid]);
    g.x = fma(-tm[b], y.x, g.x); g.y = fma(-tm[b], y.y, g.y);  // tm[0] = 0
    y = g;
    CB[(2 * b + 1) * PSB_NT + tid] = y;
  }
  // backward: x_b = (y_b - u_b x_(b+1)) / w_b  (u_(nb-1) = 0)
  cplx x = mkc(0, 0);
  for (int b = nb - 1; b >= 0; --b) {
    cplx v = CB[(2 * b + 1) * PSB_NT + tid];
    v.x = fma(-tu[b], x.x, v.x); v.y = fma(-tu[b], x.y, v.y);
    x = mkc(v.x * tw[b], v.y * tw[b]);
    xb[(size_t)b * npair] = x;
  }
  // t = fac1 sum_e tpart_e, in element order
  cplx t = mkc(0, 0);
  for (int e = 0; e < nfe; ++e) t = cadd(t, TP[e * PSB_NT + tid]);
  a.t[(size_t)l * npair + p] = cscale(t, a.fac1[l]);
}

// 3. v on the element's owned points: inside, v(k) = sum_j W(k, j) rho(j)
// - fac2 GL x(left) - fac2 GR x(right) + fac2 rpl1 t; at the left bridge,
// v = fac2 x(bridge) + fac2 rpl1 t; zeros for l < |m|.  The interior
// products run on the FP64 tensor cores (mma m8n8k4): W is the A operand,
// rows k and depth j padded to multiples of 8 and 4 with zeros; the staged
// rho is the B operand with the columns (pair, re|im), so a lane's two
// accumulators are the real and imaginary part of one x(k, pair).  Warp w
// takes multipole w / 2 and pairs 16 (w % 2) .. + 15 as four 8-column tiles;
// its A fragments stay in registers across the tiles.
__device__ __forceinline__ void ps_dmma(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

constexpr int PSE_MT = 3;  // 8-row tiles of the interior (ni <= 24)
constexpr int PSE_KS = 6;  // 4-deep steps (ni <= 24)

// pair stride of the staged interior rows (16-byte units): at least LC ni and
// 4 or 12 mod 16, so the four pairs of a B fragment load fall in distinct banks
__host__ __device__ inline int ps_elem_stride(int nd) {
  int s = PSE_LC * (nd - 1);
  while (s % 16 != 4 && s % 16 != 12) ++s;
  return s;
}
size_t ps_elem_smem(int nd, int er) {
  return sizeof(cplx) * ((size_t)PSE_PC * ps_elem_stride(nd) + 3 * (size_t)PSE_LC * PSE_PC) +
         sizeof(double) * (size_t)PSE_LC * er + sizeof(int) * PSE_PC;
}

// mixed mode 3: the interior products in split TF32 (x = x_hi + x_lo, three mma.sync m16n8k8
// per depth step of 8, lo terms first, FP32 accumulation), the bridge and boundary terms in FP64.
// The 19 x 19 element blocks are far below tcgen05's 64- and 128-row tiles, so the warp-level
// MMA is the tensor path here.
__device__ __forceinline__ void ps_mma_tf32(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
               : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
               : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

template <int NDT, bool TF32>
__global__ void __launch_bounds__(PSE_NT, 3) ps_elem_kernel(PsCondArgs a) {
  extern __shared__ __align__(16) unsigned char ps_sm[];
  const PsCond& F = a.f;
  const int nd = NDT > 0 ? NDT : F.nd, er = F.er;
  const int ni = nd - 1, nfe = F.nfe, nb = F.nb, Nr = a.Nr, L2 = a.L2, npair = a.npair, tid = threadIdx.x;
  const int e = blockIdx.x, l0 = blockIdx.y * PSE_LC, p0 = blockIdx.z * PSE_PC, ir0 = nd * e;
  const int S = ps_elem_stride(nd);
  cplx* RHO = reinterpret_cast<cplx*>(ps_sm);                          // [PC][S]: [LC][ni] per pair
  cplx* XB = RHO + (size_t)PSE_PC * S;                                 // [LC][2][PC] bridge x (left, right)
  cplx* TS = XB + 2 * PSE_LC * PSE_PC;                                 // [LC][PC] t
  double* REC = reinterpret_cast<double*>(TS + PSE_LC * PSE_PC);       // [LC][er]
  int* PM = reinterpret_cast<int*>(REC + (size_t)PSE_LC * er);         // [PC]
  for (int q = tid; q < PSE_PC * PSE_LC * ni; q += PSE_NT) {
    const int pc = q / (PSE_LC * ni), lc = (q / ni) % PSE_LC, k = q % ni;
    const int p = p0 + pc, l = l0 + lc;
    const bool ok = p < npair && l < L2;
    psc_cp16(RHO + pc * S + lc * ni + k, a.rho2 + (ok ? ((size_t)p * L2 + l) * Nr + ir0 + k : 0), ok);  // point ir0 + k + 1
  }
  {
    const int lc = tid / (PSE_NT / PSE_LC), l = l0 + lc;  // PSE_NT / LC threads per record
    const bool ok = l < L2;
    const double* src = F.erec + (ok ? ((size_t)l * nfe + e) * er : 0);
    for (int c = tid % (PSE_NT / PSE_LC); c < er / 2; c += PSE_NT / PSE_LC)
      psc_cp16(REC + lc * er + 2 * c, src + (ok ? 2 * c : 0), ok);
  }
  for (int q = tid; q < 3 * PSE_LC * PSE_PC; q += PSE_NT) {
    // q < 2 LC PC: bridge values (side 0: bridge e - 1, side 1: bridge e), zero where the
    // element has no such bridge; then t
    const int pc = q % PSE_PC, p = p0 + pc;
    if (q < 2 * PSE_LC * PSE_PC) {
      const int side = (q / PSE_PC) & 1, lc = q / (2 * PSE_PC), l = l0 + lc, b = e - 1 + side;
      const bool ok = p < npair && l < L2 && b >= 0 && b < nb;
      psc_cp16(XB + q, a.xb + (ok ? ((size_t)l * nb + b) * npair + p : 0), ok);
    } else {
      const int lc = (q - 2 * PSE_LC * PSE_PC) / PSE_PC, l = l0 + lc;
      const bool ok = p < npair && l < L2;
      psc_cp16(TS + (q - 2 * PSE_LC * PSE_PC), a.t + (ok ? (size_t)l * npair + p : 0), ok);
    }
  }
  for (int q = tid; q < PSE_PC; q += PSE_NT) psc_cp4(PM + q, a.pair_m + (p0 + q < npair ? p0 + q : 0), p0 + q < npair);
  psc_wait_all();
  __syncthreads();
  const int warp = tid >> 5, lane = tid & 31, lc = warp >> 1, half = warp & 1, l = l0 + lc;
  if (l < L2) {
    const int mt_n = (ni + 7) >> 3, ks_n = (ni + 3) >> 2;
    const double* rec = REC + (size_t)lc * er;
    const double* gls = rec + ni * ni;  // fac2 GL, fac2 GR, fac2 rpl1
    const double* grs = gls + ni;
    const double* q1 = grs + ni;
    const double* rd = reinterpret_cast<const double*>(RHO);
    if constexpr (TF32) {
      const int gid = lane >> 2, tig = lane & 3;
      for (int mt = 0; mt < 2; ++mt) {
        if (16 * mt >= ni) break;
        uint32_t ah[3][4], al[3][4];  // A(k, j) = W(k, j) = rec[j ni + k]: rows 16 mt + gid (+8), depths 8 ks + tig (+4)
#pragma unroll
        for (int ks = 0; ks < 3; ++ks)
#pragma unroll
          for (int r = 0; r < 4; ++r) {
            const int k = 16 * mt + gid + 8 * (r & 1), j = 8 * ks + tig + 4 * (r >> 1);
            tc_split((k < ni && j < ni) ? rec[j * ni + k] : 0.0, ah[ks][r], al[ks][r]);
          }
        for (int nt = 0; nt < 4; ++nt) {
          const int pcb = 16 * half + 4 * nt + (gid >> 1), part = gid & 1;  // this lane's B column
          float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
          for (int ks = 0; ks < 3; ++ks) {
            const int j0 = 8 * ks + tig, j1 = j0 + 4;
            uint32_t bh0, bl0, bh1, bl1;
            tc_split(j0 < ni ? rd[2 * (pcb * S + lc * ni + j0) + part] : 0.0, bh0, bl0);
            tc_split(j1 < ni ? rd[2 * (pcb * S + lc * ni + j1) + part] : 0.0, bh1, bl1);
            ps_mma_tf32(acc, al[ks], bh0, bh1);
            ps_mma_tf32(acc, ah[ks], bl0, bl1);
            ps_mma_tf32(acc, ah[ks], bh0, bh1);
          }
          const int pc = 16 * half + 4 * nt + tig;  // C(16 mt + gid (+8), 2 tig | 2 tig + 1): re, im of x(k, pc)
          const int p = p0 + pc;
          if (p >= npair) continue;
          const int m = PM[pc];
          const bool zero = l < (m < 0 ? -m : m);
          const cplx bl = XB[(2 * lc) * PSE_PC + pc], br = XB[(2 * lc + 1) * PSE_PC + pc];
          const cplx tt = TS[lc * PSE_PC + pc];
          cplx* out = a.v2sph + ((size_t)p * L2 + l) * Nr + ir0;
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int k = 16 * mt + gid + 8 * h;
            if (k >= ni) continue;
            if (zero) { out[k] = mkc(0, 0); continue; }
            const double gl = gls[k], gr = grs[k], qq = q1[k];
            double vx = (double)acc[2 * h], vy = (double)acc[2 * h + 1];
            vx = fma(-gl, bl.x, vx); vy = fma(-gl, bl.y, vy);
            vx = fma(-gr, br.x, vx); vy = fma(-gr, br.y, vy);
            out[k] = mkc(fma(qq, tt.x, vx), fma(qq, tt.y, vy));
          }
        }
      }
    } else {
    double af[PSE_MT][PSE_KS];  // A(k, j) = W(k, j) = rec[j ni + k], k = 8 mt + lane / 4, j = 4 ks + lane % 4
#pragma unroll
    for (int mt = 0; mt < PSE_MT; ++mt)
#pragma unroll
      for (int ks = 0; ks < PSE_KS; ++ks) {
        const int k = 8 * mt + (lane >> 2), j = 4 * ks + (lane & 3);
        af[mt][ks] = (mt < mt_n && ks < ks_n && k < ni && j < ni) ? rec[j * ni + k] : 0.0;
      }
    for (int nt = 0; nt < 4; ++nt) {
      const int pcb = 16 * half + 4 * nt + (lane >> 3), part = (lane >> 2) & 1;  // this lane's B column
      double acc[PSE_MT][2];
#pragma unroll
      for (int mt = 0; mt < PSE_MT; ++mt) acc[mt][0] = acc[mt][1] = 0.0;
#pragma unroll
      for (int ks = 0; ks < PSE_KS; ++ks) {
        if (ks < ks_n) {
          const int j = 4 * ks + (lane & 3);
          const double b = j < ni ? rd[2 * (pcb * S + lc * ni + j) + part] : 0.0;
#pragma unroll
          for (int mt = 0; mt < PSE_MT; ++mt)
            if (mt < mt_n) ps_dmma(acc[mt][0], acc[mt][1], af[mt][ks], b);
        }
      }
      const int pc = 16 * half + 4 * nt + (lane & 3);  // the pair of this lane's accumulators
      const int p = p0 + pc;
      if (p >= npair) continue;
      const int m = PM[pc];
      const bool zero = l < (m < 0 ? -m : m);  // rows below |m| are written as zeros
      const cplx bl = XB[(2 * lc) * PSE_PC + pc], br = XB[(2 * lc + 1) * PSE_PC + pc];  // zero where absent
      const cplx tt = TS[lc * PSE_PC + pc];
      cplx* out = a.v2sph + ((size_t)p * L2 + l) * Nr + ir0;  // out[k] is radial point ir0 + k + 1
#pragma unroll
      for (int mt = 0; mt < PSE_MT; ++mt) {
        const int k = 8 * mt + (lane >> 2);
        if (mt >= mt_n || k >= ni) continue;
        if (zero) { out[k] = mkc(0, 0); continue; }
        const double gl = gls[k], gr = grs[k], qq = q1[k];
        double vx = acc[mt][0], vy = acc[mt][1];
        vx = fma(-gl, bl.x, vx); vy = fma(-gl, bl.y, vy);
        vx = fma(-gr, br.x, vx); vy = fma(-gr, br.y, vy);
        out[k] = mkc(fma(qq, tt.x, vx), fma(qq, tt.y, vy));
      }
    }
    }  // FP64 DMMA
  }
  // the left bridge point
  if (e >= 1) {
    for (int it = tid; it < PSE_PC * PSE_LC; it += PSE_NT) {
      const int pc = it % PSE_PC, lc2 = it / PSE_PC;
      const int p = p0 + pc, l2 = l0 + lc2;
      if (p >= npair || l2 >= L2) continue;
      cplx* out = a.v2sph + ((size_t)p * L2 + l2) * Nr + ir0 - 1;
      const int m = PM[pc];
      if (l2 < (m < 0 ? -m : m)) { *out = mkc(0, 0); continue; }
      const double* qb = REC + (size_t)lc2 * er + ni * ni + 3 * ni;  // fac2, fac2 rpl1 at the bridge
      const cplx x = XB[(2 * lc2) * PSE_PC + pc], tt = TS[lc2 * PSE_PC + pc];
      *out = mkc(fma(qb[0], x.x, qb[1] * tt.x), fma(qb[0], x.y, qb[1] * tt.y));
    }
  }
}

template <class K>
int ps_launch(K kernel, size_t smem, dim3 grid, int nt, const PsCondArgs& a, cudaStream_t st, size_t& cur) {
  if (smem > 227 * 1024) return ST_CONFIG;
  if (smem > 48 * 1024 && smem > cur) {
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return (int)e;
    cur = smem;
  }
  kernel<<<grid, nt, smem, st>>>(a);
  return (int)cudaGetLastError();
}

template <int NDT>
int launch_ps_tiles(const PsCondArgs& a, bool share, cudaStream_t st) {
  static size_t cur[3] = {0, 0, 0};
  const dim3 grid(a.f.nfe, (a.L2 + PSE_LC - 1) / PSE_LC, (a.npair + PSE_PC - 1) / PSE_PC);
  if (share) return ps_launch(ps_share_kernel<NDT>, ps_share_smem(a.f.nd, a.f.sr), grid, PSE_NT, a, st, cur[1]);
  if (a.tf32) return ps_launch(ps_elem_kernel<NDT, true>, ps_elem_smem(a.f.nd, a.f.er), grid, PSE_NT, a, st, cur[2]);
  return ps_launch(ps_elem_kernel<NDT, false>, ps_elem_smem(a.f.nd, a.f.er), grid, PSE_NT, a, st, cur[0]);
}

int launch_ps_pass(const PsCondArgs& a, bool share, cudaStream_t st) {
  switch (a.f.nd) {  // 21-, 9- and 8-point Lobatto elements get the unrolled rows
    case 20: return launch_ps_tiles<20>(a, share, st);
    case 8: return launch_ps_tiles<8>(a, share, st);
    case 7: return launch_ps_tiles<7>(a, share, st);
    default: return launch_ps_tiles<0>(a, share, st);
  }
}

int launch_ps_cond(const PsCondArgs& a, cudaStream_t st) {
  static_assert(PSE_NT == 64 * PSE_LC && PSE_PC == 32, "element pass: two warps of 16 pairs per multipole");
  static_assert(PSE_NT % PSE_LC == 0, "record staging: PSE_NT / LC threads per record");
  if (a.npair <= 0) return 0;
  if (a.f.nd - 1 > 8 * PSE_MT || a.f.nd - 1 > 4 * PSE_KS) return ST_CONFIG;
  int rc = launch_ps_pass(a, true, st);
  if (rc) return rc;
  {
    const size_t smem = ps_bridge_smem(a.f.nfe, a.f.nb);
    static size_t cur = 0;
    if (smem > 220 * 1024) return ST_CONFIG;
    if (smem > 48 * 1024 && smem > cur) {
      cudaError_t e = cudaFuncSetAttribute(ps_bridge_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return (int)e;
      cur = smem;
    }
    ps_bridge_kernel<<<dim3(a.L2, (a.npair + PSB_NT - 1) / PSB_NT), PSB_STAGE, smem, st>>>(a);
    rc = (int)cudaGetLastError();
    if (rc) return rc;
  }
  return launch_ps_pass(a, false, st);
}

}  // namespace td1c
