// h1prop.cu -- one-body propagators of the split schemes: the inverse of
// M_l = 1 + c T_l on every (orbital, l) channel and the correction cycles
// that add the laser coupling.
//
//   dpade_gen  (dpade_gen.F90:2-63)        LU of 1 + (i dt / alpha) T_l
//   h1itr_gen_cninv (h1itr_gen_cninv.F90:2-63)  LU of 1 + (i dt / 2) T_l
//   dpade_h0inv / h1itr_cninv               x <- M_l^-1 x, l >= |m|
//   dpade_prod (dpade_prod.F90:2-124), h1itr_prop (h1itr_prop.F90:2-175):
//     torb = sum_k (M^-1 zfac V)^k M^-1 b, cycles stop once
//     sqrt(sum_f |corr_f|^2 / nfun) < thresh or after maxcyc cycles.
//
// T_l is the FEDVR kinetic + nuclear (+ frozen-core Hartree) operator of
// channel l: its rows couple only points of one finite element, and
// neighbouring elements share one bridge point.  Instead of the reference's
// banded LU with partial pivoting (ZGBTRF / ZGBTRS, sequential over the
// nrad - 1 rows), the inverse is applied by static condensation:
//   1. per element e: z_e = A_e^-1 b(I_e), A_e the interior block of M
//      (nd - 1 points) -- all elements at once;
//   2. bridge right-hand sides g = b(B) - M(B, I) z;
//   3. the tridiagonal Schur complement S = M(B,B) - M(B,I) A^-1 M(I,B) over
//      the nfe - 1 bridge points, factored with row interchanges (LAPACK
//      ZGTTRF / ZGTTRS algorithm), gives x(B);
//   4. x(I_e) = z_e - (A_e^-1 M(I_e, B)) x(B).
// Steps 1, 2 and 4 are dense element-local products; only step 3 (59 points
// for 60 elements) is sequential.  The set-up inverts each interior block by
// Gauss-Jordan elimination with partial pivoting and builds S once per c.
#include "common.cuh"
#include "kernels.cuh"

namespace td1c {

__device__ __forceinline__ double cabs1(cplx z) { return fabs(z.x) + fabs(z.y); }
__device__ __forceinline__ cplx crecip(cplx z) {
  const double s = 1.0 / (z.x * z.x + z.y * z.y);
  return mkc(z.x * s, -z.y * s);
}

// M(i, j) = delta_ij + c T(j, i) for 1-based radial indices i, j (dpade_gen.F90:41-52:
// the stored A(jrad, irad) = delta + fac tmat(jb1, irad, l), tmat row irad)
struct MatM {
  const double* rk;   // radk (l = 0) or radk0 (l >= 1): (2nd+1) x (nrad+1) band, row-major by irad
  const double* td;   // tdiag of channel l [Nr]
  cplx c;
  int nd;
  __device__ cplx operator()(int i, int j) const {
    double t;
    if (i == j) t = td[i - 1];
    else t = rk[(size_t)(2 * nd + 1) * j + nd + i - j];  // row j, column i
    cplx m = mkc(c.x * t, c.y * t);
    if (i == j) m.x += 1.0;
    return m;
  }
};

// ---------------------------------------------------------------------------
// set-up 1: per (element, l) the interior inverse and its bridge couplings
// ---------------------------------------------------------------------------
constexpr int H1F_NT = 64;

__global__ void __launch_bounds__(H1F_NT) h1fac_elem_kernel(H1FacSrc s, H1Fac f) {
  extern __shared__ cplx sa[];  // [ni][2 ni] augmented [A | I], row-major
  __shared__ int piv_row;
  const int e = blockIdx.x, l = blockIdx.y, ni = f.ni, nd = f.nd, w = 2 * ni;
  const int tid = threadIdx.x;
  MatM M{l == 0 ? s.radk : s.radk0, s.tdiag + (size_t)l * s.Nr, s.c, nd};
  const int i0 = nd * e;  // irad of the element's left end
  for (int q = tid; q < ni * w; q += H1F_NT) {
    const int a = q / w, b = q % w;
    sa[q] = b < ni ? M(i0 + a + 1, i0 + b + 1) : mkc(b - ni == a ? 1.0 : 0.0, 0.0);
  }
  __syncthreads();
  bool singular = false;
  for (int p = 0; p < ni; ++p) {
    if (tid == 0) {
      int best = p;
      double bv = -1.0;
      for (int r = p; r < ni; ++r) {
        const double v = cabs1(sa[r * w + p]);
        if (v > bv) { bv = v; best = r; }
      }
      piv_row = best;
    }
    __syncthreads();
    const int pr = piv_row;
    if (pr != p)
      for (int b = tid; b < w; b += H1F_NT) { cplx t = sa[p * w + b]; sa[p * w + b] = sa[pr * w + b]; sa[pr * w + b] = t; }
    __syncthreads();
    const cplx pv = sa[p * w + p];
    if (pv.x == 0.0 && pv.y == 0.0) { singular = true; break; }
    const cplx rp = crecip(pv);
    __syncthreads();
    for (int b = tid; b < w; b += H1F_NT) sa[p * w + b] = cmul(sa[p * w + b], rp);
    __syncthreads();
    for (int q = tid; q < ni * w; q += H1F_NT) {
      const int r = q / w, b = q % w;
      if (r == p || b == p) continue;  // column p is cleared after the sweep
      const cplx fct = sa[r * w + p];
      sa[q] = csub(sa[q], cmul(fct, sa[p * w + b]));
    }
    __syncthreads();
    for (int r = tid; r < ni; r += H1F_NT)
      if (r != p) sa[r * w + p] = mkc(0.0, 0.0);
    __syncthreads();
  }
  if (singular) {
    if (tid == 0) atomicOr(s.status, ST_SINGULAR);
    return;
  }
  const size_t base = ((size_t)l * f.nfe + e) * ni;
  // ainv[..][j][k] = Ainv(k, j)
  for (int q = tid; q < ni * ni; q += H1F_NT) {
    const int j = q / ni, k = q % ni;
    f.ainv[base * ni + q] = sa[k * w + ni + j];
  }
  const bool hasl = e >= 1, hasr = e + 1 < f.nfe;
  for (int k = tid; k < ni; k += H1F_NT) {
    cplx gl = mkc(0, 0), gr = mkc(0, 0);
    for (int j = 0; j < ni; ++j) {
      const cplx a = sa[k * w + ni + j];
      if (hasl) cfma(gl, a, M(i0 + j + 1, i0));
      if (hasr) cfma(gr, a, M(i0 + j + 1, i0 + nd));
    }
    f.gl[base + k] = gl;
    f.gr[base + k] = gr;
    f.vl[base + k] = hasl ? M(i0, i0 + k + 1) : mkc(0, 0);
    f.vr[base + k] = hasr ? M(i0 + nd, i0 + k + 1) : mkc(0, 0);
  }
}

// ---------------------------------------------------------------------------
// set-up 2: per l the bridge Schur complement and its pivoted tridiagonal LU
// (LAPACK ZGTTRF algorithm; pivots by |re| + |im|)
// ---------------------------------------------------------------------------
__device__ cplx h1_dot(const cplx* a, const cplx* b, int n) {
  cplx s = mkc(0, 0);
  for (int k = 0; k < n; ++k) cfma(s, a[k], b[k]);
  return s;
}

__global__ void h1fac_bridge_kernel(H1FacSrc s, H1Fac f) {
  const int l = blockIdx.x;
  if (threadIdx.x != 0) return;
  const int nb = f.nb, ni = f.ni, nd = f.nd;
  if (nb <= 0) return;
  MatM M{l == 0 ? s.radk : s.radk0, s.tdiag + (size_t)l * s.Nr, s.c, nd};
  const size_t eb = (size_t)l * f.nfe * ni;  // element block base of channel l
  cplx* dl = f.tdl + (size_t)l * nb;
  cplx* di = f.tdi + (size_t)l * nb;
  cplx* du = f.tdu + (size_t)l * nb;
  cplx* du2 = f.tdu2 + (size_t)l * nb;
  int* ip = f.tpiv + (size_t)l * nb;
  // S(bb, bb), S(bb, bb+1) in du, S(bb+1, bb) in dl; bridge bb sits at irad nd (bb + 1)
  for (int bb = 0; bb < nb; ++bb) {
    const int ib = nd * (bb + 1);
    cplx d = M(ib, ib);
    d = csub(d, h1_dot(f.vr + eb + (size_t)bb * ni, f.gr + eb + (size_t)bb * ni, ni));
    d = csub(d, h1_dot(f.vl + eb + (size_t)(bb + 1) * ni, f.gl + eb + (size_t)(bb + 1) * ni, ni));
    di[bb] = d;
    du2[bb] = mkc(0, 0);
    if (bb + 1 < nb) {
      du[bb] = csub(M(ib, ib + nd), h1_dot(f.vl + eb + (size_t)(bb + 1) * ni, f.gr + eb + (size_t)(bb + 1) * ni, ni));
      dl[bb] = csub(M(ib + nd, ib), h1_dot(f.vr + eb + (size_t)(bb + 1) * ni, f.gl + eb + (size_t)(bb + 1) * ni, ni));
    } else {
      du[bb] = mkc(0, 0);
      dl[bb] = mkc(0, 0);
    }
  }
  // factorisation in place (di holds d until the reciprocals are taken)
  for (int i = 0; i + 1 < nb; ++i) {
    if (cabs1(di[i]) >= cabs1(dl[i])) {
      ip[i] = i;
      if (di[i].x != 0.0 || di[i].y != 0.0) {
        const cplx fct = cmul(dl[i], crecip(di[i]));
        dl[i] = fct;
        di[i + 1] = csub(di[i + 1], cmul(fct, du[i]));
      }
    } else {
      ip[i] = i + 1;
      const cplx fct = cmul(di[i], crecip(dl[i]));
      di[i] = dl[i];
      dl[i] = fct;
      const cplx tmp = du[i];
      du[i] = di[i + 1];
      di[i + 1] = csub(tmp, cmul(fct, di[i + 1]));
      if (i + 2 < nb) {
        du2[i] = du[i + 1];
        du[i + 1] = mkc(-(fct.x * du[i + 1].x - fct.y * du[i + 1].y), -(fct.x * du[i + 1].y + fct.y * du[i + 1].x));
      }
    }
  }
  ip[nb - 1] = nb - 1;
  for (int i = 0; i < nb; ++i) {
    if (di[i].x == 0.0 && di[i].y == 0.0) { atomicOr(s.status, ST_SINGULAR); return; }
    di[i] = crecip(di[i]);
  }
}

int launch_h1fac(const H1FacSrc& s, H1Fac& f, cudaStream_t st) {
  const size_t smem = sizeof(cplx) * (size_t)f.ni * 2 * f.ni;
  if (smem > 48 * 1024) return ST_CONFIG;
  h1fac_elem_kernel<<<dim3(f.nfe, f.L1), H1F_NT, smem, st>>>(s, f);
  h1fac_bridge_kernel<<<f.L1, 32, 0, st>>>(s, f);
  return (int)cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Application of M^-1 with the correction cycles, element by element.
//
// One pass of the element kernel, per (finite element e, chunk of LC l):
//   1. x on the element's points (both bridges included) for l in the chunk
//      and its l +- 1 halo: the input vector (first pass), or the previous
//      correction finished from its interior part z and bridge values xb,
//      x(I_e) = z_e - GL_e xb(left) - GR_e xb(right);
//   2. finished corrections go to torb (= or +=) and into the residual norm;
//      each point counted once: interior points and the element's left bridge;
//   3. the next right-hand side  r = a x + b T x + cz V1 x  (V1 the unit-field
//      laser coupling l <-> l +- 1, T the kinetic + nuclear band) on the
//      element's points.  T and the radial derivative in V1 couple only the
//      points of one element, so a bridge point gets each element's share
//      from that element's CTA; its diagonal and point-local terms come from
//      the element to its right (the bridge's owner);
//   4. z_e = A_e^-1 r(I_e) and the bridge shares r(bridge) - v.z_e.
// The bridge kernel, per l, adds the two shares of every bridge point and
// solves the tridiagonal bridge system for xb.  Channels l < |m| pass
// through (z = r, xb = r), as the reference skips their solve.  z is read
// and written by the same pass (halo rows of the neighbouring chunks), so
// consecutive passes alternate between two z buffers.
// ---------------------------------------------------------------------------
constexpr int H1E_NT = 256;
constexpr int H1E_LC = 3;   // l channels per CTA (about 64 KB of shared memory: 3 CTAs per SM)
constexpr int H1E_FG = 3;   // orbital groups of the interior solve
constexpr int H1E_RMAX = 6; // right-hand sides a thread holds while the band products are read

__device__ __forceinline__ void h1_dmma(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

// shared memory of one element pass; ZI (the previous z rows, read once in
// step 1) aliases R and Z, which are written only afterwards
struct H1ElemSmem {
  int np, nf, lh;  // points per element (nd + 1), orbitals, halo rows (LC + 2)
  __host__ __device__ int ni() const { return np - 2; }
  __host__ __device__ size_t x_off() const { return 0; }
  __host__ __device__ size_t r_off() const { return x_off() + (size_t)nf * lh * np; }
  __host__ __device__ size_t z_off() const { return r_off() + (size_t)nf * H1E_LC * np; }
  __host__ __device__ size_t rz_end() const {
    const size_t rz = z_off() + (size_t)nf * H1E_LC * ni();
    const size_t zi = r_off() + (size_t)nf * lh * ni();
    return rz > zi ? rz : zi;
  }
  __host__ __device__ size_t ts_off() const { return rz_end(); }
  __host__ __device__ size_t xb_off() const { return ts_off() + (size_t)nf * H1E_LC * np; }
  __host__ __device__ size_t g_off() const { return xb_off() + (size_t)nf * lh * 2; }
  __host__ __device__ size_t v_off() const { return g_off() + (size_t)2 * lh * ni(); }
  __host__ __device__ size_t cplx_count() const { return v_off() + (size_t)2 * H1E_LC * ni(); }
  __host__ __device__ size_t dbl_count() const { return (size_t)3 * np * np + 2 * np + (size_t)H1E_LC * np + (size_t)nf * lh; }
  __host__ __device__ size_t bytes() const { return sizeof(cplx) * cplx_count() + sizeof(double) * dbl_count(); }
};

// asynchronous global -> shared copies (LDGSTS); a copy with ok == false
// reads nothing and zero-fills its destination
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void cpa16(void* dst, const void* src, bool ok) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst)), "l"(src), "r"(ok ? 16u : 0u) : "memory");
}
__device__ __forceinline__ void cpa8(void* dst, const void* src, bool ok) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(smem_u32(dst)), "l"(src), "r"(ok ? 8u : 0u) : "memory");
}
__device__ __forceinline__ void cpa_wait_all() {
  asm volatile("cp.async.commit_group;" ::: "memory");
  asm volatile("cp.async.wait_group 0;" ::: "memory");
}

template <int NDT>
__global__ void __launch_bounds__(H1E_NT, 3) h1elem_kernel(H1ElemArgs a) {
  if (a.check_skip && *a.done) return;
  extern __shared__ cplx sm[];
  const H1Fac& F = a.fac;
  const int nd = NDT > 0 ? NDT : F.nd;
  const int np = nd + 1, ni = nd - 1, nfe = F.nfe, nb = F.nb, L1 = a.L1, Nr = a.Nr, nfun = a.nfun;
  const int e = blockIdx.x, l0 = blockIdx.y * H1E_LC, lh = H1E_LC + 2;
  const int tid = threadIdx.x;
  const H1ElemSmem lay{np, nfun, lh};
  cplx* X = sm + lay.x_off();     // [f][lh][np]  rows l0-1 .. l0+LC
  cplx* R = sm + lay.r_off();     // [f][LC][np]
  cplx* Z = sm + lay.z_off();     // [f][LC][ni]
  cplx* ZI = sm + lay.r_off();    // [f][lh][ni] previous z (step 1 only; aliases R, Z)
  cplx* TS = sm + lay.ts_off();   // [f][LC][np] torb before the update
  cplx* XB = sm + lay.xb_off();   // [f][lh][2] bridge values left / right of the element
  cplx* GLs = sm + lay.g_off();   // [lh][ni]
  cplx* GRs = GLs + lh * ni;      // [lh][ni]
  cplx* VLs = sm + lay.v_off();   // [LC][ni]
  cplx* VRs = VLs + H1E_LC * ni;  // [LC][ni]
  double* Pb = reinterpret_cast<double*>(sm + lay.cplx_count());  // [np][np] derivative, off-diagonal
  double* Tb0 = Pb + np * np;     // [np][np] kinetic off-diagonal, l = 0 (radk)
  double* Tb1 = Tb0 + np * np;    // l >= 1 (radk0)
  double* Pd = Tb1 + np * np;     // [np] derivative diagonal of owned points
  double* Xr = Pd + np;           // [np] radial coordinate
  double* TD = Xr + np;           // [LC][np] kinetic diagonal
  double* AL = TD + H1E_LC * np;  // [f][lh] alpha_lm of l0-1 .. l0+LC
  __shared__ double red[H1E_NT / 32];
  __shared__ bool last;
  const int ir0 = nd * e;  // irad of local point 0
  const cplx* z_in = a.z_in;
  cplx* z_out = a.z_out;
  int f_fin = a.f_fin, accumulate = a.accumulate;
  if (a.iter_mode == 1) {
    const int k = *a.iter + 1;
    f_fin = k == 1 ? a.f_first : a.nfcore;
    accumulate = k > 1;
    z_in = ((k - 1) & 1) ? a.zb1 : a.zb0;
    z_out = (k & 1) ? a.zb1 : a.zb0;
  } else if (a.iter_mode == 2) {
    z_in = (*a.iter & 1) ? a.zb1 : a.zb0;
  }
  const int f_lo = a.finalize ? min(f_fin, a.f_rhs) : a.f_rhs;
  const size_t eb = (size_t)e * ni;
  const int bw = 2 * nd + 1;
  auto valid = [&](int ip) { return ip >= 1 && ip <= Nr; };
  // 0. every table and input of the pass, copied asynchronously
  for (int q2 = tid; q2 < np * np; q2 += H1E_NT) {
    const int p = q2 / np, q = q2 % np, ip = ir0 + p, iq = ir0 + q;
    const bool ok = p != q && valid(ip) && valid(iq);
    const size_t o = ok ? (size_t)bw * ip + nd + iq - ip : 0;
    cpa8(Pb + q2, a.radp + o, ok);
    cpa8(Tb0 + q2, a.radk + o, ok);
    cpa8(Tb1 + q2, a.radk0 + o, ok);
  }
  for (int p = tid; p < np; p += H1E_NT) {
    const int ip = ir0 + p;
    const bool ok = valid(ip);
    cpa8(Pd + p, a.radp + (ok ? (size_t)bw * ip + nd : 0), ok && p != nd);
    cpa8(Xr + p, a.xrad + (ok ? ip : 0), ok);
  }
  for (int q2 = tid; q2 < H1E_LC * np; q2 += H1E_NT) {
    const int lc = q2 / np, p = q2 % np, l = l0 + lc, ip = ir0 + p;
    const bool ok = l < L1 && valid(ip);
    cpa8(TD + q2, a.tdiag + (ok ? (size_t)l * Nr + ip - 1 : 0), ok);
  }
  for (int q2 = tid; q2 < nfun * lh; q2 += H1E_NT) {
    const int f = q2 / lh, lq = q2 % lh, l = l0 - 1 + lq;
    const bool lok = l >= 0 && l < L1;
    cpa8(AL + q2, a.alph + (lok ? (size_t)(a.mv[f] + a.mmax1) * L1 + l : 0), lok);
    const bool fok = a.finalize && f >= f_lo && lok;
    const size_t row = (size_t)f * L1 + (lok ? l : 0);
    cpa16(XB + 2 * q2, a.xb + (fok && e >= 1 ? row * nb + e - 1 : 0), fok && e >= 1);
    cpa16(XB + 2 * q2 + 1, a.xb + (fok && e + 1 < nfe ? row * nb + e : 0), fok && e + 1 < nfe);
  }
  if (a.finalize) {
    for (int q2 = tid; q2 < lh * ni; q2 += H1E_NT) {
      const int lq = q2 / ni, k = q2 % ni, l = l0 - 1 + lq;
      const bool ok = l >= 0 && l < L1;
      const size_t gi = ok ? (size_t)l * nfe * ni + eb + k : 0;
      cpa16(GLs + q2, F.gl + gi, ok);
      cpa16(GRs + q2, F.gr + gi, ok);
    }
    for (int q2 = tid; q2 < nfun * lh * ni; q2 += H1E_NT) {
      const int f = q2 / (lh * ni), lq = (q2 / ni) % lh, k = q2 % ni, l = l0 - 1 + lq;
      const bool ok = f >= f_lo && l >= 0 && l < L1;
      cpa16(ZI + q2, z_in + (ok ? ((size_t)f * L1 + l) * nfe * ni + eb + k : 0), ok);
    }
    if (accumulate) {
      for (int q2 = tid; q2 < nfun * H1E_LC * np; q2 += H1E_NT) {
        const int f = q2 / (H1E_LC * np), lc = (q2 / np) % H1E_LC, p = q2 % np, l = l0 + lc, ip = ir0 + p;
        const bool ok = f >= f_fin && f >= a.nfcore && l < L1 && p != nd && valid(ip);
        cpa16(TS + q2, a.torb + (ok ? ((size_t)f * L1 + l) * Nr + ip - 1 : 0), ok);
      }
    }
  } else {
    for (int q2 = tid; q2 < nfun * lh * np; q2 += H1E_NT) {
      const int f = q2 / (lh * np), lq = (q2 / np) % lh, p = q2 % np, l = l0 - 1 + lq, ip = ir0 + p;
      const bool ok = f >= f_lo && l >= 0 && l < L1 && valid(ip);
      cpa16(X + q2, a.in + (ok ? ((size_t)f * L1 + l) * Nr + ip - 1 : 0), ok);
    }
  }
  if (a.make_rhs) {
    for (int q2 = tid; q2 < H1E_LC * ni; q2 += H1E_NT) {
      const int lc = q2 / ni, k = q2 % ni, l = l0 + lc;
      const bool ok = l < L1;
      const size_t vi = ok ? (size_t)l * nfe * ni + eb + k : 0;
      cpa16(VLs + q2, F.vl + vi, ok);
      cpa16(VRs + q2, F.vr + vi, ok);
    }
  }
  cpa_wait_all();
  __syncthreads();
  // 1. x on the element for l0-1 .. l0+LC (the previous correction finished)
  if (a.finalize) {
    for (int it = tid; it < nfun * lh * np; it += H1E_NT) {
      const int f = it / (lh * np), lq = (it / np) % lh, p = it % np;
      const int l = l0 - 1 + lq, ip = ir0 + p;
      cplx x = mkc(0, 0);
      if (f >= f_lo && l >= 0 && l < L1 && valid(ip)) {
        const cplx* xbr = XB + 2 * ((size_t)f * lh + lq);
        if (p == 0) {
          x = xbr[0];
        } else if (p == nd) {
          x = xbr[1];
        } else {
          const int k = p - 1;
          const int m = a.mv[f];
          x = ZI[((size_t)f * lh + lq) * ni + k];
          if (l >= (m < 0 ? -m : m)) {
            x = csub(x, cmul(GLs[lq * ni + k], xbr[0]));
            x = csub(x, cmul(GRs[lq * ni + k], xbr[1]));
          }
        }
      }
      X[it] = x;
    }
    __syncthreads();
  }
  // 2. finished corrections: torb and the residual norm (owned points)
  if (a.finalize) {
    double nrm = 0.0;
    for (int it = tid; it < nfun * H1E_LC * np; it += H1E_NT) {
      const int f = it / (H1E_LC * np), lc = (it / np) % H1E_LC, p = it % np;
      const int l = l0 + lc, ip = ir0 + p;
      if (f < f_fin || l >= L1 || p == nd || !valid(ip)) continue;
      const cplx x = X[((size_t)f * lh + lc + 1) * np + p];
      nrm += cabs2(x);
      if (f >= a.nfcore) a.torb[((size_t)f * L1 + l) * Nr + ip - 1] = accumulate ? cadd(TS[it], x) : x;
    }
    for (int o = 16; o > 0; o >>= 1) nrm += __shfl_xor_sync(0xffffffffu, nrm, o);
    if ((tid & 31) == 0) red[tid >> 5] = nrm;
  }
  // 3. right-hand side r = a x + b T x + cz V1 x on the element's points
  const double zf = a.lfield ? a.lfield[2] : 0.0;
  const cplx cz = mkc(a.cz0.x * zf, a.cz0.y * zf);
  const bool do_t = a.b.x != 0.0 || a.b.y != 0.0;
  const bool do_v = cz.x != 0.0 || cz.y != 0.0;
  const bool vel = a.igauge == 1;
  // The band products of the element, T x (kinetic, l >= 1, own rows) and P x (radial
  // derivative, every staged row), run on the FP64 tensor cores: C(p, n) = sum_q A(p, q) B(q, n)
  // with A = Tb1 or Pb and B's columns the (re, im) parts of the staged rows, as m8n8k4 DMMA
  // tiles (rows and depth padded to 8 and 4 with zeros). T x goes to TS (free after step 2),
  // P x over R and Z (written only after the products are read; the right-hand sides wait in
  // registers). l = 0 keeps the scalar product with its own table.
  const int n_t = nfun * H1E_LC, n_p = nfun * lh, n_it = nfun * H1E_LC * np;
  const bool gem = a.make_rhs && np <= 24 && n_it <= H1E_RMAX * H1E_NT && (do_t || (do_v && vel)) &&
                   (size_t)n_p * np <= lay.rz_end() - lay.r_off();
  cplx* TXs = TS;  // [nfun][LC][np]
  cplx* PXs = R;   // [nfun][lh][np]
  if (gem) {
    __syncthreads();  // step 2 has read TS
    const int warp = tid >> 5, lane = tid & 31, gid = lane >> 2, tig = lane & 3;
    const int MT = (np + 7) >> 3, KS = (np + 3) >> 2;
    const int ntT = do_t ? (n_t + 3) >> 2 : 0, ntP = (do_v && vel) ? (n_p + 3) >> 2 : 0;
    for (int item = warp; item < MT * (ntT + ntP); item += H1E_NT / 32) {
      const int mt = item % MT, q = item / MT;
      const bool isT = q < ntT;
      const int nt = isT ? q : q - ntT, nrows = isT ? n_t : n_p;
      const double* A = isT ? Tb1 : Pb;
      const int brow = 4 * nt + (gid >> 1), part = gid & 1;  // this lane's B column: a complex row, re | im
      int xrow = -1;
      if (brow < nrows) xrow = isT ? (brow / H1E_LC) * lh + brow % H1E_LC + 1 : brow;
      const double* xb = reinterpret_cast<const double*>(X) + (xrow >= 0 ? (size_t)xrow * np * 2 + part : 0);
      const int pa = 8 * mt + gid;
      double c0 = 0.0, c1 = 0.0;
      for (int ks = 0; ks < KS; ++ks) {
        const int qq = 4 * ks + tig;
        const double av = (pa < np && qq < np) ? A[pa * np + qq] : 0.0;
        const double bv = (xrow >= 0 && qq < np) ? xb[2 * qq] : 0.0;
        h1_dmma(c0, c1, av, bv);
      }
      const int crow = 4 * nt + tig;  // C(pa, 8 nt + 2 tig + {0, 1}): Re, Im of complex row crow
      if (pa < np && crow < nrows) (isT ? TXs : PXs)[(size_t)crow * np + pa] = mkc(c0, c1);
    }
    __syncthreads();
  }
  // the right-hand side at (orbital, own row, point) of item it (f >= f_rhs, l < L1)
  auto rhs_of = [&](int it) -> cplx {
    const int f = it / (H1E_LC * np), lc = (it / np) % H1E_LC, p = it % np;
    const int l = l0 + lc, ip = ir0 + p;
    cplx r = mkc(0, 0);
    if (valid(ip)) {
      const int m = a.mv[f], am = m < 0 ? -m : m;
      const bool owner = p != nd;       // the right bridge belongs to the next element
      const bool dyn = f >= a.nfcore;   // frozen-core rows take the a-term only
      const cplx* xl = X + ((size_t)f * lh + lc + 1) * np;  // x(l, .)
      if (owner) r = cmul(a.a, xl[p]);
      if (do_t && dyn && l >= am) {
        cplx t = mkc(0, 0);
        if (gem && l > 0) {
          t = TXs[((size_t)f * H1E_LC + lc) * np + p];
        } else {
          const double* tb = (l == 0 ? Tb0 : Tb1) + p * np;
          for (int q = 0; q < np; ++q) { t.x = fma(tb[q], xl[q].x, t.x); t.y = fma(tb[q], xl[q].y, t.y); }
        }
        if (owner) {
          const double d = TD[lc * np + p];
          t.x = fma(d, xl[p].x, t.x); t.y = fma(d, xl[p].y, t.y);
        }
        cfma(r, a.b, t);
      }
      if (do_v && dyn) {
        const double* alq = AL + (size_t)f * lh;  // alq[lq] = alpha(l0 - 1 + lq)
        const double xr = Xr[p];
        cplx h = mkc(0, 0);
        for (int side = 0; side < 2; ++side) {
          // side 0: coupling from l-1 (l-1 >= |m|); side 1: from l+1 (l >= |m|, l+1 < L1)
          if (side == 0 ? (l - 1 < am) : (l < am || l + 1 >= L1)) continue;
          const double alp = side == 0 ? alq[lc] : alq[lc + 1];
          const int lq = lc + (side == 0 ? 0 : 2);
          const cplx* xs = X + ((size_t)f * lh + lq) * np;
          if (vel) {
            // -i alpha (d/dr x_s) (this element's share) and -/+ i alpha (l_s/r) x_s (owner)
            cplx dw = mkc(0, 0);
            if (gem) {
              dw = PXs[((size_t)f * lh + lq) * np + p];
            } else {
              const double* pr = Pb + p * np;
              for (int q = 0; q < np; ++q) { dw.x = fma(pr[q], xs[q].x, dw.x); dw.y = fma(pr[q], xs[q].y, dw.y); }
            }
            dw.x = fma(Pd[p], xs[p].x, dw.x); dw.y = fma(Pd[p], xs[p].y, dw.y);
            const double t1 = -alp;
            h.x = h.x - dw.y * t1; h.y = h.y + dw.x * t1;
            if (owner) {
              const double t2 = side == 0 ? (-alp * (double)l) / xr : (-alp * (double)(l + 1)) / xr;
              const cplx wv = xs[p];
              if (side == 0) { h.x = h.x + wv.y * t2; h.y = h.y - wv.x * t2; }
              else { h.x = h.x - wv.y * t2; h.y = h.y + wv.x * t2; }
            }
          } else if (owner) {
            const double t = xr * alp;
            h.x = fma(xs[p].x, t, h.x); h.y = fma(xs[p].y, t, h.y);
          }
        }
        cfma(r, cz, h);
      }
    }
    return r;
  };
  if (a.make_rhs) {
    if (gem) {
      cplx racc[H1E_RMAX];
#pragma unroll
      for (int k = 0; k < H1E_RMAX; ++k) {
        const int it = tid + k * H1E_NT;
        racc[k] = mkc(0, 0);
        if (it >= n_it) continue;
        const int f = it / (H1E_LC * np), lc = (it / np) % H1E_LC;
        if (f >= a.f_rhs && l0 + lc < L1) racc[k] = rhs_of(it);
      }
      __syncthreads();  // every product has been read: R may be written
#pragma unroll
      for (int k = 0; k < H1E_RMAX; ++k) {
        const int it = tid + k * H1E_NT;
        if (it >= n_it) continue;
        const int f = it / (H1E_LC * np), lc = (it / np) % H1E_LC;
        if (f >= a.f_rhs && l0 + lc < L1) R[it] = racc[k];
      }
    } else {
      for (int it = tid; it < n_it; it += H1E_NT) {
        const int f = it / (H1E_LC * np), lc = (it / np) % H1E_LC;
        if (f >= a.f_rhs && l0 + lc < L1) R[it] = rhs_of(it);
      }
    }
  }
  __syncthreads();
  if (a.make_rhs) {
    // 4. z_e = A_e^-1 r(I_e) for every orbital column at once: complex DMMA tiles (rows the
    //    element's interior points, columns the orbitals, four real products per depth step in
    //    separate accumulators); channels below |m| pass through
    const int nfo = nfun - a.f_rhs;
    if (ni <= 24 && nfo <= 16) {
      const int warp = tid >> 5, lane = tid & 31, gid = lane >> 2, tig = lane & 3;
      const int MT = (ni + 7) >> 3, KS = (ni + 3) >> 2, NTo = (nfo + 7) >> 3;
      for (int item = warp; item < H1E_LC * MT * NTo; item += H1E_NT / 32) {
        const int lc = item / (MT * NTo), mt = (item / NTo) % MT, nt = item % NTo;
        const int l = l0 + lc;
        if (l >= L1) continue;  // the whole warp: one item per warp
        const cplx* Ag = F.ainv + ((size_t)l * nfe * ni + eb) * ni;  // (A_e^-1)(k, j) at [j ni + k], L2-resident
        const int ka = 8 * mt + gid;            // this lane's A row: interior point ka
        const int fb = a.f_rhs + 8 * nt + gid;  // this lane's B column: orbital fb
        const cplx* rb = R + ((size_t)(fb < nfun ? fb : 0) * H1E_LC + lc) * np + 1;
        double acc[4][2] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
        for (int ks = 0; ks < KS; ++ks) {
          const int j = 4 * ks + tig;
          const cplx av = (ka < ni && j < ni) ? __ldg(Ag + (size_t)j * ni + ka) : mkc(0, 0);  // Ainv(ka, j)
          const cplx bv = (fb < nfun && j < ni) ? rb[j] : mkc(0, 0);
          h1_dmma(acc[0][0], acc[0][1], av.x, bv.x);
          h1_dmma(acc[1][0], acc[1][1], av.y, -bv.y);
          h1_dmma(acc[2][0], acc[2][1], av.x, bv.y);
          h1_dmma(acc[3][0], acc[3][1], av.y, bv.x);
        }
        if (ka < ni) {
#pragma unroll
          for (int i = 0; i < 2; ++i) {  // C(ka, 8 nt + 2 tig + i): orbital f
            const int f = a.f_rhs + 8 * nt + 2 * tig + i;
            if (f >= nfun) continue;
            const int m = a.mv[f];
            cplx zv = mkc(acc[0][i] + acc[1][i], acc[2][i] + acc[3][i]);
            if (l < (m < 0 ? -m : m)) zv = R[((size_t)f * H1E_LC + lc) * np + 1 + ka];
            Z[((size_t)f * H1E_LC + lc) * ni + ka] = zv;
            z_out[((size_t)f * L1 + l) * nfe * ni + eb + ka] = zv;
          }
        }
      }
    } else {
      for (int it = tid; it < H1E_LC * ni * H1E_FG; it += H1E_NT) {
        const int g = it / (H1E_LC * ni), lc = (it / ni) % H1E_LC, k = it % ni;
        const int l = l0 + lc;
        if (l >= L1) continue;
        const cplx* av = F.ainv + ((size_t)l * nfe * ni + eb) * ni + k;  // av[j * ni] = Ainv(k, j)
        for (int f = a.f_rhs + g; f < nfun; f += H1E_FG) {
          const int m = a.mv[f];
          const cplx* rf = R + ((size_t)f * H1E_LC + lc) * np + 1;
          cplx zv;
          if (l < (m < 0 ? -m : m)) {
            zv = rf[k];
          } else {
            zv = mkc(0, 0);
#pragma unroll
            for (int j = 0; j < (NDT > 0 ? NDT - 1 : 0); ++j) cfma(zv, av[(size_t)j * ni], rf[j]);
            for (int j = (NDT > 0 ? NDT - 1 : 0); j < ni; ++j) cfma(zv, av[(size_t)j * ni], rf[j]);
          }
          Z[((size_t)f * H1E_LC + lc) * ni + k] = zv;
          z_out[((size_t)f * L1 + l) * nfe * ni + eb + k] = zv;
        }
      }
    }
    __syncthreads();
    // bridge shares: left (e >= 1) r(0) - vL.z, right (e < nfe - 1) r(nd) - vR.z
    for (int it = tid; it < nfun * H1E_LC * 2; it += H1E_NT) {
      const int f = it / (H1E_LC * 2), lc = (it / 2) % H1E_LC, side = it % 2;
      const int l = l0 + lc;
      if (f < a.f_rhs || l >= L1) continue;
      if (side == 0 ? e < 1 : e + 1 >= nfe) continue;
      const int m = a.mv[f];
      const cplx* rf = R + ((size_t)f * H1E_LC + lc) * np;
      cplx c = side == 0 ? rf[0] : rf[nd];
      if (l >= (m < 0 ? -m : m)) {
        const cplx* v = (side == 0 ? VLs : VRs) + (size_t)lc * ni;
        const cplx* zr = Z + ((size_t)f * H1E_LC + lc) * ni;
        cplx s = mkc(0, 0);
        for (int k = 0; k < ni; ++k) cfma(s, v[k], zr[k]);
        c = csub(c, s);
      }
      a.cb[(((size_t)f * L1 + l) * nfe + e) * 2 + side] = c;
    }
  }
  // residual norm of the finished corrections: the last CTA decides
  if (a.finalize && a.do_norm) {
    const int nblk = gridDim.x * gridDim.y;
    if (tid == 0) {
      double s = 0.0;
      for (int w = 0; w < H1E_NT / 32; ++w) s += red[w];
      a.partial[blockIdx.y * gridDim.x + blockIdx.x] = s;
      __threadfence();
      last = atomicAdd(a.ticket, 1u) == (unsigned)(nblk - 1);
    }
    __syncthreads();
    if (last && tid < 32) {
      __threadfence();
      double s = 0.0;
      for (int b = tid; b < nblk; b += 32) s += __ldcg(a.partial + b);
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      if (tid == 0) {
        *a.done = sqrt(s / a.norm_div) < a.thresh ? 1 : 0;
        *a.ticket = 0u;
      }
    }
  }
}

// per l: bridge right-hand sides from the two element shares, then the
// pivoted tridiagonal solve (ZGTTRS algorithm) for every orbital column
constexpr int H1B_NT = 256;

__global__ void __launch_bounds__(H1B_NT) h1bridge_kernel(H1ElemArgs a) {
  if (a.check_skip && *a.done) return;
  extern __shared__ cplx sb2[];
  const H1Fac& F = a.fac;
  const int l = blockIdx.x, nb = F.nb, nfe = F.nfe, L1 = a.L1, nfun = a.nfun, tid = threadIdx.x;
  if (nb <= 0) return;
  cplx* dl = sb2;
  cplx* di = dl + nb;
  cplx* du = di + nb;
  cplx* du2 = du + nb;
  cplx* g = du2 + nb;  // [nfun][nb]
  int* ip = reinterpret_cast<int*>(g + (size_t)3 * nfun * nb);
  // factors and both bridge shares copied asynchronously; the shares are
  // added once they have landed
  cplx* gs = g + (size_t)nfun * nb;  // [nfun][nb][2] shares (right of element b, left of b+1)
  for (int q = tid; q < nb; q += H1B_NT) {
    const size_t o = (size_t)l * nb + q;
    cpa16(dl + q, F.tdl + o, true); cpa16(di + q, F.tdi + o, true);
    cpa16(du + q, F.tdu + o, true); cpa16(du2 + q, F.tdu2 + o, true);
  }
  for (int it = tid; it < nfun * nb; it += H1B_NT) {
    const int f = it / nb, b = it % nb;
    const bool ok = f >= a.f_rhs;
    const size_t c0 = ((size_t)f * L1 + l) * nfe;
    cpa16(gs + 2 * it, a.cb + (ok ? (c0 + b) * 2 + 1 : 0), ok);
    cpa16(gs + 2 * it + 1, a.cb + (ok ? (c0 + b + 1) * 2 : 0), ok);
  }
  for (int q = tid; q < nb; q += H1B_NT) ip[q] = F.tpiv[(size_t)l * nb + q];
  cpa_wait_all();
  __syncthreads();
  for (int it = tid; it < nfun * nb; it += H1B_NT) g[it] = cadd(gs[2 * it], gs[2 * it + 1]);
  __syncthreads();
  if (tid == 0 && l == 0 && a.ncyc && a.check_skip) atomicAdd(a.ncyc, 1);
  const int f = a.f_rhs + tid;
  if (f >= nfun) return;
  const int m = a.mval[f];
  cplx* x = g + (size_t)f * nb;
  if (l >= (m < 0 ? -m : m)) {
    for (int i = 0; i + 1 < nb; ++i) {
      const cplx bi = x[i], bn = x[i + 1];
      if (ip[i] == i) {
        x[i + 1] = csub(bn, cmul(dl[i], bi));
      } else {
        x[i] = bn;
        x[i + 1] = csub(bi, cmul(dl[i], bn));
      }
    }
    x[nb - 1] = cmul(x[nb - 1], di[nb - 1]);
    if (nb > 1) x[nb - 2] = cmul(csub(x[nb - 2], cmul(du[nb - 2], x[nb - 1])), di[nb - 2]);
    for (int i = nb - 3; i >= 0; --i) {
      cplx v = csub(x[i], cmul(du[i], x[i + 1]));
      v = csub(v, cmul(du2[i], x[i + 2]));
      x[i] = cmul(v, di[i]);
    }
  }
  cplx* out = a.xb + ((size_t)f * L1 + l) * nb;
  for (int b = 0; b < nb; ++b) out[b] = x[b];
}

// raise a kernel's dynamic shared memory limit to at least smem (once per size)
template <typename K>
int ensure_smem(K kernel, size_t smem, size_t& cur) {
  if (smem <= 48 * 1024 || smem <= cur) return 0;
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return (int)e;
  cur = smem;
  return 0;
}

size_t h1elem_smem(int nd, int nfun) { return H1ElemSmem{nd + 1, nfun, H1E_LC + 2}.bytes(); }

template <int NDT>
int launch_h1elem_t(const H1ElemArgs& a, cudaStream_t st) {
  static size_t cur = 0;
  const size_t smem = h1elem_smem(a.fac.nd, a.nfun);
  if (smem > 220 * 1024) return ST_CONFIG;
  if (int e = ensure_smem(h1elem_kernel<NDT>, smem, cur)) return e;
  dim3 grid(a.fac.nfe, (a.L1 + H1E_LC - 1) / H1E_LC);
  h1elem_kernel<NDT><<<grid, H1E_NT, smem, st>>>(a);
  return (int)cudaGetLastError();
}

int launch_h1elem(const H1ElemArgs& a, cudaStream_t st) {
  switch (a.fac.nd) {  // 21-, 9- and 8-point Lobatto elements get the unrolled inverse rows
    case 20: return launch_h1elem_t<20>(a, st);
    case 8: return launch_h1elem_t<8>(a, st);
    case 7: return launch_h1elem_t<7>(a, st);
    default: return launch_h1elem_t<0>(a, st);
  }
}

int launch_h1bridge(const H1ElemArgs& a, cudaStream_t st) {
  if (a.fac.nb <= 0) return 0;
  if (a.nfun - a.f_rhs > H1B_NT) return ST_CONFIG;
  const size_t smem = sizeof(cplx) * (size_t)a.fac.nb * (4 + 3 * a.nfun) + sizeof(int) * a.fac.nb;
  static size_t cur = 0;
  if (smem > 220 * 1024) return ST_CONFIG;
  if (int e = ensure_smem(h1bridge_kernel, smem, cur)) return e;
  h1bridge_kernel<<<a.L1, H1B_NT, smem, st>>>(a);
  return (int)cudaGetLastError();
}

__global__ void h1loop_ctl_kernel(int* iter, const int* done, int maxcyc, cudaGraphConditionalHandle h) {
  const int k = *iter + 1;
  *iter = k;
  cudaGraphSetConditional(h, (*done == 0 && k < maxcyc) ? 1u : 0u);
}

int launch_h1loop_ctl(int* iter, const int* done, int maxcyc, cudaGraphConditionalHandle h, cudaStream_t st) {
  h1loop_ctl_kernel<<<1, 1, 0, st>>>(iter, done, maxcyc, h);
  return (int)cudaGetLastError();
}

size_t h1elem_partials(int nfe, int L1) { return (size_t)nfe * ((L1 + H1E_LC - 1) / H1E_LC); }

}  // namespace td1c
