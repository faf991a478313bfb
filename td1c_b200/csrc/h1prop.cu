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
// out = a in + b T in + (cz0 lfield[2]) V1 in for the orbitals f >= nfcore,
// out = afc in below; V1 the unit-field laser coupling (hprod_zprod /
// hprod_pzprod of the 'dyn' orbitals).  Same tiling as the one-body kernel:
// one CTA per (orbital, 32-point radial tile), all l channels and a +-nd halo
// in shared memory.
// ---------------------------------------------------------------------------
constexpr int H1O_TILE = 32;

__global__ void __launch_bounds__(256) h1op_kernel(H1OpArgs a) {
  if (a.skip && *a.skip) return;
  extern __shared__ double smem_d[];
  const int Nr = a.Nr, L1 = a.L1, nd = a.nd, bw = 2 * nd + 1;
  const int W = H1O_TILE + 2 * nd;
  cplx* so = reinterpret_cast<cplx*>(smem_d);  // [L1][W]
  cplx* sdw = so + (size_t)L1 * W;             // [L1][TILE] radial derivative
  cplx* sh = sdw + (size_t)L1 * H1O_TILE;      // [L1][TILE] T in
  double* sb = reinterpret_cast<double*>(sh + (size_t)L1 * H1O_TILE);  // [3][bw][TILE]
  const int f = a.f0 + blockIdx.y;
  const int r0 = blockIdx.x * H1O_TILE;
  const cplx* __restrict__ in = a.in + (size_t)f * L1 * Nr;
  cplx* __restrict__ out = a.out + (size_t)f * L1 * Nr;
  if (f < a.nfcore) {
    for (int e = threadIdx.x; e < L1 * H1O_TILE; e += blockDim.x) {
      const int l = e / H1O_TILE, r = r0 + e % H1O_TILE;
      if (r < Nr) out[(size_t)l * Nr + r] = cmul(a.afc, in[(size_t)l * Nr + r]);
    }
    return;
  }
  for (int e = threadIdx.x; e < H1O_TILE * bw; e += blockDim.x) {
    const int q = e / bw, jb = e % bw;
    const int ir = r0 + q + 1;
    double k0 = 0.0, k1 = 0.0, pp = 0.0;
    if (ir <= Nr) {
      const size_t o = (size_t)bw * ir + jb;
      k0 = a.radk[o]; k1 = a.radk0[o]; pp = a.radp[o];
    }
    const int d = jb * H1O_TILE + q;
    sb[d] = k0; sb[H1O_TILE * bw + d] = k1; sb[2 * H1O_TILE * bw + d] = pp;
  }
  const int m = a.mval[f];
  const int am = m < 0 ? -m : m;
  for (int e = threadIdx.x; e < L1 * W; e += blockDim.x) {
    const int l = e / W, q = e % W;
    const int r = r0 - nd + q;
    so[e] = (r >= 0 && r < Nr) ? in[(size_t)l * Nr + r] : mkc(0.0, 0.0);
  }
  __syncthreads();
  const bool vel = a.igauge == 1;
  const bool need_t = a.b.x != 0.0 || a.b.y != 0.0;
  for (int e = threadIdx.x; e < L1 * H1O_TILE; e += blockDim.x) {
    const int l = e / H1O_TILE, q = e % H1O_TILE;
    const int r = r0 + q;
    cplx hs = mkc(0.0, 0.0), ds = mkc(0.0, 0.0);
    if (r < Nr && l >= am) {
      const int ir = r + 1;
      const int jll = max(1, ir - nd), jul = min(Nr, ir + nd);
      const double* rk = sb + (l == 0 ? 0 : H1O_TILE * bw) + q;
      const double* rp = sb + 2 * H1O_TILE * bw + q;
      const double td = a.tdiag[(size_t)l * Nr + r];
      const cplx* srow = so + (size_t)l * W + (nd + q);
      for (int jr = jll; jr <= jul; ++jr) {
        const int jb = nd + jr - ir;
        const cplx w = srow[jr - ir];
        if (need_t) {
          const double t = (jr == ir) ? td : rk[jb * H1O_TILE];
          hs.x = fma(w.x, t, hs.x); hs.y = fma(w.y, t, hs.y);
        }
        if (vel) { const double p = rp[jb * H1O_TILE]; ds.x = fma(w.x, p, ds.x); ds.y = fma(w.y, p, ds.y); }
      }
    }
    sh[(size_t)l * H1O_TILE + q] = hs;
    sdw[(size_t)l * H1O_TILE + q] = ds;
  }
  __syncthreads();
  const double zf = a.lfield ? a.lfield[2] : 0.0;
  const cplx cz = mkc(a.cz0.x * zf, a.cz0.y * zf);
  const double* __restrict__ al = a.alph + (size_t)(m + a.mmax1) * L1;
  for (int e = threadIdx.x; e < L1 * H1O_TILE; e += blockDim.x) {
    const int l = e / H1O_TILE, q = e % H1O_TILE;
    const int r = r0 + q;
    if (r >= Nr) continue;
    const double x = a.xrad[r + 1];
    const cplx* sc = so + nd + q;  // sc[l * W] = in(r, l)
    cplx h = mkc(0.0, 0.0);
    if (vel) {  // unit-field velocity-gauge coupling (hprod_pzprod.F90:114-213)
      if (l - 1 >= am) {
        const double alp = al[l - 1];
        const double t1 = -alp, t2 = (-alp * (double)l) / x;
        const cplx dwv = sdw[(size_t)(l - 1) * H1O_TILE + q], wv = sc[(size_t)(l - 1) * W];
        h.x = h.x - dwv.y * t1; h.y = h.y + dwv.x * t1;
        h.x = h.x + wv.y * t2;  h.y = h.y - wv.x * t2;
      }
      if (l >= am && l <= L1 - 2) {
        const double alp = al[l];
        const double t1 = -alp, t2 = (-alp * (double)(l + 1)) / x;
        const cplx dwv = sdw[(size_t)(l + 1) * H1O_TILE + q], wv = sc[(size_t)(l + 1) * W];
        h.x = h.x - dwv.y * t1; h.y = h.y + dwv.x * t1;
        h.x = h.x - wv.y * t2;  h.y = h.y + wv.x * t2;
      }
    } else {  // unit-field length-gauge coupling (hprod_zprod.F90:108-135)
      if (l - 1 >= am) {
        const double t = x * al[l - 1];
        const cplx wv = sc[(size_t)(l - 1) * W];
        h.x = fma(wv.x, t, h.x); h.y = fma(wv.y, t, h.y);
      }
      if (l >= am && l <= L1 - 2) {
        const double t = x * al[l];
        const cplx wv = sc[(size_t)(l + 1) * W];
        h.x = fma(wv.x, t, h.x); h.y = fma(wv.y, t, h.y);
      }
    }
    cplx o = cmul(a.a, sc[(size_t)l * W]);
    cfma(o, a.b, sh[(size_t)l * H1O_TILE + q]);
    cfma(o, cz, h);
    out[(size_t)l * Nr + r] = o;
  }
}

size_t h1op_smem(int L1, int nd) {
  const int W = H1O_TILE + 2 * nd;
  return sizeof(cplx) * ((size_t)L1 * W + 2 * (size_t)L1 * H1O_TILE) + sizeof(double) * 3 * H1O_TILE * (2 * nd + 1);
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

int launch_h1op(const H1OpArgs& a, cudaStream_t st) {
  const size_t smem = h1op_smem(a.L1, a.nd);
  static size_t cur = 0;
  if (smem > 227 * 1024) return ST_CONFIG;
  if (int e = ensure_smem(h1op_kernel, smem, cur)) return e;
  if (a.nfun - a.f0 <= 0) return 0;
  dim3 grid((a.Nr + H1O_TILE - 1) / H1O_TILE, a.nfun - a.f0);
  h1op_kernel<<<grid, 256, smem, st>>>(a);
  return (int)cudaGetLastError();
}

// ---------------------------------------------------------------------------
// x = M_l^-1 b for CG orbital columns of one l per CTA (steps 1-4 above),
// then out = x, torb = x or torb += x (orbitals >= nfcore), and the residual
// norm of the columns; the last CTA to finish sets *done = (rms < thresh).
// ---------------------------------------------------------------------------
constexpr int H1S_NT = 256;

template <int CG>
__global__ void __launch_bounds__(H1S_NT) h1solve_kernel(H1SolveArgs a) {
  if (a.check_skip && *a.done) return;
  extern __shared__ cplx s1[];
  const H1Fac& F = a.fac;
  const int Nr = a.Nr, l = blockIdx.x, ni = F.ni, nd = F.nd, nfe = F.nfe, nb = F.nb, L1 = a.L1;
  const int nint = nfe * ni;
  cplx* fr = s1;                       // [CG][Nr] right-hand side, then x
  cplx* zs = fr + (size_t)CG * Nr;     // [CG][nint] interior solutions z
  cplx* tb = zs + (size_t)CG * nint;   // [4][nb] dl, 1/d, du, du2 of channel l
  int* tp = reinterpret_cast<int*>(tb + 4 * (size_t)(nb > 0 ? nb : 1));  // [nb]
  __shared__ double red[H1S_NT / 32];
  __shared__ int col_f[CG], col_solve[CG];
  __shared__ bool last;
  const int tid = threadIdx.x;
  if (tid < CG) {
    const int fo = a.fs0 + blockIdx.y * CG + tid;
    int fv = -1, sv = 0;
    if (fo < a.nfun) {
      fv = fo;
      const int m = a.mval[fo];
      sv = l >= (m < 0 ? -m : m);  // channels l < |m| pass through (the reference skips the solve)
    }
    col_f[tid] = fv;
    col_solve[tid] = sv;
  }
  for (int q = tid; q < nb; q += H1S_NT) {
    const size_t o = (size_t)l * nb + q;
    tb[q] = F.tdl[o]; tb[nb + q] = F.tdi[o]; tb[2 * nb + q] = F.tdu[o]; tb[3 * nb + q] = F.tdu2[o];
    tp[q] = F.tpiv[o];
  }
  __syncthreads();
  for (int c = 0; c < CG; ++c) {
    const int fo = col_f[c];
    if (fo < 0) continue;
    const cplx* src = a.in + ((size_t)fo * L1 + l) * Nr;
    for (int r = tid; r < Nr; r += H1S_NT) fr[(size_t)c * Nr + r] = src[r];
  }
  __syncthreads();
  const size_t eb = (size_t)l * nfe * ni;
  // 1. z_e = A_e^-1 b(I_e)
  for (int it = tid; it < nint; it += H1S_NT) {
    const int e = it / ni, k = it % ni;
    const cplx* av = F.ainv + (eb + (size_t)e * ni) * ni + k;  // av[j * ni] = Ainv(k, j)
    cplx acc[CG];
#pragma unroll
    for (int c = 0; c < CG; ++c) acc[c] = mkc(0, 0);
    for (int j = 0; j < ni; ++j) {
      const cplx av_j = av[(size_t)j * ni];
#pragma unroll
      for (int c = 0; c < CG; ++c) cfma(acc[c], av_j, fr[(size_t)c * Nr + nd * e + j]);
    }
#pragma unroll
    for (int c = 0; c < CG; ++c) zs[(size_t)c * nint + it] = acc[c];
  }
  __syncthreads();
  // 2. bridge right-hand sides g = b(B) - M(B, I) z
  for (int it = tid; it < nb * CG; it += H1S_NT) {
    const int bb = it % nb, c = it / nb;
    if (!col_solve[c]) continue;
    const cplx* vr = F.vr + eb + (size_t)bb * ni;
    const cplx* vl = F.vl + eb + (size_t)(bb + 1) * ni;
    const cplx* zl = zs + (size_t)c * nint + (size_t)bb * ni;
    const cplx* zr = zl + ni;
    cplx s = mkc(0, 0);
    for (int j = 0; j < ni; ++j) { cfma(s, vr[j], zl[j]); cfma(s, vl[j], zr[j]); }
    cplx* g = fr + (size_t)c * Nr + nd * (bb + 1) - 1;
    *g = csub(*g, s);
  }
  __syncthreads();
  // 3. S x(B) = g (ZGTTRS algorithm on the factored tridiagonal)
  if (tid < CG && col_solve[tid] && nb > 0) {
    cplx* g = fr + (size_t)tid * Nr + nd - 1;  // g[nd * bb] = bridge bb
    const cplx *dl = tb, *di = tb + nb, *du = tb + 2 * nb, *du2 = tb + 3 * nb;
    for (int i = 0; i + 1 < nb; ++i) {
      const cplx bi = g[(size_t)nd * i], bn = g[(size_t)nd * (i + 1)];
      if (tp[i] == i) {
        g[(size_t)nd * (i + 1)] = csub(bn, cmul(dl[i], bi));
      } else {
        g[(size_t)nd * i] = bn;
        g[(size_t)nd * (i + 1)] = csub(bi, cmul(dl[i], bn));
      }
    }
    g[(size_t)nd * (nb - 1)] = cmul(g[(size_t)nd * (nb - 1)], di[nb - 1]);
    if (nb > 1) {
      const int i = nb - 2;
      g[(size_t)nd * i] = cmul(csub(g[(size_t)nd * i], cmul(du[i], g[(size_t)nd * (i + 1)])), di[i]);
    }
    for (int i = nb - 3; i >= 0; --i) {
      cplx v = csub(g[(size_t)nd * i], cmul(du[i], g[(size_t)nd * (i + 1)]));
      v = csub(v, cmul(du2[i], g[(size_t)nd * (i + 2)]));
      g[(size_t)nd * i] = cmul(v, di[i]);
    }
  }
  __syncthreads();
  // 4. x(I_e) = z_e - GL_e x(left bridge) - GR_e x(right bridge)
  for (int it = tid; it < nint * CG; it += H1S_NT) {
    const int c = it / nint, q = it % nint;
    if (!col_solve[c]) continue;
    const int e = q / ni, k = q % ni;
    cplx x = zs[(size_t)c * nint + q];
    const cplx* frc = fr + (size_t)c * Nr;
    if (e >= 1) x = csub(x, cmul(F.gl[eb + q], frc[nd * e - 1]));
    if (e + 1 < nfe) x = csub(x, cmul(F.gr[eb + q], frc[nd * (e + 1) - 1]));
    fr[(size_t)c * Nr + nd * e + k] = x;
  }
  __syncthreads();
  // write-out and residual norm
  double nrm = 0.0;
  for (int c = 0; c < CG; ++c) {
    const int fo = col_f[c];
    if (fo < 0) continue;
    const size_t row = ((size_t)fo * L1 + l) * Nr;
    const bool dyn = fo >= a.nfcore;
    for (int r = tid; r < Nr; r += H1S_NT) {
      const cplx x = fr[(size_t)c * Nr + r];
      nrm += cabs2(x);
      if (dyn) {
        if (a.out) a.out[row + r] = x;
        a.torb[row + r] = a.accumulate ? cadd(a.torb[row + r], x) : x;
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) nrm += __shfl_xor_sync(0xffffffffu, nrm, o);
  if ((tid & 31) == 0) red[tid >> 5] = nrm;
  __syncthreads();
  const int nblk = gridDim.x * gridDim.y;
  if (tid == 0) {
    double s = 0.0;
    for (int w = 0; w < H1S_NT / 32; ++w) s += red[w];
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
      const double rms = sqrt(s / a.norm_div);
      *a.done = rms < a.thresh ? 1 : 0;
      if (a.ncyc && a.check_skip) *a.ncyc += 1;
      *a.ticket = 0u;
    }
  }
}

size_t h1solve_smem(int CG, int Nr, int nfe, int ni, int nb) {
  const int nbp = nb > 0 ? nb : 1;
  return sizeof(cplx) * ((size_t)CG * Nr + (size_t)CG * nfe * ni + 4 * (size_t)nbp) + sizeof(int) * nbp;
}

int h1solve_groups(int ncol, int CG) { return (ncol + CG - 1) / CG; }

int launch_h1solve(const H1SolveArgs& a, int CG, cudaStream_t st) {
  const H1Fac& F = a.fac;
  const int ncol = a.nfun - a.fs0;
  if (ncol <= 0) return 0;
  const size_t smem = h1solve_smem(CG, a.Nr, F.nfe, F.ni, F.nb);
  if (smem > 226 * 1024) return ST_CONFIG;
  dim3 grid(a.L1, h1solve_groups(ncol, CG));
  static size_t cur[3] = {0, 0, 0};
  switch (CG) {
    case 1:
      if (int e = ensure_smem(h1solve_kernel<1>, smem, cur[0])) return e;
      h1solve_kernel<1><<<grid, H1S_NT, smem, st>>>(a);
      break;
    case 2:
      if (int e = ensure_smem(h1solve_kernel<2>, smem, cur[1])) return e;
      h1solve_kernel<2><<<grid, H1S_NT, smem, st>>>(a);
      break;
    case 4:
      if (int e = ensure_smem(h1solve_kernel<4>, smem, cur[2])) return e;
      h1solve_kernel<4><<<grid, H1S_NT, smem, st>>>(a);
      break;
    default:
      return ST_CONFIG;
  }
  return (int)cudaGetLastError();
}

// the largest column group (4, 2, 1) whose shared memory fits one CTA (the
// kernel's static arrays take well under 1 KB of the 227 KB)
int h1solve_pick_cg(int Nr, int nfe, int ni, int nb) {
  for (int cg : {4, 2, 1})
    if (h1solve_smem(cg, Nr, nfe, ni, nb) <= 226 * 1024) return cg;
  return 0;
}

}  // namespace td1c
