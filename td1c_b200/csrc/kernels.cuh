// kernels.cuh -- device data layout and kernel launchers of td1c_b200.
//
// HBM layout (all complex arrays are (re,im) double pairs, radial index
// fastest, i.e. the reference's Fortran column-major order):
//   orb, h0orb, h1orb, gorb, v2orb : [nfun][L1][Nr]        orb(irad, l, ifun)
//   orbg, gorbg, v2orbg            : [nfun][nlat][Nr]      orbg(irad, ilat, ifun)
//   rho2, v2sph                    : [npair][L2][Nr]       rho2(irad, l, a, b) for stored pair p = (a, b)
//   v2ang (W)                      : [npair][nlat][Nr]     v2ang(irad, ilat, a, b)
// Stored pairs are (a >= b, both dynamic) followed by (a dynamic, b frozen
// core); the reference's Hermitian fill v2(.., b, a) = conj(v2(.., a, b))
// (hprod_mkv2mf.F90:257-345) is never materialised -- consumers read the
// stored pair with a conjugation flag.
#pragma once
#include <cuda.h>

#include "common.cuh"

namespace td1c {

struct LegGemmBatch {
  const double* A;   // real table, M x K row-major, row pitch lda (16-byte aligned rows, zero past K up to lda)
  const double* B0;  // slab (K rows x ldb reals) or conj operand for pair mode
  const double* B1;  // second operand for pair mode
  double* C;         // output, M rows x ldc reals
  int ldb, ldc, lda, pad;
};
// row pitch of the padded Legendre tables: depth rounded up to the GEMM's 32-deep chunks
__host__ __device__ inline int legendre_lda(int k) { return (k + 31) / 32 * 32; }
int launch_legendre_gemm(const LegGemmBatch* d_batches, int nbatch, int M, int K, int N, bool pair,
                         cudaStream_t st);
int launch_legendre_gemm_mt(const LegGemmBatch* d_batches, int nbatch, int M, int K, int N, bool pair, int mt,
                            cudaStream_t st);
// the same transform in split TF32 on tcgen05 (FP32 accumulation, FP64 in and out);
// a bounded wait that runs out sets ST_TIMEOUT in *status
int launch_legendre_gemm_tf32(const LegGemmBatch* d_batches, int nbatch, int M, int K, int N, bool pair, int* status,
                              cudaStream_t st);

// the same transform in split TF32 as a persistent warp-specialised kernel
// (legendre_tc.cu): tables split once at set-up and resident per CTA, a ring
// of staged slab chunks, two TMEM accumulators; for M <= 128
struct LegTcArgs {
  const LegGemmBatch* batches;
  const int* order;        // batch of each group-ordered batch slot
  const int4* work;        // per CTA: (table, first tile, end tile, -)
  const uint32_t* tables;  // per table: hi then lo plane, np x kp each, tensor-core layout
  const int2* zc;          // per batch: tensor-map slab index of B0 and B1
  int* status;
  int M, K, N, np, kp, ntn, stages, raw_slots, tmem_cols;
};
struct LegTcPlan {
  CUtensorMap tmap;        // the slab array (3-d: N doubles x K rows x slabs), boxes of 128 x 16
  LegTcArgs args{};
  int ncta = 0, smem = 0;
  bool pair = false;
};
int launch_legendre_tc(const LegTcPlan& p, int* status, cudaStream_t st);

// ---- the learned predictor's data path (predictor.cu)
constexpr int LP_REC = 41;  // doubles per training record: Gram matrix (16 complex), targets (4 complex), |W_n|^2
struct LpArgs {
  int nu, nfe, nd, Nr, nlat, npair, ni;  // units (pair x element), grid, pairs, int2e entries
  size_t nw;                             // complex values of one W field
  cplx* W;                               // the context's pair potentials (exact value in, stage value out)
  cplx* ring;                            // [5][nw] history of W at the step start states
  cplx* int2e;                           // the context's int2e
  cplx* iring;                           // [5][ni]
  cplx* gram;                            // [nu][4][4] Gram matrix of each unit's last four history values
  cplx* weights;                         // [nu][4] weights of the c = 1 prediction
  double *err, *tnorm;                   // [nu] judge terms
  double* judge;                         // [0] this step's relative error, [1] running maximum
  int* counter;                          // history index of the newest value
  float* feat;                           // [nu][32] network inputs
  const float* net_out;                  // [nu][8] network outputs
  int use_net;
  const int* pair_kind;                  // [npair] 0 diagonal, 1 off-diagonal, 2 with the frozen core
  double* record;                        // training records [steps][nu][LP_REC] (null: none)
  int* rec_count;
};
int launch_lp_push_judge(const LpArgs& a, cudaStream_t st);
int launch_lp_features(const LpArgs& a, cudaStream_t st);
int launch_lp_weights(const LpArgs& a, cudaStream_t st);
int launch_lp_stage(const LpArgs& a, int half, cudaStream_t st);

// ---- the learned predictor's network (mlp.cu)
constexpr int MLP_MAXDEPTH = 8;
struct MlpInferArgs {
  int depth, rows, nin, ldx, ldy;
  const float* x;
  float* y;
  int* status;
  int n[MLP_MAXDEPTH], np[MLP_MAXDEPTH], kp[MLP_MAXDEPTH];  // width, padded width, padded depth of each layer
  const float* b[MLP_MAXDEPTH];
  const unsigned short* wbf16[MLP_MAXDEPTH];  // BF16 weight planes (tensor-core layout)
};
int launch_mlp_infer_bf16(const MlpInferArgs& a, cudaStream_t st);
int mlp_infer_prepare();

// ---- one-body: tprod + zprod/pzprod (hprod_tprod.F90, hprod_zprod.F90, hprod_pzprod.F90)
struct OneBodyArgs {
  int Nr, L1, nd, nfun, nfcore, mmax1, igauge;
  const double* radk;    // (2nd+1) x (nrad+1) band, reference layout
  const double* radk0;
  const double* radp;
  const double* tdiag;   // [L1][Nr] diagonal of tmat (centrifugal + nuclear + radk diag + v2jfc)
  const double* xrad;    // [nrad+1]
  const double* alph;    // [(2 mmax1 + 1)][L1]
  const int* mval;       // [nfun]
  const cplx* orb;
  cplx* h0orb;
  cplx* h1orb;
  const double* lfield;  // device: lfield(1:3,1:3) column-major (9 doubles)
};
int launch_onebody(const OneBodyArgs& a, cudaStream_t st);

// ---- Poisson (hprod_mkv2mf.F90:118-182): per (pair, l) banded Cholesky solve
struct PoissonArgs {
  int Nr, L2, nd, npair;
  const double* d2ll;    // [L2][Nr][nd+1] band Cholesky factor (LAPACK 'L' storage per l)
  const double* d2rinv;  // [L2][Nr] reciprocal diagonal of the factor
  const double* rpl0;    // [L2][Nr]
  const double* rpl1;
  const double* invr;
  const double* fac2;
  const double* fac1;    // [L2]
  const int* pair_m;     // [npair] m of the pair (m_b - m_a)
  const cplx* rho2;      // [npair][L2][Nr]
  cplx* v2sph;           // [npair][L2][Nr]
  const double* tabf;    // [L2][Np][W] forward row tables (launch_poisson_tables)
  const double* tabb;    // [L2][Np][W] backward row tables
  int* status;           // device status word (ST_TIMEOUT on a stalled copy)
  int boxp;              // pairs per TMA box (min(16, npair)), set by poisson_encode_maps
  CUtensorMap tm_rho;    // rho2 viewed as (re|im, pair, row, l) float64, box (2, boxp, nd, 1)
  CUtensorMap tm_v2;     // v2sph, same view
};
// doubles per row of the Poisson row tables: nd band values + 3, even
__host__ __device__ inline int poisson_row_width(int nd) { return (nd + 5) / 2 * 2; }
int poisson_encode_maps(PoissonArgs& a);  // fills boxp, tm_rho, tm_v2 from rho2, v2sph, npair
int launch_poisson_tables(const PoissonArgs& a, double* tabf, double* tabb, cudaStream_t st);
int launch_poisson(const PoissonArgs& a, cudaStream_t st);

// ---- Poisson by static condensation (poisson_cond.cu): A_l = l(l+1)/r^2 + 2T
// inverted element by element; the bridge Schur complement is tridiagonal
struct PsCond {
  int nfe = 0, nd = 0, ni = 0, nb = 0, L2 = 0, Nr = 0;  // ni = nd - 1 interior points, nb = nfe - 1 bridges
  int er = 0, sr = 0;      // doubles per element / share record (even)
  double* erec = nullptr;  // [L2][nfe][er]: W(j, k) = fac2(k) (A_e^-1)(k, j) invr(j) as [j][k]; fac2 GL; fac2 GR;
                           //   fac2 rpl1 (interior points); fac2 and fac2 rpl1 at the left bridge
  double* srec = nullptr;  // [L2][nfe][sr]: coefficient rows (t, left share, right share) over the nd owned points
  double* gl = nullptr;    // [L2][nfe][ni]: A_e^-1 A(I_e, left bridge)   (set-up)
  double* gr = nullptr;    // [L2][nfe][ni]: A_e^-1 A(I_e, right bridge)  (set-up)
  double* vl = nullptr;    // [L2][nfe][ni]: A(left bridge, I_e)          (set-up)
  double* vr = nullptr;    // [L2][nfe][ni]: A(right bridge, I_e)         (set-up)
  double* tm = nullptr;    // [L2][nb] LU of the bridge system: multipliers,
  double* tw = nullptr;    //   reciprocal pivots,
  double* tu = nullptr;    //   superdiagonal
};
struct PsCondArgs {
  PsCond f;
  int Nr, L2, npair;
  const int* pair_m;     // [npair]
  const cplx* rho2;      // [npair][L2][Nr]
  cplx* v2sph;           // [npair][L2][Nr]
  const double* fac1;    // [L2]
  cplx* cb;              // [L2][nfe][2][npair] element shares of the bridge right-hand sides
  cplx* tpart;           // [L2][nfe][npair] element shares of t
  cplx* xb;              // [L2][nb][npair] bridge values
  cplx* t;               // [L2][npair]
  int tf32;              // element pass: interior products in split TF32 (mixed mode 3)
};
int launch_ps_cond_setup(PsCond& f, const double* xrad, const double* radk, const double* invr, const double* rpl0,
                         const double* rpl1, const double* fac2, int* status, cudaStream_t st);
int launch_ps_cond(const PsCondArgs& a, cudaStream_t st);

// ---- mean-field action on the (r, theta) grid (hprod_mfprod2.F90)
struct Act2Block {     // one dense (ij) x (kl) block of the 2-RDM contraction
  int row0, nrow;      // rows: (ia, ja) entries rows[row0 .. row0+nrow)
  int col0, ncol;      // cols: (pair, conj) entries cols[col0 .. col0+ncol)
  int coff, pad0, pad1, pad2;  // coefficient offset, coef[coff + kl * nrow + ij]
};
struct Act2Coef { int d2idx, dst; };  // den2 element -> coefficient slot
// one Delta-m block of the act2 contraction on the FP64 tensor cores:
// coefficients C[row][kl] padded to mt m-tiles of 8 rows x kpad (multiple of
// 4) columns, row pitch pa (double2, 4 mod 8) from coff; columns
// dcol[col0 .. col0+kpad) (padding: the zero W row npair); D2V rows
// drow0 .. drow0+nr
struct MfdBlock { int coff, pa, mt, kpad, col0, drow0, nr, pad; };
struct MfprodArgs {
  size_t ngrid;
  int nfun, npair;
  const cplx* W;        // [npair][ngrid]
  const cplx* orbg;     // [nfun][ngrid]
  cplx* gorbg;          // [nfun][ngrid] (fully written for dynamic orbitals)
  cplx* v2orbg;         // [nfun][ngrid] (fully written for dynamic orbitals)
  int nact, ncore, nfcore;
  const cplx* den1;     // [nact][nact] (Fortran order)
  const cplx* den2;     // [nact^4]
  const cplx* rden;     // [nact][nact]
  const int* mval;
  const int* pair_of;   // [nfun][nfun]: stored pair index of (a, b) or of (b, a)
  const int* pair_cj;   // [nfun][nfun]: 1 when (a, b) is read as conj of stored (b, a)
  int nelact;           // total active electrons
  // act2 blocks (host-built), coefficients filled on the device each RHS
  int nblk, nrow, ncol, ncoef;
  const Act2Block* blk;
  const int2* rows;
  const int2* cols;
  const Act2Coef* coef_map;
  cplx* coef;
  // tensor-core form of act2 (used when dmma != 0): its own padded
  // coefficient layout and map, per-target epilogue lists
  int dmma, nblk_d, ndcol, ncoef_d, nelist;
  int max_cta;          // cap of the persistent DMMA grid (0: as many CTAs as are resident)
  const MfdBlock* dblk;
  const int2* dcol;       // (pair, conj) of every padded column
  const Act2Coef* dmap;   // den2 element -> padded coefficient slot
  cplx* dcoef;            // [ncoef_d]
  const int2* elist;      // per active target x: (D2V row, other orbital | conj << 16), in row order
  const int* eoff;        // [nact + 1] offsets into elist
  int2 witem[4][8];       // per warp: (block, m-tile) items, -1 ends the list
};
int launch_mfprod(const MfprodArgs& a, cudaStream_t st);

// ---- observables: length-form dipole (hprod_dipole.F90)
struct DipoleArgs {
  int Nr, L1, mmax1, ncore, nact, nent;
  const double* xrad;    // [Nr + 2] radial points (index r + 1)
  const double* alph;    // [2 mmax1 + 1][L1]
  const int* mval;       // [nfun]
  const int2* ent;       // [nent] (i, j): core (f, f) first, then active pairs of equal m
  const cplx* wfn;       // [nfun][L1][Nr]
  const cplx* den1;      // [nact][nact]
  cplx* partial;         // [nchunk][nent]
  double* out;           // device scalar
  int mode = 0;          // operator: 0 z (radial factor r), 1 acceleration (radial factor -Z / r^2), 2 pv
  double znuc = 0;       // nuclear charge (mode 1)
  const cplx* pv = nullptr;  // mode 2: the operator applied to the orbitals, [nfun][L1][Nr]
};
int launch_dipole(const DipoleArgs& a, cudaStream_t st);
int dipole_partial_size(int Nr, int nent);
// wfn_orth_cic + wfn_orth_orb on device-resident orbitals and CI
int launch_orth(int Nr, int L1, int nfun, int nfcore, int lcic, const int* mval, cplx* wfn, cplx* cic, cudaStream_t st);


// ---- CI (ormas_*), full string-product formulation
struct CiTables {
  int nact, nstr_a, nstr_b, mtot, spin_sym;
  int smin, nsec;         // sectors of total M: S = smin .. smin + nsec - 1
  const unsigned* stra;   // [nstr_a] bit strings sorted by (M, mask)
  const unsigned* strb;
  const int* idx_a;       // [2^nact] mask -> string index
  const int* idx_b;
  const int* Ma;          // [nstr_a]
  const int* Mb;
  const int* sec_off;     // [nsec][nstr_b] offset of beta string block in sector, -1 if empty
  const int* sec_first;   // [nsec][nstr_b] first alpha string index of the block
  const int* sec_cnt;     // [nsec][nstr_b]
  const int* sec_size;    // [nsec]
  const long* dvec_off;   // [nact*nact] offset of D_pq in the D arrays (complex elements)
  const int* det_b;       // [lcic] beta string of each determinant of the CI vector (sector mtot)
  const int* det_a;       // [lcic]
  const int* orb_m;       // [nact] m of active orbitals
  int lcic;
  const int* sec_detA;    // [sum of sector sizes] alpha string of each sector determinant
  const int* sec_detB;
  const int* sec_base;    // [nsec] start of each sector in sec_detA/B
  const int* dgrp;        // pq indices grouped by m_p - m_q
  const int* dgrp_off;    // [nsec + 1]
  const int4* quads;      // m-allowed (p,q,r,s) of den2
  int nquad;
};
struct CiArgs {
  CiTables t;
  const cplx* cic;
  cplx* Da;       // alpha part of E_pq c, per pq in its sector
  cplx* Db;
  cplx* T;        // T_rs (same layout as D)
  cplx* den1;     // [nact^2]
  cplx* den2;     // [nact^4]
  cplx* sigma;    // [lcic] (output hcic)
  const cplx* int1e;
  const cplx* int2e;
  const double* ene_act;  // device scalar
  double dtime; int icomp;
};
int launch_ci_dvec(const CiArgs& a, int maxsec, cudaStream_t st);
int launch_ci_rdm(const CiArgs& a, cudaStream_t st);
int launch_ci_tvec(const CiArgs& a, int maxsec, cudaStream_t st);  // T_rs = sum_pq (rs|pq) D_pq: int2e and D only
int launch_ci_sigma(const CiArgs& a, cudaStream_t st);              // sigma from T, D and int1e

// Columns coupled to row ir (1-based radial index) by the FEDVR kinetic and
// derivative operators: the points of the row's finite element, both
// elements for a bridge point (ir a multiple of nd); clipped to 1..Nr.
__device__ __forceinline__ void fedvr_row_span(int ir, int nd, int Nr, int& jlo, int& jhi) {
  const int e = ir / nd;
  if (ir == e * nd) { jlo = ir - nd; jhi = ir + nd; }
  else { jlo = e * nd; jhi = e * nd + nd; }
  jlo = jlo < 1 ? 1 : jlo;
  jhi = jhi > Nr ? Nr : jhi;
}

// ---- one-body propagators of the split schemes (h1prop.cu) ----------------
// Condensed inverse of M_l = 1 + c T_l, l = 0..L1-1: per finite element the
// inverse of the interior block and its couplings to the two bridge points,
// per l the pivoted tridiagonal LU of the bridge Schur complement.
struct H1Fac {
  int nfe = 0, nd = 0, ni = 0, nb = 0, L1 = 0;  // ni = nd - 1 interior points, nb = nfe - 1 bridges
  cplx* ainv = nullptr;  // [L1][nfe][ni][ni]: ainv[..][j][k] = (A_e^-1)(k, j)
  cplx* gl = nullptr;    // [L1][nfe][ni]: A_e^-1 M(I_e, left bridge)
  cplx* gr = nullptr;    // [L1][nfe][ni]: A_e^-1 M(I_e, right bridge)
  cplx* vl = nullptr;    // [L1][nfe][ni]: M(left bridge, I_e)
  cplx* vr = nullptr;    // [L1][nfe][ni]: M(right bridge, I_e)
  cplx* tdl = nullptr;   // [L1][nb] tridiagonal factors: multipliers,
  cplx* tdi = nullptr;   //   reciprocal pivots,
  cplx* tdu = nullptr;   //   first and
  cplx* tdu2 = nullptr;  //   second superdiagonal of U
  int* tpiv = nullptr;   // [L1][nb] row interchanges
};
struct H1FacSrc {
  int Nr, L1, nd, nfe;
  cplx c;                // M = 1 + c T
  const double* radk;    // (2nd+1) x (nrad+1) bands (l = 0 / l >= 1)
  const double* radk0;
  const double* tdiag;   // [L1][Nr] diagonal of T
  int* status;           // ST_SINGULAR on a zero pivot
};
int launch_h1fac(const H1FacSrc& s, H1Fac& f, cudaStream_t st);

// One pass of the element-by-element application of M^-1 (h1prop.cu):
// finish the previous correction (finalize), add it to torb and the residual
// norm, and form the next right-hand side r = a x + b T x + (cz0 lfield[2]) V1 x
// (make_rhs) with its interior solutions z and bridge shares cb; the bridge
// kernel then solves for the bridge values xb.
struct H1ElemArgs {
  H1Fac fac;
  int Nr, L1, nfun, nfcore, mmax1, igauge;
  int f_fin, f_rhs;      // first orbital of the finalize / right-hand-side work
  int finalize, make_rhs, accumulate, do_norm, check_skip;
  const int* mval;
  const double* radk;
  const double* radk0;
  const double* radp;
  const double* tdiag;
  const double* xrad;
  const double* alph;
  const double* lfield;  // device lfield(1:3,1:3) (may be null: no laser term)
  cplx a, b, cz0;
  const cplx* in;        // input vector of a first pass (finalize == 0), [nfun][L1][Nr]
  const cplx* z_in;      // [nfun][L1][nfe][nd - 1] interior solutions of the previous pass
  cplx* z_out;           // same layout, this pass (a different buffer than z_in)
  cplx* cb;              // [nfun][L1][nfe][2] bridge shares (left, right)
  cplx* xb;              // [nfun][L1][nfe - 1] bridge solutions
  cplx* torb;            // rows of orbitals >= nfcore: = x or += x
  double thresh, norm_div;
  double* partial;       // [h1elem_partials]
  unsigned* ticket;      // zero between launches
  int* done;             // residual norm below thresh (set by finalize passes with do_norm)
  int* ncyc;             // correction cycles run (bridge passes with check_skip)
  // device-driven cycles (the body of a graph loop): iter_mode 1 takes the
  // cycle k = *iter + 1 from the device and derives f_fin (f_first on cycle 1),
  // accumulate (k > 1) and the z buffers (zb[(k-1)&1] in, zb[k&1] out);
  // iter_mode 2 (the last pass) reads z from zb[*iter & 1]
  int iter_mode, f_first;
  int mv[16];            // m of every orbital (nfun <= 16)
  const int* iter;
  cplx* zb0;
  cplx* zb1;
};
int launch_h1elem(const H1ElemArgs& a, cudaStream_t st);
// graph-loop control: *iter += 1, then the loop continues while the residual
// norm is not below thresh (*done == 0) and *iter < maxcyc
int launch_h1loop_ctl(int* iter, const int* done, int maxcyc, cudaGraphConditionalHandle h, cudaStream_t st);
int launch_h1bridge(const H1ElemArgs& a, cudaStream_t st);
size_t h1elem_smem(int nd, int nfun);
size_t h1elem_partials(int nfe, int L1);

}  // namespace td1c
