// hprod.cu -- orchestration of the B200 orbital-equation RHS and the C-ABI.
//
// hprod_htot (src/hprod/hprod_htot.F90:2-208) as a fixed sequence of device
// kernels on one stream, all data resident in HBM:
//   orbin        sph2ang1 GEMM (+ frozen-core gauge phase)   hprod_orbin.F90
//   CI           D = E_pq c, 1-/2-RDM, regularised 1/D        ormas_mkden1/2, hprod_invden.F90
//   one-body     tprod + zprod/pzprod stencil                 hprod_tprod/zprod/pzprod.F90
//   pair density fused into the theta->l GEMM                 hprod_mkrho2.F90, bas_ang2sph2.F90
//   Poisson      banded Cholesky solves per (pair, l)         hprod_mkv2mf.F90
//   l->theta     GEMM (Hermitian half read with conj)         bas_sph2ang2.F90
//   mfprod       core J/K, active J/K, 2-RDM contraction      hprod_mfprod2.F90
//   theta->l     GEMM for g and v2 orbitals                   bas_ang2sph1.F90
//   integrals    orbital matrix elements, int2e block GEMM    hprod_mkint1/2_sph.F90
//   small        int1e, energies, X matrix                    hprod_ene_*.F90, hprod_htot_mkxmat.F90
//   sigma        CI sigma vector                              ormas_xact2/ormas_hcic
//   dtorb        hwfn = -i dt (h0+h1+g+v2) phi + sum_j phi_j X_ji  hprod_htot_dtorb.F90
// Set-up (the bas_gen_* tables, the band Cholesky factors, the CI string
// tables, pair and batch lists) happens once in hprod_init_.  There is no
// host fallback: every RHS value is produced by the kernels in this library.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include "common.cuh"
#include "kernels.cuh"
#include "reductions.cuh"
#include "tma.cuh"
#include "../../include/td1c_b200.h"

using namespace td1c;

namespace td1c {
int legendre_tc_plan(const std::vector<LegGemmBatch>& h_batches, const LegGemmBatch* d_batches, int M, int K, int N, bool pair,
                     const double* slab_base, int slab_count, int nsm, LegTcPlan* out, std::vector<void*>& allocs,
                     cudaStream_t st);
}

namespace {

const double PI = 3.14159265358979323846264338327950288;

std::vector<void*>& cur_allocs();  // every device allocation of the current context, freed by hprod_final_

template <class T>
T* dalloc(size_t n) {
  T* p = nullptr;
  if (n == 0) n = 1;
  if (cudaMalloc(&p, n * sizeof(T)) != cudaSuccess) {
    fprintf(stderr, "td1c_b200: cudaMalloc of %zu bytes failed\n", n * sizeof(T));
    return nullptr;
  }
  // zero it on the legacy stream and wait: the library stream does not
  // synchronise with the legacy stream, so work queued on it right after the
  // allocation must not race the clearing
  cudaMemset(p, 0, n * sizeof(T));
  cudaStreamSynchronize(cudaStreamLegacy);
  cur_allocs().push_back(p);
  return p;
}
template <class T>
T* dupload(const std::vector<T>& v) {
  T* p = dalloc<T>(v.size());
  if (p && !v.empty()) cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
  return p;
}

struct RkBufs {
  cplx *y0 = nullptr, *yt = nullptr, *k = nullptr, *k2 = nullptr;  // orbitals then CI, contiguous
  double* lf_cur = nullptr;
  int* counter = nullptr;
  size_t cap = 0;
  const cplx* reset_orb = nullptr;  // optional: every step starts from this state
  const cplx* reset_cic = nullptr;
  // cached graph of one step and what it was captured with
  const void* g_y = nullptr; const void* g_yc = nullptr; const void* g_tab = nullptr;
  const void* g_ro = nullptr; double g_dt = 0; long g_per = 0;
  int h_counter[2] = {0, 0};
  // cached graphs of one split2 / ETD-RK2 / ETD-RK4 step
  const void* s_y[3] = {nullptr, nullptr, nullptr}; const void* s_yc[3] = {nullptr, nullptr, nullptr};
  const void* s_tab[3] = {nullptr, nullptr, nullptr}; double s_dt[3] = {0, 0, 0}; int s_cyc[3] = {0, 0, 0};
  double s_thr[3] = {0, 0, 0}; int s_split[3] = {-1, -1, -1}; int s_mask[3] = {-1, -1, -1}; long s_per[3] = {0, 0, 0};
  const void* s_ro[3] = {nullptr, nullptr, nullptr};
  int g_ctl = -1, s_ctl[3] = {-1, -1, -1};  // control flags (icomp, igauge) the graphs were captured with
};
struct Etd4Bufs {
  cplx *w1 = nullptr, *w2 = nullptr, *w3 = nullptr, *h2 = nullptr, *h3 = nullptr, *tmp = nullptr;
  size_t cap = 0;
};
struct Ctx {
  std::vector<void*> allocs;  // device allocations of this context
  RkBufs rk;                  // propagation buffers and cached step graphs
  Etd4Bufs e4;
  bool own_streams = false;   // contexts other than the default one own their streams
  int tune_mt = 0, tune_mf_cap = 0, tune_i2_split = 0;  // launch shapes (0: the built-in choice)
  // ---- bound inputs
  bool have_rad = false, have_sph = false, have_bas = false, initialized = false;
  int nfe = 0, nd = 0, nrad = 0, Nr = 0;
  double rmask = 0;
  std::vector<double> h_xrad, h_wrad, h_radp, h_radk, h_radk0, h_mask;
  int lmax1 = 0, lmax2 = 0, mmax1 = 0, mmax2 = 0, nlat = 0, L1 = 0, L2 = 0;
  std::vector<double> h_wlat, h_cost, h_legf1, h_legb1, h_legf2, h_legb2;
  double znuc = 0; int smul = 1, mtot = 0, nfun = 0, nela = 0, nelb = 0;
  std::vector<int> otype, mval, lval;
  int icomp = 1, igauge = 0;
  int isplit = 0;  // split_type (clcontrol.cpp:98): one-body terms left out of the orbital RHS
  int nfcore = 0, ndcore = 0, nact = 0, ncore = 0, nelact = 0, neltot = 0;
  int nsub = 1;  // ORMAS subspaces of the active space (ormas_bind_ nsub); 1 = CAS
  // ---- hprod_bind_ outputs
  double *p_ene_fcore = nullptr, *p_ene_dcore = nullptr, *p_ene_core = nullptr, *p_ene_act = nullptr, *p_ene_tot = nullptr;
  // ---- device tables
  double *xrad = nullptr, *mask = nullptr, *radk = nullptr, *radk0 = nullptr, *radp = nullptr, *cost = nullptr;
  double *legf1 = nullptr, *legb1 = nullptr, *legf2 = nullptr, *legb2 = nullptr, *alph = nullptr;
  double *tdiag = nullptr, *d2ll = nullptr, *d2rinv = nullptr, *rpl0 = nullptr, *rpl1 = nullptr, *invr = nullptr, *fac2 = nullptr, *fac1 = nullptr;
  double *ps_tabf = nullptr, *ps_tabb = nullptr;  // Poisson row tables (forward, backward)
  PoissonArgs ps_main{}, ps_fcfc{};  // Poisson arguments with encoded tensor maps (RHS pairs, fcfc pairs)
  PsCondArgs ps_cond{};  // condensed Poisson of the RHS pairs (factors and work buffers)
  MfprodArgs mf{};  // mean-field action arguments with encoded tensor maps
  int* d_mval = nullptr;
  // ---- pairs
  int npair = 0, npair_all = 0, nfcfc = 0;
  std::vector<int> pa, pb;  // stored pair p = (a, b)
  int *pair_m = nullptr, *pair_of = nullptr, *pair_cj = nullptr;
  // ---- state
  size_t nbas = 0, nbas2 = 0, ngrid = 0;
  cplx *orb = nullptr, *orb0 = nullptr, *orbg0 = nullptr, *orbg = nullptr, *h0orb = nullptr, *h1orb = nullptr;
  cplx *gorb = nullptr, *v2orb = nullptr, *gorbg = nullptr, *v2orbg = nullptr, *rho2 = nullptr, *v2sph = nullptr, *W = nullptr;
  cplx *wfn_io = nullptr, *cic_io = nullptr, *hwfn_io = nullptr, *hcic_io = nullptr;
  double* lfield = nullptr;  // device [9]
  double* v2jfc = nullptr;   // device [Nr] (real)
  // ---- CI
  int lcic = 1, nstr_a = 0, nstr_b = 0, smin = 0, nsec = 0, maxsec = 0, spin_sym = 0;
  std::vector<unsigned> h_stra, h_strb;
  std::vector<int> h_detoff, h_afirst, h_acount;
  CiTables cit{};
  cplx *Da = nullptr, *Db = nullptr, *T = nullptr, *den1 = nullptr, *den2 = nullptr, *rden = nullptr, *rrden = nullptr;
  cplx *int1e = nullptr, *int2e = nullptr, *cic = nullptr;
  // ---- reductions
  OrbdotsArgs od{};
  std::vector<int4> h_ent;
  int* ent_index = nullptr;  // [5][nfun][nfun] -> entry id or -1 (A, B, C, E, GV)
  Int2eArgs i2{};
  int i2_nsplit = 128;
  I2dArgs i2d{};          // int2e on the FP64 tensor cores
  bool i2_dmma = false;   // the DMMA plan fits in shared memory
  I2tArgs i2t{};          // int2e in split TF32 on tcgen05 (mixed-precision form)
  bool i2_tc = false;     // its plan fits (at most 64 stored active pairs)
  // act2 blocks
  int a2_nblk = 0, a2_nrow = 0, a2_ncol = 0, a2_ncoef = 0;
  Act2Block* a2_blk = nullptr; int2* a2_rows = nullptr; int2* a2_cols = nullptr;
  Act2Coef* a2_map = nullptr; cplx* a2_coef = nullptr;
  // ---- small matrices
  cplx *xmat = nullptr;
  double* ene = nullptr;  // device [5]
  double h_ene[5] = {0, 0, 0, 0, 0};
  double ene_fcore = 0;
  // ---- GEMM batches
  LegGemmBatch *b_orbg = nullptr, *b_orbfc = nullptr, *b_rho = nullptr, *b_rho_fcfc = nullptr, *b_W = nullptr,
               *b_W_fcfc = nullptr, *b_gorb = nullptr, *b_orbg0 = nullptr, *b_gorbfc = nullptr;
  int n_orbg = 0, n_orbfc = 0, n_gorb = 0;
  // ---- RK4
  cplx *y0 = nullptr, *yacc = nullptr, *ytmp = nullptr, *kbuf = nullptr;
  double* field_tab = nullptr; long field_cap = 0;  // field table, capacity in doubles
  cudaGraphExec_t graph_exec[4] = {nullptr, nullptr, nullptr, nullptr};
  long launches = 0;
  // ---- misc
  cudaStream_t st = nullptr;
  int status = 0;
  int* d_status = nullptr;  // device status word (ST_* bits)
  double* d_scalar = nullptr;
  int2* dip_ent = nullptr; int dip_nent = 0; cplx* dip_partial = nullptr;  // dipole entries and chunk sums
  double* dip_lf = nullptr;   // unit lfield(3,1) for the velocity operator
  double* dip_out = nullptr;  // [3] traces of z, p_z and the acceleration operator
  // frozen-core dipole: z phi, p_z phi, the generalized-Fock vectors, the caller's field, and the
  // overlaps of the generalized-Fock corrections (entries and their host-side index maps)
  cplx *dip_z = nullptr, *dip_p = nullptr, *dip_g = nullptr, *dip_rd = nullptr;
  double* dip_lfd = nullptr;
  int4* dip_rd_ent = nullptr;
  int dip_rd_n = 0;
  std::vector<int> dip_ia, dip_ib, dip_if, dip_isz, dip_isp;
  cplx *relax_hw = nullptr, *relax_hc = nullptr;  // RHS outputs of the energy evaluation in td1c_gpu_relax
  // one-body propagators: condensed factors of 1 + c T per c, and scratch
  struct H1Slot { double cre = 0, cim = 0; H1Fac f; };
  static constexpr int kH1Slots = 16;  // factor sets kept: split2/ETD-RK2 use 1-2, ETD-RK4 12
  H1Slot h1slot[kH1Slots];
  int n_h1 = 0;
  cplx* h1_z[2] = {nullptr, nullptr};  // interior solutions (alternating passes)
  cplx *h1_cb = nullptr, *h1_xb = nullptr;  // bridge shares, bridge values
  double* h1_partial = nullptr;
  unsigned* h1_ticket = nullptr;
  int* h1_flags = nullptr;  // [0] done, [1] cycles of the last application, [2] cycle counter of a graph loop
  cudaStream_t st4 = nullptr;  // stream on which graph-loop bodies are captured
  // phase timing (off during graph capture)
  bool profile = false;
  int mixed = 0;  // 1: the mean field's pair-density and pair-potential transforms in split TF32 (tcgen05)
  // persistent split-TF32 plans of the two pair-field transforms (built on the first switch to mixed)
  std::vector<LegGemmBatch> h_b_rho, h_b_W;
  LegTcPlan tc_rho, tc_W;
  bool tc_built = false, tc_ok_rho = false, tc_ok_W = false;
  int mf_external = 0;  // 1: the RHS takes W and int2e as they stand (the learned form's predicted stages)
  // learned form: predictor data path (predictor.cu), the caller's network, and the captured steps
  LpArgs lp{};
  bool lp_alloc = false;
  MlpInferArgs lp_mi{};
  bool lp_has_net = false;
  float* lp_out = nullptr;
  int* lp_mi_status = nullptr;
  int lp_use_net = 0;
  double lp_bound = 1e-6;
  cplx* lp_save = nullptr;  // the state at the start of a judged window (orbitals, then CI)
  cudaGraphExec_t lp_exec[3] = {nullptr, nullptr, nullptr};  // E, H, P steps
  long lp_exec_launch[3] = {0, 0, 0};
  // what the captured steps and the window schedule belong to: a call that starts where the last
  // one ended (same state buffers, field and step) continues its history and schedule
  const void* lp_key_y = nullptr; const void* lp_key_yc = nullptr; const void* lp_key_tab = nullptr;
  double lp_key[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  double lp_t_end = -1e300;
  int lp_mode = 0, lp_backoff = 0, lp_plain_left = 0;
  int lp_screen = 1;  // 1: predicted windows only after a fill window whose judge values pass
  cudaEvent_t ev[16] = {};
  cudaStream_t st2 = nullptr;  // side stream of the CI RDM chain (process lifetime, like st)
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  cudaStream_t st3 = nullptr;  // side stream of the one-body stencil and of int2e
  cudaEvent_t ev_ob_fork = nullptr, ev_ob_join = nullptr, ev_i2_fork = nullptr, ev_i2_join = nullptr;
  cudaEvent_t ev_sig_fork = nullptr, ev_sig_join = nullptr;
  int nev = 0;
};

// phases of run_htot, in order (td1c_gpu_profile reports their durations)
const char* kPhaseNames[] = {"orbin", "ci_rdm", "onebody", "rho_gemm", "poisson", "w_gemm", "mfprod",
                             "gorb_gemm", "orbdots", "int2e", "smallmat", "ci_sigma", "dtorb"};
const int kNumPhases = 13;

// contexts: [0] is the default one the drop-in entry points use; further
// contexts (td1c_gpu_ctx_create) hold independent jobs of an ensemble
std::vector<Ctx*> g_ctxs(1, nullptr);
int g_cur = 0;
Ctx* g = nullptr;  // the current context, g_ctxs[g_cur]
Ctx& ctx() {
  if (!g) { g = new Ctx(); g_ctxs[g_cur] = g; }
  return *g;
}
std::vector<void*>& cur_allocs() { return ctx().allocs; }

// ===========================================================================
// set-up kernels
// ===========================================================================
// band Cholesky (dpbtrf 'L') of A_l = l(l+1)/r^2 + 2 radk (bas_gen_d2ll.F90:2-140),
// one thread per l; factor stored as ab[(i-j) + (nd+1) j] for each l.
__global__ void d2ll_factor_kernel(int Nr, int nd, int L2, const double* __restrict__ xrad,
                                   const double* __restrict__ radk, double* __restrict__ d2ll,
                                   double* __restrict__ rinv, int* status) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= L2) return;
  const int ld1 = nd + 1, bw = 2 * nd + 1;
  double* ab = d2ll + (size_t)l * ld1 * Nr;
  const double l2 = (double)l * (l + 1);
  for (int ir = 1; ir <= Nr; ++ir) {
    double ak = 1.0 / xrad[ir];
    ab[(size_t)ld1 * (ir - 1)] = ak * ak * l2;
    for (int k = 1; k <= nd; ++k) ab[(size_t)ld1 * (ir - 1) + k] = 0.0;
  }
  for (int ir = 1; ir <= Nr; ++ir) {
    int jul = min(Nr, ir + nd);
    for (int jr = ir; jr <= jul; ++jr) ab[(size_t)ld1 * (ir - 1) + (jr - ir)] += 2.0 * radk[(size_t)bw * ir + (jr - ir + nd)];
  }
  for (int j = 0; j < Nr; ++j) {
    double d = ab[ld1 * j];
    for (int k = max(0, j - nd); k < j; ++k) { double v = ab[(j - k) + ld1 * k]; d -= v * v; }
    if (!(d > 0)) { atomicOr(status, ST_CHOLESKY); return; }
    d = sqrt(d);
    ab[ld1 * j] = d;
    for (int i = j + 1; i <= min(Nr - 1, j + nd); ++i) {
      double s = ab[(i - j) + ld1 * j];
      for (int k = max(0, i - nd); k < j; ++k) s -= ab[(i - k) + ld1 * k] * ab[(j - k) + ld1 * k];
      ab[(i - j) + ld1 * j] = s / d;
    }
  }
  for (int j = 0; j < Nr; ++j) rinv[(size_t)l * Nr + j] = 1.0 / ab[ld1 * j];
}

// tmat diagonal (bas_gen_tmat.F90:30-75) plus the frozen-core Hartree
// potential (hprod_addfc_tmat.F90:2-33)
__global__ void tdiag_kernel(int Nr, int L1, int nd, double znuc, const double* __restrict__ xrad,
                             const double* __restrict__ radk, const double* __restrict__ radk0,
                             const double* __restrict__ v2jfc, double* __restrict__ tdiag) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= Nr * L1) return;
  int l = t / Nr, r = t % Nr, ir = r + 1;
  const int bw = 2 * nd + 1;
  double oor = 1.0 / xrad[ir];
  double zor = oor * (-znuc + (double)(l * (l + 1)) * oor * 0.5);
  double rk = (l == 0 ? radk : radk0)[(size_t)bw * ir + nd];
  double v = zor + rk;
  if (v2jfc) v += v2jfc[r];
  tdiag[t] = v;
}

// frozen-core Hartree potential v2jfc: l = 0 Poisson of the frozen-core
// density (hprod_set_wfn0.F90:221-335); one thread, set-up only
__global__ void v2jfc_kernel(int Nr, int nd, int L1, int nfcore, const int* __restrict__ mval, const int* __restrict__ lvalv,
                             const cplx* __restrict__ orb, const double* __restrict__ d2ll, const double* __restrict__ rinv,
                             const double* __restrict__ rpl0, const double* __restrict__ rpl1, const double* __restrict__ invr,
                             const double* __restrict__ fac2, double rmax, double* __restrict__ v) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  const int ld1 = nd + 1;
  double t = 0.0;
  for (int r = 0; r < Nr; ++r) {
    double rho = 0.0;
    for (int f = 0; f < nfcore; ++f)
      if (mval[f] == 0) { cplx o = orb[((size_t)f * L1 + lvalv[f]) * Nr + r]; rho += cabs2(o) * (2.0 * lvalv[f] + 1.0); }
    t += rho * rpl0[r];
    v[r] = rho * invr[r];
  }
  t *= 1.0 / rmax;
  for (int j = 0; j < Nr; ++j) {
    double s = v[j];
    for (int k = max(0, j - nd); k < j; ++k) s -= d2ll[(j - k) + ld1 * k] * v[k];
    v[j] = s * rinv[j];
  }
  for (int j = Nr - 1; j >= 0; --j) {
    double s = v[j];
    for (int i = min(Nr - 1, j + nd); i >= j + 1; --i) s -= d2ll[(i - j) + ld1 * j] * v[i];
    v[j] = s * rinv[j];
  }
  for (int r = 0; r < Nr; ++r) v[r] = (v[r] + t * rpl1[r]) * fac2[r];
}

// frozen-core mean field on the frozen core for the frozen-core energy
// (hprod_v2fc_enefc: fcj and fcx1 with dofc, hprod_set_wfn0.F90:823-833)
__global__ void fc_g_kernel(int Nr, int nlat, int nfcore, int nfun, const cplx* __restrict__ orbg, const cplx* __restrict__ W,
                            const int* __restrict__ pair_of, const int* __restrict__ pair_cj, const double* __restrict__ v2jfc,
                            cplx* __restrict__ gorbg) {
  const size_t ng = (size_t)Nr * nlat;
  size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ng * nfcore) return;
  const int i = (int)(t / ng);
  const size_t q = t % ng;
  const int r = (int)(q % Nr);
  cplx v = cscale(orbg[(size_t)i * ng + q], v2jfc[r]);
  for (int j = 0; j < nfcore; ++j) {
    int p = pair_of[j * nfun + i], cj = pair_cj[j * nfun + i];
    cplx w = W[(size_t)p * ng + q];
    if (cj) w = cconj(w);
    v = csub(v, cmul(w, orbg[(size_t)j * ng + q]));
  }
  gorbg[(size_t)i * ng + q] = v;
}

// the mean field on the frozen-core rows of the generalized-Fock vectors
// (hprod_mfprod2_gfock, hprod_mfprod2.F90:59-84: the dofc parts of fcx1
// 158-200, dcj 242-306, dcx 308-366, actj 368-437 and actx 439-514; the
// frozen-core Coulomb is in the kinetic diagonal).  For frozen core i at grid
// point q, g + v2 =
//   - sum_{j < nfcore} W(j,i) phi_j + sum_{j dynamic core} (2 W(j,j) phi_i - W(j,i) phi_j)
//   + sum_{ja,ka} den1(ka,ja) W(ja,ka) phi_i - 1/2 sum_{ja} sum_{ka, m equal} den1(ka,ja) phi_ka W(ja,i)
// written to gorbg[i]; W(j,i) is pair_of/pair_cj's pair potential (conjugated
// for the swapped pair).
__global__ void fc_gfock_kernel(int Nr, int nlat, int nfcore, int ncore, int nact, int nfun, const int* __restrict__ mval,
                                const cplx* __restrict__ orbg, const cplx* __restrict__ W, const int* __restrict__ pair_of,
                                const int* __restrict__ pair_cj, const cplx* __restrict__ den1, cplx* __restrict__ gorbg) {
  const size_t ng = (size_t)Nr * nlat;
  size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ng * nfcore) return;
  const int i = (int)(t / ng);
  const size_t q = t % ng;
  auto w = [&](int j, int k) {  // W(j, k) at q
    cplx v = W[(size_t)pair_of[j * nfun + k] * ng + q];
    return pair_cj[j * nfun + k] ? cconj(v) : v;
  };
  auto o = [&](int j) { return orbg[(size_t)j * ng + q]; };
  const cplx oi = o(i);
  cplx g = mkc(0.0, 0.0);
  for (int j = 0; j < nfcore; ++j) g = csub(g, cmul(w(j, i), o(j)));                  // fcx1
  for (int j = nfcore; j < ncore; ++j) g = cadd(g, csub(cscale(cmul(w(j, j), oi), 2.0), cmul(w(j, i), o(j))));  // dcj, dcx
  if (ncore > 0 && nact > 0) {
    cplx d2v = mkc(0.0, 0.0);
    for (int ja = 0; ja < nact; ++ja)
      for (int ka = 0; ka < nact; ++ka) d2v = cadd(d2v, cmul(w(ncore + ja, ncore + ka), den1[ka + nact * ja]));  // actj
    g = cadd(g, cmul(d2v, oi));
    for (int ja = 0; ja < nact; ++ja) {  // actx
      cplx wd = mkc(0.0, 0.0);
      for (int ka = 0; ka < nact; ++ka)
        if (mval[ncore + ja] == mval[ncore + ka]) wd = cadd(wd, cmul(o(ncore + ka), cscale(den1[ka + nact * ja], -0.5)));
      g = cadd(g, cmul(wd, w(ncore + ja, i)));
    }
  }
  gorbg[(size_t)i * ng + q] = g;
}

// hprod_gfock_sum (hprod_gfock.F90:198-230) plus, in the velocity gauge, the
// E_z z phi that hprod_dipole adds to the dynamic rows (hprod_dipole.F90:61-64).
// The frozen-core rows' h1 already holds that term: the RHS one-body coupling
// adds E_z z phi to them in the velocity gauge (hprod_htot.F90 via hprod_zprod).
__global__ void gfock_sum_kernel(size_t n, size_t nfc, double ef, const cplx* __restrict__ gorb, const cplx* __restrict__ v2orb,
                                 const cplx* __restrict__ h0orb, const cplx* __restrict__ h1orb, const cplx* __restrict__ zo,
                                 cplx* __restrict__ g) {
  size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  cplx v = cadd(cadd(gorb[t], v2orb[t]), cadd(h1orb[t], h0orb[t]));
  if (t >= nfc) v = cadd(v, cscale(zo[t], ef));
  g[t] = v;
}

// out[e] = sum_k conj(A_k) B_k over one orbital (nbas values) for each entry
// e = (buffer of A, row of A, buffer of B, row of B): one block per entry,
// fixed summation order
struct RowDotBufs { const cplx* b[4]; };
__global__ void __launch_bounds__(256) rowdot_kernel(size_t nbas, RowDotBufs bufs, const int4* __restrict__ ent,
                                                     cplx* __restrict__ out) {
  __shared__ double re[256], im[256];
  const int4 e = ent[blockIdx.x];
  const cplx* A = bufs.b[e.x] + (size_t)e.y * nbas;
  const cplx* B = bufs.b[e.z] + (size_t)e.w * nbas;
  double sr = 0.0, si = 0.0;
  for (size_t k = threadIdx.x; k < nbas; k += blockDim.x) {
    cplx a = A[k], b = B[k];
    sr += a.x * b.x + a.y * b.y;
    si += a.x * b.y - a.y * b.x;
  }
  re[threadIdx.x] = sr; im[threadIdx.x] = si;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) { re[threadIdx.x] += re[threadIdx.x + w]; im[threadIdx.x] += im[threadIdx.x + w]; }
    __syncthreads();
  }
  if (threadIdx.x == 0) out[blockIdx.x] = mkc(re[0], im[0]);
}

// out = Re sum conj(a) b over n complex values (one block, fixed order)
__global__ void __launch_bounds__(256) dot_re_kernel(const cplx* __restrict__ a, const cplx* __restrict__ b, size_t n, double* out) {
  __shared__ double red[256];
  double s = 0.0;
  for (size_t k = threadIdx.x; k < n; k += blockDim.x) s += a[k].x * b[k].x + a[k].y * b[k].y;
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) { if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w]; __syncthreads(); }
  if (threadIdx.x == 0) *out = red[0];
}

// ===========================================================================
// per-RHS small kernels
// ===========================================================================
// frozen core in the velocity gauge: orbg_fc = sph2ang1(orb0_fc) exp(-i A r cos th)
// (hprod_orbin.F90:68-105)
__global__ void fc_phase_kernel(int Nr, int nlat, int nfcore, const double* __restrict__ xrad, const double* __restrict__ cost,
                                const double* __restrict__ lfield, const cplx* __restrict__ orbg0, cplx* __restrict__ orbg) {
  size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  size_t n = (size_t)Nr * nlat * nfcore;
  if (t >= n) return;
  int r = t % Nr, th = (t / Nr) % nlat;
  double ph = lfield[8] * xrad[r + 1] * cost[th];
  double s, c;
  sincos(ph, &s, &c);
  orbg[t] = cmul(orbg0[t], mkc(c, -s));
}

// Hermitian regularised inverse U diag(d/(d^2+thr)) U^H (hprod_invden.F90:62-107;
// zheev replaced by a complex Jacobi).  One warp; the rotations of a sweep are
// grouped into rounds of disjoint (p,q) pairs (round-robin ordering), so each
// round applies all its rotations at once: columns (A U, V U) then rows
// (U^H A).  n <= 16.
__device__ void herm_reg_inverse_warp(int n, double thr, const cplx* a, cplx* inv, cplx* A, cplx* V, int* status) {
  const int lane = threadIdx.x & 31;
  __shared__ double rc[2][8], rs[2][8];
  __shared__ cplx re[2][8];
  __shared__ int rp[2][8], rq[2][8];
  const int wsel = (threadIdx.x >> 5) & 1;
  for (int e = lane; e < n * n; e += 32) { A[e] = a[e]; V[e] = mkc((e % n) == (e / n) ? 1.0 : 0.0, 0.0); }
  __syncwarp();
  const int N = (n + 1) & ~1;  // players of the round-robin schedule (one dummy if n is odd)
  bool conv = (n <= 1);
  for (int sweep = 0; sweep < 60 && !conv; ++sweep) {
    double off = 0, dg = 0;
    for (int e = lane; e < n * n; e += 32) { if ((e % n) != (e / n)) off += cabs2(A[e]); else dg += cabs2(A[e]); }
    for (int o = 16; o > 0; o >>= 1) { off += __shfl_xor_sync(0xffffffff, off, o); dg += __shfl_xor_sync(0xffffffff, dg, o); }
    // converged at the rounding floor of a cyclic Jacobi, |off|^2 ~ (n eps)^2 |diag|^2
    if (off <= 1e-30 * fmax(dg, 1e-300)) { conv = true; break; }
    for (int rnd = 0; rnd < N - 1; ++rnd) {
      // rotation parameters of this sweep stage's disjoint pairs
      if (lane < N / 2) {
        const int i = lane;
        auto player = [&](int pos) { return pos == 0 ? 0 : ((pos - 1 + rnd) % (N - 1)) + 1; };
        int p = player(i), q = player(N - 1 - i);
        if (p > q) { int tt = p; p = q; q = tt; }
        double c = 1.0, sn = 0.0;
        cplx e = mkc(1.0, 0.0);
        bool valid = q < n;
        if (valid) {
          cplx apq = A[p + n * q];
          double b = sqrt(cabs2(apq));
          if (b < 1e-300) valid = false;
          else {
            e = cscale(apq, 1.0 / b);
            double app = A[p + n * p].x, aqq = A[q + n * q].x;
            double tau = (aqq - app) / (2 * b);
            double tt = (tau >= 0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1 + tau * tau));
            c = 1 / sqrt(1 + tt * tt); sn = tt * c;
          }
        }
        rp[wsel][i] = valid ? p : -1; rq[wsel][i] = q; rc[wsel][i] = c; rs[wsel][i] = sn; re[wsel][i] = e;
      }
      __syncwarp();
      // columns: A <- A U, V <- V U
      for (int w = lane; w < (N / 2) * n; w += 32) {
        const int i = w / n, k = w % n;
        const int p = rp[wsel][i];
        if (p < 0) continue;
        const int q = rq[wsel][i];
        const double c = rc[wsel][i], sn = rs[wsel][i];
        const cplx em = cconj(re[wsel][i]);
        cplx akp = A[k + n * p], akq = A[k + n * q];
        A[k + n * p] = csub(cscale(akp, c), cscale(cmul(em, akq), sn));
        A[k + n * q] = cadd(cscale(akp, sn), cscale(cmul(em, akq), c));
        cplx vkp = V[k + n * p], vkq = V[k + n * q];
        V[k + n * p] = csub(cscale(vkp, c), cscale(cmul(em, vkq), sn));
        V[k + n * q] = cadd(cscale(vkp, sn), cscale(cmul(em, vkq), c));
      }
      __syncwarp();
      // rows: A <- U^H A
      for (int w = lane; w < (N / 2) * n; w += 32) {
        const int i = w / n, k = w % n;
        const int p = rp[wsel][i];
        if (p < 0) continue;
        const int q = rq[wsel][i];
        const double c = rc[wsel][i], sn = rs[wsel][i];
        const cplx e = re[wsel][i];
        cplx apk = A[p + n * k], aqk = A[q + n * k];
        A[p + n * k] = csub(cscale(apk, c), cscale(cmul(e, aqk), sn));
        A[q + n * k] = cadd(cscale(apk, sn), cscale(cmul(e, aqk), c));
      }
      __syncwarp();
    }
  }
  if (!conv) {  // the sweep limit ran out: fail only when far from converged
    double off = 0, dg = 0;
    for (int e = lane; e < n * n; e += 32) { if ((e % n) != (e / n)) off += cabs2(A[e]); else dg += cabs2(A[e]); }
    for (int o = 16; o > 0; o >>= 1) { off += __shfl_xor_sync(0xffffffff, off, o); dg += __shfl_xor_sync(0xffffffff, dg, o); }
    if (off > 1e-24 * fmax(dg, 1e-300) && lane == 0) atomicOr(status, ST_JACOBI);
  }
  __syncwarp();
  for (int e = lane; e < n * n; e += 32) {
    int i = e % n, j = e / n;
    cplx s = mkc(0, 0);
    for (int k = 0; k < n; ++k) {
      double d = A[k + n * k].x;
      double invd = thr > 0 ? d / (d * d + thr) : 1.0 / d;
      s = cadd(s, cscale(cmulc(V[j + n * k], V[i + n * k]), invd));
    }
    inv[e] = s;
  }
}

__global__ void invden_kernel(int nact, int need_rr, const cplx* __restrict__ den1, cplx* rden, cplx* rrden, int* status) {
  __shared__ cplx sA[2][16 * 16], sV[2][16 * 16], sT[16 * 16];  // nact <= 16
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (w == 0) {
    herm_reg_inverse_warp(nact, 1.0e-15, den1, rden, sA[0], sV[0], status);
  } else if (w == 1) {
    if (need_rr) {
      for (int e = lane; e < nact * nact; e += 32) {
        cplx v = cscale(den1[e], -1.0);
        if ((e % nact) == (e / nact)) v.x += 2.0;
        sT[e] = v;
      }
      __syncwarp();
      herm_reg_inverse_warp(nact, 1.0e-15, sT, rrden, sA[1], sV[1], status);
    } else {
      for (int e = lane; e < nact * nact; e += 32) rrden[e] = mkc(0, 0);
    }
  }
}

struct SmallArgs {
  int nfun, nfcore, ndcore, nact, ncore, nelact, icomp;
  double dtime, ene_fcore;
  const int* mval;
  const int* ent_index;  // [5][nfun][nfun]
  const cplx* res;       // orbdots results
  const cplx* den1; const cplx* den2; const cplx* rrden;
  cplx* int1e; const cplx* int2e;
  cplx* xmat;
  double* ene;           // [5]
};

__device__ __forceinline__ cplx resv(const SmallArgs& a, int kind, int j, int i) {
  int e = a.ent_index[(kind * a.nfun + j) * a.nfun + i];
  return e >= 0 ? a.res[e] : mkc(0, 0);
}

// int1e, energies and the X matrix (hprod_mkint1_sph.F90, hprod_ene_act.F90,
// hprod_ene_dcore.F90, hprod_htot_mkxmat.F90 _fc/_cc/_ca/_ca0/_aa1)
__global__ void __launch_bounds__(256) smallmat_kernel(SmallArgs a) {
  __shared__ double red[256];
  __shared__ cplx F[16 * 16];
  const int n = a.nact, nf = a.nfun, nc = a.ncore, nfc = a.nfcore;
  const int tid = threadIdx.x;
  // int1e(ja, ia) = A(j, i) for ja <= ia, conj fill
  for (int e = tid; e < n * n; e += blockDim.x) {
    int ja = e % n, ia = e / n;
    int j = nc + ja, i = nc + ia;
    cplx v = mkc(0, 0);
    if (a.mval[j] == a.mval[i]) v = (ja <= ia) ? resv(a, 0, j, i) : cconj(resv(a, 0, i, j));
    a.int1e[e] = v;
  }
  // Fock elements F(j,i) = A + B for dynamic j, i of equal m
  for (int e = tid; e < nf * nf; e += blockDim.x) {
    int j = e % nf, i = e / nf;
    F[e] = (j >= nfc && i >= nfc && a.mval[j] == a.mval[i]) ? cadd(resv(a, 0, j, i), resv(a, 1, j, i)) : mkc(0, 0);
  }
  __syncthreads();
  // ene_act = Re sum int1e(i,j) den1(j,i) + 1/2 Re sum int2e(i,j,k,l) den2(j,i,l,k)
  double part = 0.0;
  const int n2 = n * n;
  // thread (ij, g) sums the l = g, g + ng, ... slices of its (i, j): int2e index ij + n2 (k + n l),
  // den2 index ji + n2 (l + n k), no divisions inside the loop
  if (n2 > 0) {
    const int ng = blockDim.x / n2, ij = tid % n2, g = tid / n2;
    if (g < ng) {
      const int i = ij % n, j = ij / n, ji = j + n * i;
      for (int l = g; l < n; l += ng)
        for (int k = 0; k < n; ++k) {
          const cplx p = cmul(a.int2e[ij + n2 * (k + n * l)], a.den2[ji + n2 * (l + n * k)]);
          part += 0.5 * p.x;
        }
    }
  }
  for (int e = tid; e < n2; e += blockDim.x) {
    int i = e % n, j = e / n;
    cplx p = cmul(a.int1e[i + n * j], a.den1[j + n * i]);
    part += p.x;
  }
  red[tid] = part;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) { if (tid < s) red[tid] += red[tid + s]; __syncthreads(); }
  const double ene_act = red[0];
  __syncthreads();
  // ene_dcore = Re sum_{dc} <phi|g + 2(h0+h1)|phi> = Re [A(i,i) + E(i)]
  double ed = 0.0;
  for (int i = nfc; i < nc; ++i) ed += resv(a, 0, i, i).x + resv(a, 3, i, i).x;
  if (tid == 0) {
    a.ene[0] = a.ene_fcore; a.ene[1] = ed; a.ene[2] = a.ene_fcore + ed; a.ene[3] = ene_act;
    a.ene[4] = a.ene_fcore + ed + ene_act;
  }
  // X matrix
  const cplx tfac = a.icomp == 0 ? mkc(a.dtime, 0) : mkc(0, a.dtime);
  for (int e = tid; e < nf * nf; e += blockDim.x) a.xmat[e] = mkc(0, 0);
  __syncthreads();
  // _fc: X(j,i) = tfac (<(h0+h1) phi_j|phi_i> + <phi_j|(g+v2) phi_i>), j frozen, i dynamic
  for (int e = tid; e < nfc * (nf - nfc); e += blockDim.x) {
    int j = e % nfc, i = nfc + e / nfc;
    cplx v = mkc(0, 0);
    if (a.mval[j] == a.mval[i]) v = cadd(resv(a, 2, j, i), resv(a, 4, j, i));
    a.xmat[j + nf * i] = cmul(v, tfac);
  }
  // _cc
  for (int e = tid; e < (nc - nfc) * (nc - nfc); e += blockDim.x) {
    int j = nfc + e % (nc - nfc), i = nfc + e / (nc - nfc);
    a.xmat[j + nf * i] = cmul(F[j + nf * i], tfac);
  }
  // _aa1 (nsub = 1)
  for (int e = tid; e < n * n; e += blockDim.x) {
    int j = nc + e % n, i = nc + e / n;
    if (a.mval[j] == a.mval[i]) a.xmat[j + nf * i] = cmul(F[j + nf * i], tfac);
  }
  // _ca0 / _ca
  if (n > 0 && nc > nfc) {
    if (n * 2 == a.nelact) {
      for (int e = tid; e < (nc - nfc) * n; e += blockDim.x) {
        int i = nfc + e % (nc - nfc), j = nc + e / (nc - nfc);
        a.xmat[j + nf * i] = cmul(F[j + nf * i], tfac);
        a.xmat[i + nf * j] = cmul(F[i + nf * j], tfac);
      }
    } else if (tid == 0) {
      // fmat(j,i) = 2 F(j,i) - sum_k den1(ja,ka) conj(F(i,k)); bmat = -tfac rrden fmat
      for (int i = nfc; i < nc; ++i) {
        cplx Fm[16];
        for (int ja = 0; ja < n; ++ja) {
          int jf = nc + ja;
          cplx t = mkc(0, 0);
          for (int ka = 0; ka < n; ++ka) t = cadd(t, cmul(a.den1[ja + n * ka], cconj(F[i + nf * (nc + ka)])));
          Fm[ja] = csub(cadd(F[jf + nf * i], F[jf + nf * i]), t);
        }
        for (int ja = 0; ja < n; ++ja) {
          int jf = nc + ja;
          cplx t = mkc(0, 0);
          for (int ka = 0; ka < n; ++ka) t = cadd(t, cmul(a.rrden[ja + n * ka], Fm[ka]));
          cplx bm = cscale(cmul(tfac, t), -1.0);
          a.xmat[jf + nf * i] = cadd(cmul(F[jf + nf * i], tfac), bm);
          a.xmat[i + nf * jf] = cadd(cmul(F[i + nf * jf], tfac), cscale(cconj(bm), -1.0));
        }
      }
    }
  }
}

// hwfn_i = tf2 (v2 + g [+ h1 [+ h0]])_i + sum_{j, m_j = m_i} orb_j X(j,i)
// (hprod_htot_dtorb.F90:54-104); frozen-core rows are zero.
__global__ void dtorb_kernel(int Nr, int L1, int nfun, int nfcore, int icomp, int isplit, double dtime, const int* __restrict__ mval,
                             const cplx* __restrict__ orb, const cplx* __restrict__ h0, const cplx* __restrict__ h1,
                             const cplx* __restrict__ gg, const cplx* __restrict__ v2, const cplx* __restrict__ xmat,
                             cplx* __restrict__ hwfn) {
  const size_t nb = (size_t)Nr * L1;
  size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nb * nfun) return;
  const int i = (int)(t / nb);
  const size_t k = t % nb;
  if (i < nfcore) { hwfn[t] = mkc(0, 0); return; }
  const cplx tf2 = icomp == 0 ? mkc(-dtime, 0) : mkc(0, -dtime);
  // isplit 0: v2 + g + h1 + h0; 2: without h0; 1: without h1 and h0 (hprod_htot_dtorb.F90:58-84)
  cplx h = cadd(v2[t], gg[t]);
  if (isplit != 1) h = cadd(h, h1[t]);
  if (isplit == 0) h = cadd(h, h0[t]);
  cplx o = cmul(h, tf2);
  const int mi = mval[i];
  for (int j = 0; j < nfun; ++j) {
    if (mval[j] != mi) continue;
    o = cadd(o, cmul(orb[(size_t)j * nb + k], xmat[j + nfun * i]));
  }
  hwfn[t] = o;
}

// ===========================================================================
// host set-up helpers
// ===========================================================================
// Poisson arguments for the stored pairs pair0 .. pair0 + npair - 1
PoissonArgs poisson_args(const Ctx& c, int npair, int pair0) {
  PoissonArgs pa{};
  pa.Nr = c.Nr; pa.L2 = c.L2; pa.nd = c.nd; pa.npair = npair; pa.d2ll = c.d2ll; pa.d2rinv = c.d2rinv;
  pa.rpl0 = c.rpl0; pa.rpl1 = c.rpl1; pa.invr = c.invr; pa.fac2 = c.fac2; pa.fac1 = c.fac1;
  pa.pair_m = c.pair_m ? c.pair_m + pair0 : nullptr;
  pa.rho2 = c.rho2 ? c.rho2 + (size_t)pair0 * c.nbas2 : nullptr;
  pa.v2sph = c.v2sph ? c.v2sph + (size_t)pair0 * c.nbas2 : nullptr;
  pa.tabf = c.ps_tabf; pa.tabb = c.ps_tabb; pa.status = c.d_status;
  return pa;
}

int build_tables(Ctx& c) {
  const int bw = 2 * c.nd + 1;
  c.xrad = dupload(c.h_xrad);
  c.mask = dupload(c.h_mask);
  c.radk = dupload(c.h_radk);
  c.radk0 = dupload(c.h_radk0);
  c.radp = dupload(c.h_radp);
  c.cost = dupload(c.h_cost);
  // Legendre tables with rows padded to legendre_lda(K) (16-byte aligned, zeros
  // past K) for the tensor-core GEMM: legf (l, theta) -> [theta][l]-major
  // as the reference stores them, i.e. table(m) is [rows][K] with K contiguous
  auto pad_tables = [&](const std::vector<double>& h, int nm, int rows, int K) {
    const int lda = legendre_lda(K);
    std::vector<double> p((size_t)nm * rows * lda, 0.0);
    for (int m = 0; m < nm; ++m)
      for (int r = 0; r < rows; ++r)
        for (int k = 0; k < K; ++k) p[((size_t)m * rows + r) * lda + k] = h[((size_t)m * rows + r) * K + k];
    return dupload(p);
  };
  c.legf1 = pad_tables(c.h_legf1, 2 * c.mmax1 + 1, c.nlat, c.L1);
  c.legb1 = pad_tables(c.h_legb1, 2 * c.mmax1 + 1, c.L1, c.nlat);
  c.legf2 = pad_tables(c.h_legf2, 2 * c.mmax2 + 1, c.nlat, c.L2);
  c.legb2 = pad_tables(c.h_legb2, 2 * c.mmax2 + 1, c.L2, c.nlat);
  (void)bw;
  // alph_lm (bas_gen_alph.F90:2-26)
  std::vector<double> alph((size_t)c.L1 * (2 * c.mmax1 + 1), 0.0);
  for (int m = -c.mmax1; m <= c.mmax1; ++m)
    for (int l = std::abs(m); l <= c.lmax1; ++l)
      alph[(size_t)(m + c.mmax1) * c.L1 + l] = std::sqrt(((l + 1.0) * (l + 1.0) - (double)m * m) / ((2.0 * l + 1) * (2.0 * l + 3)));
  c.alph = dupload(alph);
  // Poisson factors (bas_gen_d2fac.F90:2-60, hprod_mkv2mf.F90:140-142)
  const int Nr = c.Nr;
  std::vector<double> rpl0((size_t)Nr * c.L2), rpl1(rpl0.size()), invr(rpl0.size()), fac2(rpl0.size()), fac1(c.L2);
  const double r2pi = 0.5 / PI;
  for (int l = 0; l <= c.lmax2; ++l) {
    for (int ir = 1; ir <= Nr; ++ir) {
      double x = c.h_xrad[ir], sw = std::sqrt(c.h_wrad[ir]);
      size_t k = (size_t)l * Nr + ir - 1;
      double xl = 1.0;
      for (int e = 0; e < l; ++e) xl *= x;
      rpl0[k] = xl * r2pi;
      rpl1[k] = xl * x * sw;
      invr[k] = (2 * l + 1) / (x * sw) * r2pi;
      fac2[k] = 4.0 * PI / (2 * l + 1) / (x * sw);
    }
    double xr = c.h_xrad[Nr + 1], p = 1.0;
    for (int e = 0; e < 2 * l + 1; ++e) p *= xr;
    fac1[l] = 1.0 / p;
  }
  c.rpl0 = dupload(rpl0); c.rpl1 = dupload(rpl1); c.invr = dupload(invr); c.fac2 = dupload(fac2); c.fac1 = dupload(fac1);
  // Cholesky factors on the device
  c.d2ll = dalloc<double>((size_t)(c.nd + 1) * Nr * c.L2);
  c.d2rinv = dalloc<double>((size_t)Nr * c.L2);
  int* dstat = dalloc<int>(1);
  d2ll_factor_kernel<<<(c.L2 + 31) / 32, 32>>>(Nr, c.nd, c.L2, c.xrad, c.radk, c.d2ll, c.d2rinv, dstat);
  int hst = 0;
  cudaMemcpy(&hst, dstat, sizeof(int), cudaMemcpyDeviceToHost);
  if (hst) { fprintf(stderr, "td1c_b200: Poisson band factorisation failed\n"); return ST_CHOLESKY; }
  {
    const size_t nrow = (size_t)c.L2 * ((Nr + c.nd - 1) / c.nd * c.nd) * poisson_row_width(c.nd);
    c.ps_tabf = dalloc<double>(nrow);
    c.ps_tabb = dalloc<double>(nrow);
    PoissonArgs pa = poisson_args(c, c.npair, 0);
    if (launch_poisson_tables(pa, c.ps_tabf, c.ps_tabb, 0)) return ST_CUDA;
  }
  {
    // condensed factors of the same matrices for the per-RHS solve (the banded
    // factor above serves the frozen-core set-up)
    if (c.nd < 2 || c.nfe < 1 || c.nfe * c.nd - 1 != Nr) return ST_CONFIG;
    PsCond& f = c.ps_cond.f;
    f.nfe = c.nfe; f.nd = c.nd; f.ni = c.nd - 1; f.nb = c.nfe - 1; f.L2 = c.L2; f.Nr = Nr;
    f.er = (f.ni * f.ni + 3 * f.ni + 2 + 1) / 2 * 2;
    f.sr = (3 * f.nd + 1) / 2 * 2;
    const size_t ne = (size_t)c.L2 * f.nfe * f.ni, nbt = (size_t)c.L2 * std::max(1, f.nb);
    f.erec = dalloc<double>((size_t)c.L2 * f.nfe * f.er);
    f.srec = dalloc<double>((size_t)c.L2 * f.nfe * f.sr);
    f.gl = dalloc<double>(ne); f.gr = dalloc<double>(ne); f.vl = dalloc<double>(ne); f.vr = dalloc<double>(ne);
    f.tm = dalloc<double>(nbt); f.tw = dalloc<double>(nbt); f.tu = dalloc<double>(nbt);
    if (launch_ps_cond_setup(f, c.xrad, c.radk, c.invr, c.rpl0, c.rpl1, c.fac2, dstat, 0)) return ST_CUDA;
    cudaMemcpy(&hst, dstat, sizeof(int), cudaMemcpyDeviceToHost);
    if (hst) { fprintf(stderr, "td1c_b200: condensed Poisson factorisation failed\n"); return ST_CHOLESKY; }
  }
  c.tdiag = dalloc<double>((size_t)Nr * c.L1);
  c.v2jfc = dalloc<double>(Nr);
  tdiag_kernel<<<(Nr * c.L1 + 255) / 256, 256>>>(Nr, c.L1, c.nd, c.znuc, c.xrad, c.radk, c.radk0, nullptr, c.tdiag);
  c.d_mval = dupload(c.mval);
  return (int)cudaGetLastError();
}

int build_pairs(Ctx& c) {
  // 'dyn' pairs (a >= b, both dynamic), then 'fc1dyn' (a dynamic, b frozen),
  // then 'fcfc' (set-up only)
  c.pa.clear(); c.pb.clear();
  for (int b = c.nfcore; b < c.nfun; ++b)
    for (int a = b; a < c.nfun; ++a) { c.pa.push_back(a); c.pb.push_back(b); }
  for (int b = 0; b < c.nfcore; ++b)
    for (int a = c.nfcore; a < c.nfun; ++a) { c.pa.push_back(a); c.pb.push_back(b); }
  c.npair = (int)c.pa.size();
  for (int b = 0; b < c.nfcore; ++b)
    for (int a = b; a < c.nfcore; ++a) { c.pa.push_back(a); c.pb.push_back(b); }
  c.npair_all = (int)c.pa.size();
  c.nfcfc = c.npair_all - c.npair;
  std::vector<int> pm(c.npair_all), po(c.nfun * c.nfun, -1), pc(c.nfun * c.nfun, 0);
  for (int p = 0; p < c.npair_all; ++p) {
    int a = c.pa[p], b = c.pb[p];
    pm[p] = c.mval[b] - c.mval[a];
    po[a * c.nfun + b] = p; pc[a * c.nfun + b] = 0;
    if (a != b) { po[b * c.nfun + a] = p; pc[b * c.nfun + a] = 1; }
  }
  c.pair_m = dupload(pm); c.pair_of = dupload(po); c.pair_cj = dupload(pc);
  return 0;
}

int build_state(Ctx& c) {
  c.nbas = (size_t)c.Nr * c.L1; c.nbas2 = (size_t)c.Nr * c.L2; c.ngrid = (size_t)c.Nr * c.nlat;
  const size_t so = c.nbas * c.nfun, sg = c.ngrid * c.nfun;
  c.orb = dalloc<cplx>(so); c.orb0 = dalloc<cplx>(so); c.h0orb = dalloc<cplx>(so); c.h1orb = dalloc<cplx>(so);
  c.gorb = dalloc<cplx>(so); c.v2orb = dalloc<cplx>(so);
  c.orbg0 = dalloc<cplx>(c.ngrid * std::max(1, c.nfcore));
  c.orbg = dalloc<cplx>(sg); c.gorbg = dalloc<cplx>(sg); c.v2orbg = dalloc<cplx>(sg);
  c.rho2 = dalloc<cplx>(c.nbas2 * c.npair_all); c.v2sph = dalloc<cplx>(c.nbas2 * c.npair_all);
  c.W = dalloc<cplx>(c.ngrid * c.npair_all);
  c.wfn_io = dalloc<cplx>(so); c.hwfn_io = dalloc<cplx>(so);
  c.lfield = dalloc<double>(9);
  c.xmat = dalloc<cplx>((size_t)c.nfun * c.nfun);
  c.ene = dalloc<double>(5);
  c.d_status = dalloc<int>(1);
  c.d_scalar = dalloc<double>(4);
  if (!c.orb || !c.W || !c.rho2 || !c.v2sph) return ST_CUDA;
  c.ps_main = poisson_args(c, c.npair, 0);
  c.ps_fcfc = poisson_args(c, c.nfcfc, c.npair);
  if (poisson_encode_maps(c.ps_main) || poisson_encode_maps(c.ps_fcfc)) return ST_CUDA;
  {
    PsCondArgs& a = c.ps_cond;
    a.Nr = c.Nr; a.L2 = c.L2; a.npair = c.npair; a.pair_m = c.pair_m; a.rho2 = c.rho2; a.v2sph = c.v2sph;
    a.fac1 = c.fac1;
    const size_t nl = (size_t)c.L2 * std::max(1, c.npair);
    a.cb = dalloc<cplx>(nl * c.nfe * 2);
    a.tpart = dalloc<cplx>(nl * c.nfe);
    a.xb = dalloc<cplx>(nl * std::max(1, c.nfe - 1));
    a.t = dalloc<cplx>(nl);
  }
  return 0;
}

void batch_upload(LegGemmBatch*& dst, const std::vector<LegGemmBatch>& v) { dst = v.empty() ? nullptr : dupload(v); }

int build_batches(Ctx& c) {
  const int N = 2 * c.Nr;
  const int ld1 = legendre_lda(c.L1), ldn = legendre_lda(c.nlat), ld2 = legendre_lda(c.L2);
  auto lf1 = [&](int m) { return c.legf1 + (size_t)(m + c.mmax1) * c.nlat * ld1; };
  auto lb1 = [&](int m) { return c.legb1 + (size_t)(m + c.mmax1) * c.L1 * ldn; };
  auto lf2 = [&](int m) { return c.legf2 + (size_t)(m + c.mmax2) * c.nlat * ld2; };
  auto lb2 = [&](int m) { return c.legb2 + (size_t)(m + c.mmax2) * c.L2 * ldn; };
  std::vector<LegGemmBatch> v;
  // sph2ang1 of dynamic orbitals: orbg[f] = legf1[m] (nlat x L1) * orb[f] (L1 x 2Nr)
  for (int f = c.nfcore; f < c.nfun; ++f)
    v.push_back({lf1(c.mval[f]), (const double*)(c.orb + f * c.nbas), nullptr, (double*)(c.orbg + f * c.ngrid), N, N, ld1, 0});
  c.n_orbg = (int)v.size(); batch_upload(c.b_orbg, v); v.clear();
  // sph2ang1 of the stored frozen core (set-up): orbg0[f] = legf1 * orb0[f]
  for (int f = 0; f < c.nfcore; ++f)
    v.push_back({lf1(c.mval[f]), (const double*)(c.orb0 + f * c.nbas), nullptr, (double*)(c.orbg0 + f * c.ngrid), N, N, ld1, 0});
  batch_upload(c.b_orbg0, v); v.clear();
  // ang2sph1 of the gauge-transformed frozen core: orb[f] = legb1 (L1 x nlat) * orbg[f]
  for (int f = 0; f < c.nfcore; ++f)
    v.push_back({lb1(c.mval[f]), (const double*)(c.orbg + f * c.ngrid), nullptr, (double*)(c.orb + f * c.nbas), N, N, ldn, 0});
  c.n_orbfc = (int)v.size(); batch_upload(c.b_orbfc, v); v.clear();
  // pair density -> rho2 (M = L2, K = nlat)
  for (int p = 0; p < c.npair; ++p) {
    int a = c.pa[p], b = c.pb[p];
    v.push_back({lb2(c.mval[b] - c.mval[a]), (const double*)(c.orbg + a * c.ngrid), (const double*)(c.orbg + b * c.ngrid),
                 (double*)(c.rho2 + (size_t)p * c.nbas2), N, N, ldn, 0});
  }
  batch_upload(c.b_rho, v); c.h_b_rho = v; v.clear();
  for (int p = c.npair; p < c.npair_all; ++p) {
    int a = c.pa[p], b = c.pb[p];
    v.push_back({lb2(c.mval[b] - c.mval[a]), (const double*)(c.orbg + a * c.ngrid), (const double*)(c.orbg + b * c.ngrid),
                 (double*)(c.rho2 + (size_t)p * c.nbas2), N, N, ldn, 0});
  }
  batch_upload(c.b_rho_fcfc, v); v.clear();
  // W = legf2 (nlat x L2) * v2sph
  for (int p = 0; p < c.npair_all; ++p) {
    int a = c.pa[p], b = c.pb[p];
    v.push_back({lf2(c.mval[b] - c.mval[a]), (const double*)(c.v2sph + (size_t)p * c.nbas2), nullptr,
                 (double*)(c.W + (size_t)p * c.ngrid), N, N, ld2, 0});
  }
  {
    std::vector<LegGemmBatch> v1(v.begin(), v.begin() + c.npair), v2(v.begin() + c.npair, v.end());
    batch_upload(c.b_W, v1); batch_upload(c.b_W_fcfc, v2);
    c.h_b_W = v1;
  }
  v.clear();
  // ang2sph1 of g and v2 for dynamic orbitals (M = L1, K = nlat)
  for (int f = c.nfcore; f < c.nfun; ++f)
    v.push_back({lb1(c.mval[f]), (const double*)(c.gorbg + f * c.ngrid), nullptr, (double*)(c.gorb + f * c.nbas), N, N, ldn, 0});
  for (int f = c.nfcore; f < c.nfun; ++f)
    v.push_back({lb1(c.mval[f]), (const double*)(c.v2orbg + f * c.ngrid), nullptr, (double*)(c.v2orb + f * c.nbas), N, N, ldn, 0});
  c.n_gorb = (int)v.size(); batch_upload(c.b_gorb, v); v.clear();
  for (int f = 0; f < c.nfcore; ++f)
    v.push_back({lb1(c.mval[f]), (const double*)(c.gorbg + f * c.ngrid), nullptr, (double*)(c.gorb + f * c.nbas), N, N, ldn, 0});
  batch_upload(c.b_gorbfc, v);
  return 0;
}

int build_reductions(Ctx& c) {
  // orbdots entries: kind 0 (A) and 1 (B) for dynamic j, i of equal m (and the
  // frozen j for kind 2 (C) and 4 (<phi_j|(g+v2) phi_i>)); kind 3 (E) for dynamic cores
  std::vector<int> idx(5 * c.nfun * c.nfun, -1);
  c.h_ent.clear();
  auto add = [&](int kind, int j, int i) {
    idx[(kind * c.nfun + j) * c.nfun + i] = (int)c.h_ent.size();
    c.h_ent.push_back(make_int4(kind, j, i, 0));
  };
  for (int i = c.nfcore; i < c.nfun; ++i)
    for (int j = c.nfcore; j < c.nfun; ++j)
      if (c.mval[j] == c.mval[i]) { add(0, j, i); add(1, j, i); }
  for (int i = c.nfcore; i < c.nfun; ++i)
    for (int j = 0; j < c.nfcore; ++j)
      if (c.mval[j] == c.mval[i]) { add(2, j, i); add(4, j, i); }
  for (int i = c.nfcore; i < c.ncore; ++i) add(3, i, i);
  c.ent_index = dupload(idx);
  c.od.nbas = (int)c.nbas; c.od.nfun = c.nfun; c.od.nent = (int)c.h_ent.size();
  c.od.orb = c.orb; c.od.h0orb = c.h0orb; c.od.h1orb = c.h1orb; c.od.gorb = c.gorb; c.od.v2orb = c.v2orb;
  c.od.ent = dupload(c.h_ent);
  c.od.partial = dalloc<cplx>((size_t)orbdots_nchunk(c.nbas) * std::max(1, c.od.nent));
  c.od.result = dalloc<cplx>(std::max(1, c.od.nent));
  // int2e blocks by delta = m_i - m_j
  const int n = c.nact, nc = c.ncore;
  std::vector<Int2eBlock> blocks;
  std::vector<int> rows;
  std::vector<int2> cols;
  std::vector<int4> dst;
  if (n > 0) {
    int dmax = 0;
    for (int a = 0; a < n; ++a) for (int b = 0; b < n; ++b) dmax = std::max(dmax, std::abs(c.mval[nc + a] - c.mval[nc + b]));
    for (int d = -dmax; d <= dmax; ++d) {
      std::vector<int> r_ij; std::vector<std::pair<int, int>> rr;
      for (int ia = 0; ia < n; ++ia)
        for (int ja = 0; ja <= ia; ++ja)
          if (c.mval[nc + ia] - c.mval[nc + ja] == d) rr.push_back({ia, ja});
      std::vector<std::pair<int, int>> cc;
      for (int ka = 0; ka < n; ++ka)
        for (int la = 0; la < n; ++la)
          if (c.mval[nc + la] - c.mval[nc + ka] == d) cc.push_back({ka, la});
      if (rr.empty() || cc.empty()) continue;
      // split into chunks: rows <= 24, cols <= 36 (the int2e kernel's CTA tile)
      const int cchunk = std::min((int)cc.size(), 36);
      const int rchunk = 24;
      for (size_t r0 = 0; r0 < rr.size(); r0 += rchunk)
        for (size_t c0 = 0; c0 < cc.size(); c0 += cchunk) {
          int nr = (int)std::min((size_t)rchunk, rr.size() - r0), ncl = (int)std::min((size_t)cchunk, cc.size() - c0);
          Int2eBlock bk{};
          bk.row0 = (int)rows.size(); bk.nrow = nr; bk.col0 = (int)cols.size(); bk.ncol = ncl; bk.ent0 = (int)dst.size();
          for (int x = 0; x < nr; ++x) {
            int ia = rr[r0 + x].first, ja = rr[r0 + x].second;
            rows.push_back(c.pair_of ? 0 : 0);
            // stored pair of (i, j): a = i >= b = j
            int p = -1;
            for (int q = 0; q < c.npair; ++q) if (c.pa[q] == nc + ia && c.pb[q] == nc + ja) p = q;
            rows.back() = p;
          }
          for (int y = 0; y < ncl; ++y) {
            int ka = cc[c0 + y].first, la = cc[c0 + y].second;
            int kf = nc + ka, lf = nc + la, p = -1, cj = 0;
            for (int q = 0; q < c.npair; ++q) {
              if (c.pa[q] == kf && c.pb[q] == lf) { p = q; cj = 0; }
              if (c.pa[q] == lf && c.pb[q] == kf) { p = q; cj = 1; }
            }
            cols.push_back(make_int2(p, cj));
          }
          for (int x = 0; x < nr; ++x)
            for (int y = 0; y < ncl; ++y)
              dst.push_back(make_int4(rr[r0 + x].first, rr[r0 + x].second, cc[c0 + y].first, cc[c0 + y].second));
          blocks.push_back(bk);
        }
    }
  }
  c.i2.nact = n; c.i2.nblocks = (int)blocks.size(); c.i2.nblkent = (int)dst.size(); c.i2.K = c.nbas2;
  c.i2.blocks = dupload(blocks); c.i2.row_pair = dupload(rows); c.i2.col_pair = dupload(cols); c.i2.ent_dst = dupload(dst);
  c.i2.rho2 = c.rho2; c.i2.v2sph = c.v2sph;
  c.int2e = dalloc<cplx>((size_t)std::max(1, n * n * n * n));
  c.i2.int2e = c.int2e;
  // the same entries as DMMA tiles: per Delta the rows ij (i >= j) padded to
  // m-tiles of 8 pairs, the columns kl padded to n-tiles of 8, the entry of
  // (row r, column y) at ent0 + r ncol + y in the (i outer, j inner) x
  // (k outer, l inner) order of the block list above; groups (m-tile x up
  // to I2D_NTMAX n-tiles) are spread over the warps so that the four
  // schedulers of an SM get similar numbers of n-tiles
  {
    std::vector<int> a_pair, a_ent, b_col;
    std::vector<int2> b_pair;
    std::vector<I2dGroup> groups;
    std::vector<int4> dst2;
    int dmax = 0;
    for (int x = 0; x < n; ++x) for (int y = 0; y < n; ++y) dmax = std::max(dmax, std::abs(c.mval[nc + x] - c.mval[nc + y]));
    for (int d = -dmax; d <= dmax && n > 0; ++d) {
      std::vector<std::pair<int, int>> rr, cc;
      for (int ia = 0; ia < n; ++ia)
        for (int ja = 0; ja <= ia; ++ja)
          if (c.mval[nc + ia] - c.mval[nc + ja] == d) rr.push_back({ia, ja});
      for (int ka = 0; ka < n; ++ka)
        for (int la = 0; la < n; ++la)
          if (c.mval[nc + la] - c.mval[nc + ka] == d) cc.push_back({ka, la});
      if (rr.empty() || cc.empty()) continue;
      const int ent0 = (int)dst2.size(), ncl = (int)cc.size();
      const int arow0 = (int)a_pair.size(), brow0 = (int)b_pair.size();
      for (size_t r = 0; r < rr.size(); ++r) {
        int p = -1;
        for (int q = 0; q < c.npair; ++q) if (c.pa[q] == nc + rr[r].first && c.pb[q] == nc + rr[r].second) p = q;
        a_pair.push_back(p); a_ent.push_back(ent0 + (int)r * ncl);
        for (int y = 0; y < ncl; ++y) dst2.push_back(make_int4(rr[r].first, rr[r].second, cc[y].first, cc[y].second));
      }
      while ((a_pair.size() - arow0) % 8) { a_pair.push_back(-1); a_ent.push_back(-1); }
      for (int y = 0; y < ncl; ++y) {
        const int kf = nc + cc[y].first, lf = nc + cc[y].second;
        int p = -1, cj = 0;
        for (int q = 0; q < c.npair; ++q) {
          if (c.pa[q] == kf && c.pb[q] == lf) { p = q; cj = 0; }
          if (c.pa[q] == lf && c.pb[q] == kf) { p = q; cj = 1; }
        }
        b_pair.push_back(make_int2(p, cj)); b_col.push_back(y);
      }
      while ((b_pair.size() - brow0) % 8) { b_pair.push_back(make_int2(-1, 0)); b_col.push_back(-1); }
      const int mtiles = ((int)a_pair.size() - arow0) / 8, ntiles = ((int)b_pair.size() - brow0) / 8;
      for (int mt = 0; mt < mtiles; ++mt)
        for (int nt = 0; nt < ntiles; nt += I2D_NTMAX)
          groups.push_back(I2dGroup{arow0 + 8 * mt, brow0 + 8 * nt, std::min(I2D_NTMAX, ntiles - nt), 0});
    }
    if (dst2.size() != dst.size()) return ST_CONFIG;
    // warp slots: sets of I2D_NW warps x I2D_MAXG groups; within a set the
    // largest groups go first to the scheduler (warp % 4) with the least work
    std::vector<int> order(groups.size());
    for (size_t g = 0; g < order.size(); ++g) order[g] = (int)g;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return groups[x].nnt > groups[y].nnt; });
    const int slots = I2D_NW * I2D_MAXG;
    const int nsets = std::max(1, ((int)groups.size() + slots - 1) / slots);
    std::vector<int> wgrp((size_t)nsets * slots, -1);
    for (int set = 0; set < nsets; ++set) {
      int load[4] = {0, 0, 0, 0}, used[I2D_NW] = {0};
      for (int k = set * slots; k < std::min((int)order.size(), (set + 1) * slots); ++k) {
        const int g = order[k];
        int best = -1;
        for (int w = 0; w < I2D_NW; ++w)
          if (used[w] < I2D_MAXG && (best < 0 || load[w % 4] < load[best % 4])) best = w;
        wgrp[((size_t)set * I2D_NW + best) * I2D_MAXG + used[best]++] = g;
        load[best % 4] += groups[g].nnt;
      }
    }
    I2dArgs& d2 = c.i2d;
    d2.nra = (int)a_pair.size(); d2.nrb = (int)b_pair.size(); d2.ngroups = (int)groups.size(); d2.nblkent = (int)dst2.size();
    d2.K = c.nbas2; d2.rho2 = c.rho2; d2.v2sph = c.v2sph; d2.nsets = nsets;
    d2.a_pair = dupload(a_pair); d2.a_ent = dupload(a_ent); d2.b_pair = dupload(b_pair); d2.b_col = dupload(b_col);
    d2.groups = dupload(groups); d2.warp_group = dupload(wgrp);
    c.i2_dmma = n > 0 && int2e_dmma_fits(d2);
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (c.i2_dmma) {
      // the DMMA plan's entries replace the block list's (same count, its own order)
      c.i2_nsplit = nsm;
      c.i2.ent_dst = dupload(dst2);
    }
    c.i2.partial = dalloc<cplx>((size_t)c.i2_nsplit * std::max(1, c.i2.nblkent));
    d2.partial = reinterpret_cast<double*>(c.i2.partial);
    // the split-TF32 plan: the stored active pairs in compact order and, per entry of the
    // DMMA plan, its row pair, column pair and conjugation (the DMMA plan's choice)
    if (c.i2_dmma) {
      std::vector<int> cpair, compact(c.npair, -1);
      for (int q = 0; q < c.npair; ++q)
        if (c.pa[q] >= nc && c.pb[q] >= nc) { compact[q] = (int)cpair.size(); cpair.push_back(q); }
      std::vector<int4> ent(dst2.size());
      bool okp = !cpair.empty() && cpair.size() <= 64;
      for (size_t e = 0; e < dst2.size() && okp; ++e) {
        const int4 d4 = dst2[e];
        int pr = -1, pc = -1, cj = 0;
        for (int q = 0; q < c.npair; ++q) {
          if (c.pa[q] == nc + d4.x && c.pb[q] == nc + d4.y) pr = q;
          if (c.pa[q] == nc + d4.z && c.pb[q] == nc + d4.w) { pc = q; cj = 0; }
          if (c.pa[q] == nc + d4.w && c.pb[q] == nc + d4.z) { pc = q; cj = 1; }
        }
        if (pr < 0 || pc < 0 || compact[pr] < 0 || compact[pc] < 0) { okp = false; break; }
        ent[e] = make_int4(compact[pr], compact[pc], cj, 0);
      }
      I2tArgs& t = c.i2t;
      t.P = (int)cpair.size(); t.NB = (t.P + 15) / 16 * 16; t.K = c.nbas2; t.nent = (int)ent.size();
      t.rho2 = c.rho2; t.v2sph = c.v2sph; t.partial = c.i2.partial; t.status = c.d_status;
      c.i2_tc = okp && int2e_tc_fits(t);
      if (c.i2_tc) { t.pair = dupload(cpair); t.ent = dupload(ent); }
    }
  }
  // act2 dense blocks: rows ij (i >= j, m_i - m_j = d) in the reference's
  // (i outer, j inner) order, columns kl (m_l - m_k = d) in (k outer, l inner)
  // order, rows chunked by 24
  {
    std::vector<Act2Block> blks;
    std::vector<int2> rws, cls;
    std::vector<Act2Coef> map;
    int coff = 0;
    int dmax = 0;
    for (int a = 0; a < n; ++a) for (int b = 0; b < n; ++b) dmax = std::max(dmax, std::abs(c.mval[nc + a] - c.mval[nc + b]));
    for (int d = -dmax; d <= dmax && n > 0; ++d) {
      std::vector<int2> rr, cc;
      for (int ia = 0; ia < n; ++ia)
        for (int ja = 0; ja <= ia; ++ja)
          if (c.mval[nc + ia] - c.mval[nc + ja] == d) rr.push_back(make_int2(ia, ja));
      for (int ka = 0; ka < n; ++ka)
        for (int la = 0; la < n; ++la)
          if (c.mval[nc + la] - c.mval[nc + ka] == d) cc.push_back(make_int2(ka, la));
      if (rr.empty() || cc.empty()) continue;
      const int col0 = (int)cls.size();
      for (auto& kl : cc) {
        int kf = nc + kl.x, lf = nc + kl.y, p = -1, cj = 0;
        for (int q = 0; q < c.npair; ++q) {
          if (c.pa[q] == kf && c.pb[q] == lf) { p = q; cj = 0; }
          if (c.pa[q] == lf && c.pb[q] == kf) { p = q; cj = 1; }
        }
        cls.push_back(make_int2(p, cj));
      }
      for (size_t r0 = 0; r0 < rr.size(); r0 += 24) {
        Act2Block bk{};
        bk.row0 = (int)rws.size(); bk.nrow = (int)std::min((size_t)24, rr.size() - r0);
        bk.col0 = col0; bk.ncol = (int)cc.size(); bk.coff = coff;
        for (int x = 0; x < bk.nrow; ++x) rws.push_back(rr[r0 + x]);
        for (int y = 0; y < bk.ncol; ++y)
          for (int x = 0; x < bk.nrow; ++x) {
            int ia = rr[r0 + x].x, ja = rr[r0 + x].y, ka = cc[y].x, la = cc[y].y;
            Act2Coef m{};
            m.d2idx = ja + n * (ia + n * (la + n * ka));
            m.dst = coff + y * bk.nrow + x;
            map.push_back(m);
          }
        coff += bk.nrow * bk.ncol;
        blks.push_back(bk);
      }
    }
    c.a2_nblk = (int)blks.size(); c.a2_nrow = (int)rws.size(); c.a2_ncol = (int)cls.size(); c.a2_ncoef = coff;
    c.a2_blk = dupload(blks); c.a2_rows = dupload(rws); c.a2_cols = dupload(cls); c.a2_map = dupload(map);
    c.a2_coef = dalloc<cplx>(std::max(1, coff));
    // the tensor-core form: per Delta one block (rows not chunked) over the
    // same rows list; coefficients C[row][kl] at coff + row pa + kl with pa
    // = 4 mod 8 (double2) and zero padding; padded columns read the zero W row
    std::vector<MfdBlock> dblk;
    std::vector<int2> dcol;
    std::vector<Act2Coef> dmap;
    int dcoff = 0;
    for (size_t b0 = 0; b0 < blks.size();) {
      size_t b1 = b0;  // the row chunks of one Delta share col0
      int nr = 0;
      while (b1 < blks.size() && blks[b1].col0 == blks[b0].col0) nr += blks[b1++].nrow;
      const Act2Block& B = blks[b0];
      MfdBlock db{};
      db.kpad = (B.ncol + 3) / 4 * 4;
      db.pa = db.kpad % 8 == 0 ? db.kpad + 4 : db.kpad;
      db.mt = (nr + 7) / 8; db.col0 = (int)dcol.size(); db.drow0 = B.row0; db.nr = nr; db.coff = dcoff;
      for (int y = 0; y < db.kpad; ++y) dcol.push_back(y < B.ncol ? cls[B.col0 + y] : make_int2(c.npair, 0));
      for (size_t bb = b0; bb < b1; ++bb)
        for (int y = 0; y < blks[bb].ncol; ++y)
          for (int x = 0; x < blks[bb].nrow; ++x) {
            // the chunk's map entry (y, x) sits at coff + y nrow + x, like its slot
            Act2Coef m{};
            m.d2idx = map[blks[bb].coff + y * blks[bb].nrow + x].d2idx;
            m.dst = dcoff + (blks[bb].row0 + x - B.row0) * db.pa + y;
            dmap.push_back(m);
          }
      dcoff += db.mt * 8 * db.pa;
      dblk.push_back(db);
      b0 = b1;
    }
    // per target x the D2V rows in row order: (row, other orbital), conj flag in bit 16
    std::vector<int2> elist;
    std::vector<int> eoff(n + 1, 0);
    for (int x = 0; x < n; ++x) {
      eoff[x] = (int)elist.size();
      for (size_t r = 0; r < rws.size(); ++r) {
        if (rws[r].x == x) elist.push_back(make_int2((int)r, rws[r].y));
        else if (rws[r].y == x && rws[r].x > rws[r].y) elist.push_back(make_int2((int)r, rws[r].x | (1 << 16)));
      }
    }
    eoff[n] = (int)elist.size();
    // (block, m-tile) items over the 4 warps of a CTA, longest first to the
    // least loaded warp; at most 8 per warp
    std::vector<std::pair<int, int2>> items;
    for (size_t b = 0; b < dblk.size(); ++b)
      for (int mt = 0; mt < dblk[b].mt; ++mt) items.push_back({dblk[b].kpad / 4, make_int2((int)b, mt)});
    std::stable_sort(items.begin(), items.end(), [](const std::pair<int, int2>& x, const std::pair<int, int2>& y) { return x.first > y.first; });
    int wload[4] = {0, 0, 0, 0}, wcount[4] = {0, 0, 0, 0};
    bool items_fit = items.size() <= 32;
    for (int w = 0; w < 4; ++w)
      for (int k = 0; k < 8; ++k) c.mf.witem[w][k] = make_int2(-1, -1);
    for (size_t k = 0; k < items.size() && items_fit; ++k) {
      int best = -1;
      for (int w = 0; w < 4; ++w)
        if (wcount[w] < 8 && (best < 0 || wload[w] < wload[best])) best = w;
      c.mf.witem[best][wcount[best]++] = items[k].second;
      wload[best] += items[k].first;
    }
    c.mf.dmma = n > 0 && !dblk.empty() && items_fit;
    c.mf.nblk_d = (int)dblk.size(); c.mf.ndcol = (int)dcol.size(); c.mf.ncoef_d = dcoff; c.mf.nelist = (int)elist.size();
    c.mf.dblk = dupload(dblk); c.mf.dcol = dupload(dcol); c.mf.dmap = dupload(dmap); c.mf.elist = dupload(elist);
    c.mf.eoff = dupload(eoff);
    c.mf.dcoef = dalloc<cplx>(std::max(1, dcoff));
    cudaMemset(c.mf.dcoef, 0, sizeof(cplx) * std::max(1, dcoff));
  }
  // mean-field action arguments (fixed buffers; the tensor maps bind W and orbg)
  MfprodArgs& mf = c.mf;
  mf.ngrid = c.ngrid; mf.nfun = c.nfun; mf.npair = c.npair; mf.W = c.W; mf.orbg = c.orbg; mf.gorbg = c.gorbg;
  mf.v2orbg = c.v2orbg; mf.nact = c.nact; mf.ncore = c.ncore;
  mf.nblk = c.a2_nblk; mf.nrow = c.a2_nrow; mf.ncol = c.a2_ncol; mf.ncoef = c.a2_ncoef; mf.blk = c.a2_blk;
  mf.rows = c.a2_rows; mf.cols = c.a2_cols; mf.coef_map = c.a2_map; mf.coef = c.a2_coef;
  mf.nfcore = c.nfcore; mf.den1 = c.den1; mf.den2 = c.den2; mf.rden = c.rden; mf.mval = c.d_mval;
  mf.pair_of = c.pair_of; mf.pair_cj = c.pair_cj; mf.nelact = c.nelact;
  return 0;
}

int build_ci(Ctx& c) {
  const int n = c.nact;
  c.den1 = dalloc<cplx>(std::max(1, n * n)); c.rden = dalloc<cplx>(std::max(1, n * n)); c.rrden = dalloc<cplx>(std::max(1, n * n));
  c.int1e = dalloc<cplx>(std::max(1, n * n)); c.den2 = dalloc<cplx>((size_t)std::max(1, n * n * n * n));
  if (n == 0) {
    c.lcic = 1;
    c.cic = dalloc<cplx>(1); c.cic_io = dalloc<cplx>(1); c.hcic_io = dalloc<cplx>(1);
    return 0;
  }
  if (n > 16) return ST_CONFIG;
  const int na = c.nela - c.ncore, nb = c.nelb - c.ncore;
  std::vector<int> orbm(n);
  for (int a = 0; a < n; ++a) orbm[a] = c.mval[c.ncore + a];
  auto build = [&](int nel, std::vector<unsigned>& s, std::vector<int>& M, std::vector<int>& idx) {
    std::vector<std::pair<int, unsigned>> tmp;
    for (unsigned b = 0; b < (1u << n); ++b) {
      if (__builtin_popcount(b) != nel) continue;
      int mm = 0;
      for (int a = 0; a < n; ++a) if ((b >> a) & 1u) mm += orbm[a];
      tmp.push_back({mm, b});
    }
    std::sort(tmp.begin(), tmp.end());
    s.clear(); M.clear(); idx.assign(1u << n, -1);
    for (size_t k = 0; k < tmp.size(); ++k) { s.push_back(tmp[k].second); M.push_back(tmp[k].first); idx[tmp[k].second] = (int)k; }
  };
  std::vector<int> Ma, Mb, ia_idx, ib_idx;
  build(na, c.h_stra, Ma, ia_idx);
  build(nb, c.h_strb, Mb, ib_idx);
  c.nstr_a = (int)c.h_stra.size(); c.nstr_b = (int)c.h_strb.size();
  int mmaxa = 0;
  for (int a = 0; a < n; ++a) mmaxa = std::max(mmaxa, std::abs(orbm[a]));
  c.smin = c.mtot - 2 * mmaxa; c.nsec = 4 * mmaxa + 1;
  std::vector<int> soff((size_t)c.nsec * c.nstr_b, -1), sfirst((size_t)c.nsec * c.nstr_b, 0), scnt((size_t)c.nsec * c.nstr_b, 0);
  std::vector<int> ssize(c.nsec, 0), sbase(c.nsec, 0), sdetA, sdetB;
  for (int sec = 0; sec < c.nsec; ++sec) {
    int S = c.smin + sec, off = 0;
    sbase[sec] = (int)sdetA.size();
    for (int ib = 0; ib < c.nstr_b; ++ib) {
      int need = S - Mb[ib], f = -1, cnt = 0;
      for (int ia = 0; ia < c.nstr_a; ++ia) if (Ma[ia] == need) { if (f < 0) f = ia; cnt++; }
      if (cnt > 0) {
        soff[(size_t)sec * c.nstr_b + ib] = off; sfirst[(size_t)sec * c.nstr_b + ib] = f; scnt[(size_t)sec * c.nstr_b + ib] = cnt;
        for (int k = 0; k < cnt; ++k) { sdetA.push_back(f + k); sdetB.push_back(ib); }
        off += cnt;
      }
    }
    ssize[sec] = off;
    c.maxsec = std::max(c.maxsec, off);
  }
  const int sec0 = c.mtot - c.smin;
  c.lcic = ssize[sec0];
  c.h_detoff.assign(c.nstr_b, -1); c.h_afirst.assign(c.nstr_b, 0); c.h_acount.assign(c.nstr_b, 0);
  std::vector<int> deta, detb;
  for (int ib = 0; ib < c.nstr_b; ++ib) {
    c.h_detoff[ib] = soff[(size_t)sec0 * c.nstr_b + ib];
    c.h_afirst[ib] = sfirst[(size_t)sec0 * c.nstr_b + ib];
    c.h_acount[ib] = scnt[(size_t)sec0 * c.nstr_b + ib];
  }
  for (int K = 0; K < c.lcic; ++K) { deta.push_back(sdetA[sbase[sec0] + K]); detb.push_back(sdetB[sbase[sec0] + K]); }
  // D vector offsets (pq = p + n q in sector mtot + m_p - m_q)
  std::vector<long> doff(n * n, 0);
  long tot = 0;
  for (int q = 0; q < n; ++q)
    for (int p = 0; p < n; ++p) {
      int sec = c.mtot + orbm[p] - orbm[q] - c.smin;
      doff[p + n * q] = tot;
      tot += ssize[sec];
    }
  // pq groups by delta = m_p - m_q (group index delta - (smin - mtot))
  std::vector<int> dgrp, dgoff(c.nsec + 1, 0);
  for (int gI = 0; gI < c.nsec; ++gI) {
    int delta = gI + (c.smin - c.mtot);
    dgoff[gI] = (int)dgrp.size();
    for (int q = 0; q < n; ++q)
      for (int p = 0; p < n; ++p)
        if (orbm[p] - orbm[q] == delta) dgrp.push_back(p + n * q);
  }
  dgoff[c.nsec] = (int)dgrp.size();
  // den2 quadruples with m_p - m_q = m_s - m_r
  std::vector<int4> quads;
  for (int s = 0; s < n; ++s)
    for (int r = 0; r < n; ++r)
      for (int q = 0; q < n; ++q)
        for (int p = 0; p < n; ++p)
          if (orbm[p] - orbm[q] == orbm[s] - orbm[r]) quads.push_back(make_int4(p, q, r, s));
  c.spin_sym = (c.smul == 1 && na == nb) ? 1 : 0;
  CiTables& t = c.cit;
  t.nact = n; t.nstr_a = c.nstr_a; t.nstr_b = c.nstr_b; t.mtot = c.mtot; t.spin_sym = c.spin_sym;
  t.smin = c.smin; t.nsec = c.nsec;
  t.stra = dupload(c.h_stra); t.strb = dupload(c.h_strb);
  t.idx_a = dupload(ia_idx); t.idx_b = dupload(ib_idx); t.Ma = dupload(Ma); t.Mb = dupload(Mb);
  t.sec_off = dupload(soff); t.sec_first = dupload(sfirst); t.sec_cnt = dupload(scnt); t.sec_size = dupload(ssize);
  t.dvec_off = dupload(doff); t.det_a = dupload(deta); t.det_b = dupload(detb); t.orb_m = dupload(orbm);
  t.lcic = c.lcic; t.sec_detA = dupload(sdetA); t.sec_detB = dupload(sdetB); t.sec_base = dupload(sbase);
  t.dgrp = dupload(dgrp); t.dgrp_off = dupload(dgoff); t.quads = dupload(quads); t.nquad = (int)quads.size();
  c.Da = dalloc<cplx>(tot); c.Db = dalloc<cplx>(tot); c.T = dalloc<cplx>(tot);
  c.cic = dalloc<cplx>(c.lcic); c.cic_io = dalloc<cplx>(c.lcic); c.hcic_io = dalloc<cplx>(c.lcic);
  return 0;
}

// ===========================================================================
// the RHS
// ===========================================================================
int gemm(Ctx& c, const LegGemmBatch* b, int nb, int M, int K, bool pair) {
  c.launches++;
  return launch_legendre_gemm_mt(b, nb, M, K, 2 * c.Nr, pair, c.tune_mt, c.st);
}
// the int2e K split: the tuned value where one is set (at most the allocated split)
int i2_split(const Ctx& c) {
  const int k = c.tune_i2_split < 0 ? -c.tune_i2_split : c.tune_i2_split;
  return k > 1 || (k == 1 && c.tune_i2_split > 0) ? std::min(k, c.i2_nsplit) : c.i2_nsplit;
}
// the condensed Poisson solve's arguments: in mixed mode 3 the element pass's interior products
// run in split TF32
PsCondArgs ps_args(const Ctx& c) {
  PsCondArgs a = c.ps_cond;
  a.tf32 = c.mixed == 3 ? 1 : 0;
  return a;
}
// int2e: split TF32 on tcgen05 in mixed mode 3, else FP64 DMMA (or the FFMA blocks)
int int2e_run(Ctx& c, cudaStream_t s) {
  if (c.mixed == 3 && c.i2_tc) return launch_int2e_tc(c.i2t, c.i2, i2_split(c), s);
  if (c.i2_dmma) return launch_int2e_dmma(c.i2d, c.i2, i2_split(c), s);
  return launch_int2e(c.i2, i2_split(c), s);
}
int mfprod_run(Ctx& c, cudaStream_t st) {
  MfprodArgs m = c.mf;
  m.max_cta = c.tune_mf_cap;
  return launch_mfprod(m, st);
}
// the mean field's transforms (pair densities theta -> l, pair potentials l -> theta):
// FP64 DMMA, or split TF32 on tcgen05 in the mixed-precision form
int gemm_mf(Ctx& c, const LegGemmBatch* b, int nb, int M, int K, bool pair) {
  if (!c.mixed) return gemm(c, b, nb, M, K, pair);
  c.launches++;
  if (c.mixed != 2 && b == c.b_rho && c.tc_ok_rho) return launch_legendre_tc(c.tc_rho, c.d_status, c.st);
  if (c.mixed != 2 && b == c.b_W && c.tc_ok_W) return launch_legendre_tc(c.tc_W, c.d_status, c.st);
  return launch_legendre_gemm_tf32(b, nb, M, K, 2 * c.Nr, pair, c.d_status, c.st);
}

// the persistent split-TF32 plans of the pair-density (theta -> l) and
// pair-potential (l -> theta) transforms; shapes outside the persistent
// kernel's range keep the per-tile split-TF32 kernel
void build_tc_plans(Ctx& c) {
  if (c.tc_built) return;
  c.tc_built = true;
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (c.npair > 0 && !c.h_b_rho.empty())
    c.tc_ok_rho = legendre_tc_plan(c.h_b_rho, c.b_rho, c.L2, c.nlat, 2 * c.Nr, true, (const double*)c.orbg, c.nfun, nsm, &c.tc_rho,
                                   c.allocs, c.st) == 0;
  if (c.npair > 0 && !c.h_b_W.empty())
    c.tc_ok_W = legendre_tc_plan(c.h_b_W, c.b_W, c.nlat, c.L2, 2 * c.Nr, false, (const double*)c.v2sph, c.npair_all, nsm,
                                 &c.tc_W, c.allocs, c.st) == 0;
}

// report the first failing launcher of an RHS (status ST_CUDA is set by the caller)
int chk(const char* what, int rc) {
  if (rc != 0) fprintf(stderr, "td1c_b200: %s failed: %s\n", what, cudaGetErrorString((cudaError_t)rc));
  return rc;
}

// d_lf: device lfield[9]; wfn/cic device inputs; hwfn/hcic device outputs
int run_htot(Ctx& c, const double* d_lf, const cplx* wfn, const cplx* cic_in, cplx* hwfn, cplx* hcic, double dtime) {
  cudaStream_t st = c.st;
  const size_t so = c.nbas * c.nfun, sg = c.ngrid * c.nfun;
  int rc = 0;
  int iev = 0;
  auto mark = [&]() { if (c.profile && iev < 16) cudaEventRecord(c.ev[iev++], st); };
  mark();
  // scratch initialisation (hprod_htot_init.F90)
  (void)sg;  // gorbg / v2orbg rows of dynamic orbitals are fully written by mfprod
  cudaMemsetAsync(c.gorb, 0, so * sizeof(cplx), st);
  cudaMemsetAsync(c.v2orb, 0, so * sizeof(cplx), st);
  // RDMs (ormas_mkden1/2, hprod_invden)
  CiArgs ca{};
  ca.t = c.cit; ca.cic = cic_in; ca.Da = c.Da; ca.Db = c.Db; ca.T = c.T; ca.den1 = c.den1; ca.den2 = c.den2;
  ca.sigma = hcic; ca.int1e = c.int1e; ca.int2e = c.int2e; ca.ene_act = c.ene + 3; ca.dtime = dtime; ca.icomp = c.icomp;
  // The RDM chain reads only the CI vector, and its first consumer is
  // mfprod: it runs on the side stream, concurrently with the orbital
  // transform, the one-body stencil, the pair densities, the Poisson solve
  // and the l->theta transform, and joins before mfprod (the fork and join are events, so
  // the RK4 step's graph capture takes them in as graph edges).
  const bool fork = c.nact > 0;
  if (fork) {
    cudaStream_t s2 = c.st2;
    cudaEventRecord(c.ev_fork, st);
    cudaStreamWaitEvent(s2, c.ev_fork, 0);
    rc |= chk("ci dvec", launch_ci_dvec(ca, c.maxsec, s2));
    rc |= chk("ci rdm", launch_ci_rdm(ca, s2));
    int need_rr = (c.ncore > 0 && c.nact * 2 != c.nelact) ? 1 : 0;
    invden_kernel<<<1, 64, 0, s2>>>(c.nact, need_rr, c.den1, c.rden, c.rrden, c.d_status);
    cudaEventRecord(c.ev_join, s2);
    c.launches += 6;
  }
  auto join = [&]() { if (fork) cudaStreamWaitEvent(st, c.ev_join, 0); };
  // orbitals (hprod_orbin.F90)
  cudaMemcpyAsync(c.orb + c.nfcore * c.nbas, wfn + c.nfcore * c.nbas, (so - c.nfcore * c.nbas) * sizeof(cplx),
                  cudaMemcpyDeviceToDevice, st);
  if (c.n_orbg) rc |= chk("orbg gemm", gemm(c, c.b_orbg, c.n_orbg, c.nlat, c.L1, false));
  if (c.nfcore > 0) {
    if (c.igauge == 0) {
      cudaMemcpyAsync(c.orb, c.orb0, c.nfcore * c.nbas * sizeof(cplx), cudaMemcpyDeviceToDevice, st);
      cudaMemcpyAsync(c.orbg, c.orbg0, c.nfcore * c.ngrid * sizeof(cplx), cudaMemcpyDeviceToDevice, st);
    } else {
      size_t nfc = c.ngrid * c.nfcore;
      fc_phase_kernel<<<(unsigned)((nfc + 255) / 256), 256, 0, st>>>(c.Nr, c.nlat, c.nfcore, c.xrad, c.cost, d_lf, c.orbg0, c.orbg);
      c.launches++;
      rc |= chk("fc gemm", gemm(c, c.b_orbfc, c.n_orbfc, c.L1, c.nlat, false));
    }
  }
  mark();  // end orbin
  mark();  // end ci_rdm (the chain itself runs on the side stream, forked before orbin)
  // one-body
  OneBodyArgs ob{};
  ob.Nr = c.Nr; ob.L1 = c.L1; ob.nd = c.nd; ob.nfun = c.nfun; ob.nfcore = c.nfcore; ob.mmax1 = c.mmax1; ob.igauge = c.igauge;
  ob.radk = c.radk; ob.radk0 = c.radk0; ob.radp = c.radp; ob.tdiag = c.tdiag; ob.xrad = c.xrad; ob.alph = c.alph;
  ob.mval = c.d_mval; ob.orb = c.orb; ob.h0orb = c.h0orb; ob.h1orb = c.h1orb; ob.lfield = d_lf;
  // the one-body stencil reads only the orbitals and the field: it runs on
  // the third stream, overlapping the mean-field chain, and joins before
  // the orbital matrix elements
  cudaEventRecord(c.ev_ob_fork, st);
  cudaStreamWaitEvent(c.st3, c.ev_ob_fork, 0);
  rc |= chk("onebody", launch_onebody(ob, c.st3));
  cudaEventRecord(c.ev_ob_join, c.st3);
  c.launches++;
  mark();  // end onebody (the stencil itself overlaps the next phases)
  bool i2_forked = false;
  // mean field: computed from the stage's own orbitals, or (mf_external) taken
  // as it stands in W and int2e, where the mean-field predictor of the
  // learned form has written its stage values
  if (c.neltot >= 2 && c.npair > 0 && c.mf_external) {
    mark(); mark();  // no rho_gemm, no poisson
    mark();          // no w_gemm
    join();
    rc |= chk("mfprod", mfprod_run(c, st));
    c.launches += 2;
    mark();  // end mfprod
    rc |= chk("gorb gemm", gemm(c, c.b_gorb, c.n_gorb, c.L1, c.nlat, false));
  } else if (c.neltot >= 2 && c.npair > 0) {
    rc |= chk("rho gemm", gemm_mf(c, c.b_rho, c.npair, c.L2, c.nlat, true));
    mark();  // end rho_gemm
    rc |= chk("poisson", launch_ps_cond(ps_args(c), st));
    c.launches += 3;
    // int2e needs only rho2 and v2sph: third stream, overlapping l->theta,
    // mfprod and the theta->l transforms; then the CI T vectors, which need
    // only int2e and the D vectors of the CI chain; joins before smallmat
    // (a negative tuned split keeps int2e on the main stream, after the mean-field action:
    // its one-CTA-per-SM grid then does not hold the SMs the transforms and mfprod need)
    if (c.nact > 0 && c.tune_i2_split >= 0) {
      cudaEventRecord(c.ev_i2_fork, st);
      cudaStreamWaitEvent(c.st3, c.ev_i2_fork, 0);
      rc |= chk("int2e", int2e_run(c, c.st3));
      cudaStreamWaitEvent(c.st3, c.ev_join, 0);
      rc |= chk("ci tvec", launch_ci_tvec(ca, c.maxsec, c.st3));
      cudaEventRecord(c.ev_i2_join, c.st3);
      c.launches += 4;
      i2_forked = true;
    }
    mark();  // end poisson
    rc |= chk("W gemm", gemm_mf(c, c.b_W, c.npair, c.nlat, c.L2, false));
    mark();  // end w_gemm
    join();
    rc |= chk("mfprod", mfprod_run(c, st));
    c.launches += 2;
    mark();  // end mfprod
    rc |= chk("gorb gemm", gemm(c, c.b_gorb, c.n_gorb, c.L1, c.nlat, false));
  } else {
    join();
    mark(); mark(); mark(); mark();
  }
  mark();  // end gorb_gemm
  // integrals
  cudaStreamWaitEvent(st, c.ev_ob_join, 0);
  rc |= chk("orbdots", launch_orbdots(c.od, st));
  c.launches += 2;
  mark();  // end orbdots
  if (i2_forked) {
    cudaStreamWaitEvent(st, c.ev_i2_join, 0);
  } else if (c.nact > 0) {
    if (!c.mf_external || c.npair == 0) {
      rc |= chk("int2e", int2e_run(c, st));
      c.launches += 3;
    }
    rc |= chk("ci tvec", launch_ci_tvec(ca, c.maxsec, st));  // the CI chain joined before mfprod
    c.launches += 1;
  }
  mark();  // end int2e (its wait for the third stream)
  SmallArgs sa{};
  sa.nfun = c.nfun; sa.nfcore = c.nfcore; sa.ndcore = c.ndcore; sa.nact = c.nact; sa.ncore = c.ncore; sa.nelact = c.nelact;
  sa.icomp = c.icomp; sa.dtime = dtime; sa.ene_fcore = c.ene_fcore; sa.mval = c.d_mval; sa.ent_index = c.ent_index;
  sa.res = c.od.result; sa.den1 = c.den1; sa.den2 = c.den2; sa.rrden = c.rrden; sa.int1e = c.int1e; sa.int2e = c.int2e;
  sa.xmat = c.xmat; sa.ene = c.ene;
  smallmat_kernel<<<1, 256, 0, st>>>(sa);
  c.launches++;
  mark();  // end smallmat
  // CI sigma (ormas_xact2 -> ormas_hcic) on the side stream, concurrently with
  // dtorb (its T vectors were formed after int2e)
  if (c.nact > 0) {
    cudaEventRecord(c.ev_sig_fork, st);
    cudaStreamWaitEvent(c.st2, c.ev_sig_fork, 0);
    rc |= chk("ci sigma", launch_ci_sigma(ca, c.st2));
    cudaEventRecord(c.ev_sig_join, c.st2);
    c.launches += 1;
  } else {
    cudaMemsetAsync(hcic, 0, sizeof(cplx), st);
  }
  mark();  // end ci_sigma (the sigma itself overlaps dtorb)
  // dtorb
  dtorb_kernel<<<(unsigned)((so + 255) / 256), 256, 0, st>>>(c.Nr, c.L1, c.nfun, c.nfcore, c.icomp, c.isplit, dtime, c.d_mval, c.orb,
                                                             c.h0orb, c.h1orb, c.gorb, c.v2orb, c.xmat, hwfn);
  c.launches++;
  if (c.nact > 0) cudaStreamWaitEvent(st, c.ev_sig_join, 0);
  mark();  // end dtorb (and sigma)
  c.nev = iev;
  rc |= chk("rhs tail", (int)cudaGetLastError());
  return rc;
}

// ===========================================================================
// RK4 (clcrk::prop, src/prop/clcrk.cpp:55-87; tableau set_coeff_04 221-235)
// ===========================================================================
// y += wy k ;  ynext = y0 + wn k   (orbitals and CI handled as two segments)
__global__ void rk_combine_kernel(size_t n, cplx* __restrict__ y, const cplx* __restrict__ y0, const cplx* __restrict__ k,
                                  cplx* __restrict__ ynext, double wy, double wn, int do_next) {
  size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  cplx kv = k[t];
  cplx yv = y[t];
  yv.x = fma(wy, kv.x, yv.x); yv.y = fma(wy, kv.y, yv.y);
  y[t] = yv;
  if (do_next) {
    cplx a = y0[t];
    a.x = fma(wn, kv.x, a.x); a.y = fma(wn, kv.y, a.y);
    ynext[t] = a;
  }
}

// wfn_mask (src/wfn/wfn_mask.F90:2-35): orb(irad, l, i) *= mask(irad) for
// dynamic i, l >= |m_i|, irad >= min_irad
__global__ void mask_kernel(int Nr, int L1, int nfun, int nfcore, int min_irad, const int* __restrict__ mval,
                            const double* __restrict__ mask, cplx* __restrict__ y) {
  size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t nb = (size_t)Nr * L1;
  if (t >= nb * nfun) return;
  const int f = (int)(t / nb);
  const int l = (int)((t % nb) / Nr), r = (int)(t % Nr);
  const int am = mval[f] < 0 ? -mval[f] : mval[f];
  if (f < nfcore || l < am || r + 1 < min_irad) return;
  y[t] = cscale(y[t], mask[r + 1]);
}

// copy the fields of the current step (per doubles) from the table
__global__ void field_select_kernel(const double* __restrict__ tab, int* __restrict__ counter, int per,
                                    double* __restrict__ cur) {
  int s = counter[0];
  if (s >= counter[1]) s = counter[1] - 1;  // counter[1] = steps staged in the table
  if (s < 0) s = 0;
  for (int e = threadIdx.x; e < per; e += blockDim.x) cur[e] = tab[(size_t)s * per + e];
}

// z = a x + b y (mode 0) or z = (x - y) a (mode 1); the vector operations of
// the propagators (clhprod_blas.cpp: axpbyz, xmyz, xpyz, scal)
__global__ void lincomb_kernel(size_t n, cplx* __restrict__ z, const cplx* __restrict__ x, const cplx* __restrict__ y,
                               double a, double b, int mode) {
  size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const cplx xv = x[t], yv = y[t];
  cplx o;
  if (mode == 0) { o.x = a * xv.x + b * yv.x; o.y = a * xv.y + b * yv.y; }
  else { o.x = (xv.x - yv.x) * a; o.y = (xv.y - yv.y) * a; }
  z[t] = o;
}
// z = a x + b y with complex a, b (the complex axpy / scal of clh1rat)
__global__ void zaxpby_kernel(size_t n, cplx* z, const cplx* x, const cplx* y, cplx a, cplx b) {
  size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  z[t] = cadd(cmul(a, x[t]), cmul(b, y[t]));
}
__global__ void counter_inc_kernel(int* counter) { if (threadIdx.x == 0) *counter += 1; }

// ST_NONFINITE in *status when any of the n doubles is not finite (the output
// check of the drop-in RHS and of every propagation call)
__global__ void nonfinite_kernel(const double* __restrict__ a, size_t n, int* __restrict__ status) {
  bool bad = false;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    if (!isfinite(a[i])) bad = true;
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(status, ST_NONFINITE);
}
void check_finite(Ctx& c, const void* p, size_t ndouble, cudaStream_t st) {
  if (!ndouble) return;
  const unsigned grid = (unsigned)std::min<size_t>((ndouble + 255) / 256, 148 * 4);
  nonfinite_kernel<<<grid, 256, 0, st>>>((const double*)p, ndouble, c.d_status);
  c.launches++;
}

// The bounded wait of the staged kernels (mbar_wait: an mbarrier phase, given
// up after TMA_WAIT_NS) on a barrier that nothing arrives on: the wait runs
// out and the kernel records ST_TIMEOUT, as the kernels do when a copy or an
// MMA commit never completes.  No copy or MMA is in flight.
__global__ void wait_selftest_kernel(int* __restrict__ status) {
  __shared__ __align__(8) unsigned long long bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x == 0 && !mbar_wait(&bar, 0)) atomicOr(status, ST_TIMEOUT);
}

// sin^2 pulse (clfield1.cpp:15-115 set-up, 253-300 E explicit, 472-500
// A explicit, 573-620 E as the 6-point derivative of A in velocity1)
struct Pulse { double famp, freq, period, numcyc, cep; int igauge; };
double pulse_a(const Pulse& p, double t) {
  if (!(t > 0 && t < p.numcyc * p.period)) return 0.0;
  double env = std::sin(PI * t / (p.numcyc * p.period));
  env *= env;
  return env * p.famp / p.freq * std::sin(p.freq * t + p.cep);
}
double pulse_e(const Pulse& p, double t) {
  if (!(t > 0 && t < p.numcyc * p.period)) return 0.0;
  double env = std::sin(PI * t / (p.numcyc * p.period));
  env *= env;
  return env * p.famp * std::sin(p.freq * t + p.cep);
}
void pulse_lfield(const Pulse& p, double t, double* lf) {
  for (int i = 0; i < 9; ++i) lf[i] = 0.0;
  double A = pulse_a(p, t);
  if (p.igauge == 1) {
    const double dstep = 2 * PI / (1239.84190 / (800.0 * 27.2113845)) / 100000.0;
    double e = 0;
    e += pulse_a(p, t + 3 * dstep) / 60.0;
    e -= pulse_a(p, t + 2 * dstep) / 20.0 * 3.0;
    e += pulse_a(p, t + dstep) / 4.0 * 3.0;
    e -= pulse_a(p, t - dstep) / 4.0 * 3.0;
    e += pulse_a(p, t - 2 * dstep) / 20.0 * 3.0;
    e -= pulse_a(p, t - 3 * dstep) / 60.0;
    lf[2] = A; lf[5] = -e / dstep; lf[8] = A;
  } else {
    double E = pulse_e(p, t);
    lf[2] = E; lf[5] = E; lf[8] = A;
  }
}


// ---------------------------------------------------------------------------
// one-body propagators (h1prop.cu): factor cache and the application of
// h1itr_prop / dpade_prod to the orbitals of a device state
// ---------------------------------------------------------------------------
int h1_factor(Ctx& c, cplx fac, H1Fac* out) {
  for (int i = 0; i < c.n_h1; ++i)
    if (c.h1slot[i].cre == fac.x && c.h1slot[i].cim == fac.y) { *out = c.h1slot[i].f; return 0; }
  if (c.nd < 2 || c.nfe < 1 || (c.nfe * c.nd - 1) != c.Nr) return ST_CONFIG;
  Ctx::H1Slot* sl = nullptr;
  for (int i = 0; i < c.n_h1 && !sl; ++i)
    if (std::isnan(c.h1slot[i].cre)) sl = &c.h1slot[i];  // invalidated by a change of T
  if (sl) {
  } else if (c.n_h1 < Ctx::kH1Slots) {
    sl = &c.h1slot[c.n_h1++];
    H1Fac& f = sl->f;
    f.nfe = c.nfe; f.nd = c.nd; f.ni = c.nd - 1; f.nb = c.nfe - 1; f.L1 = c.L1;
    const size_t ne = (size_t)c.L1 * f.nfe * f.ni, nbt = (size_t)c.L1 * std::max(1, f.nb);
    f.ainv = dalloc<cplx>(ne * f.ni);
    f.gl = dalloc<cplx>(ne); f.gr = dalloc<cplx>(ne); f.vl = dalloc<cplx>(ne); f.vr = dalloc<cplx>(ne);
    f.tdl = dalloc<cplx>(nbt); f.tdi = dalloc<cplx>(nbt); f.tdu = dalloc<cplx>(nbt); f.tdu2 = dalloc<cplx>(nbt);
    f.tpiv = dalloc<int>(nbt);
  } else {
    // all slots taken: rebuild the oldest in place
    for (int i = 0; i < Ctx::kH1Slots - 1; ++i) std::swap(c.h1slot[i], c.h1slot[i + 1]);
    sl = &c.h1slot[Ctx::kH1Slots - 1];
  }
  sl->cre = fac.x; sl->cim = fac.y;
  H1FacSrc src{};
  src.Nr = c.Nr; src.L1 = c.L1; src.nd = c.nd; src.nfe = c.nfe; src.c = fac;
  src.radk = c.radk; src.radk0 = c.radk0; src.tdiag = c.tdiag; src.status = c.d_status;
  int rc = launch_h1fac(src, sl->f, c.st);
  *out = sl->f;
  return rc ? ST_CUDA : 0;
}

int h1_bufs(Ctx& c) {
  if (c.h1_z[0]) return 0;
  const size_t nrow = (size_t)c.nfun * c.L1;
  if (c.nfun - c.nfcore > 64 || h1elem_smem(c.nd, c.nfun) > 220 * 1024) return ST_CONFIG;
  c.h1_z[0] = dalloc<cplx>(nrow * c.nfe * (c.nd - 1));
  c.h1_z[1] = dalloc<cplx>(nrow * c.nfe * (c.nd - 1));
  c.h1_cb = dalloc<cplx>(nrow * c.nfe * 2);
  c.h1_xb = dalloc<cplx>(nrow * std::max(1, c.nfe - 1));
  c.h1_partial = dalloc<double>(h1elem_partials(c.nfe, c.L1));
  c.h1_ticket = dalloc<unsigned>(1);  // zero (dalloc clears)
  c.h1_flags = dalloc<int>(3);
  return 0;
}

// pade = false: h1itr_prop (h1itr_prop.F90:2-175) over dtime, the
// Crank-Nicolson factor 1 + (i dtime / 2) T; pade = true: dpade_prod
// (dpade_prod.F90:2-124), (1 + (i dtime / alpha) (T + V))^-1.  Imaginary
// time (icomp = 0) drops the i.  d_lf: device lfield of the call.  The
// non-frozen orbitals of wfn are replaced.  Launches are fixed in number: a
// first element pass and bridge solve, maxcyc correction cycles (element +
// bridge pass, skipped on the device once the residual norm is below thresh)
// and a last pass that adds the final correction.
int h1_run(Ctx& c, bool pade, cplx fac, cplx zf0, bool allow_cycles, const double* d_lf, cplx* wfn, int maxcyc,
           double thresh);

int h1_apply(Ctx& c, bool pade, const double* d_lf, cplx* wfn, double dtime, cplx alpha, int maxcyc, double thresh) {
  const bool rt = c.icomp == 1;
  cplx fac, zf0;  // M = 1 + fac T; laser factor zf0 * lfield[2]
  if (pade) {
    const double den = alpha.x * alpha.x + alpha.y * alpha.y;
    const cplx ia = mkc(alpha.x / den, -alpha.y / den);  // 1 / alpha
    fac = rt ? cmul(mkc(0, dtime), ia) : cmul(mkc(dtime, 0), ia);
    zf0 = rt ? cmul(mkc(0, -dtime), ia) : cmul(mkc(-dtime, 0), ia);
  } else {
    fac = rt ? mkc(0, dtime * 0.5) : mkc(dtime * 0.5, 0);
    zf0 = rt ? mkc(0, -dtime * 0.5) : mkc(-dtime * 0.5, 0);
  }
  return h1_run(c, pade, fac, zf0, true, d_lf, wfn, maxcyc, thresh);
}

// h1itr (pade false) or the shifted inverse (1 + fac (T + V))^-1 (pade true)
// of the non-frozen orbitals, the laser by correction cycles of factor
// zf0 lfield[2] when isplit is 1 and allow_cycles
int h1_run(Ctx& c, bool pade, cplx fac, cplx zf0, bool allow_cycles, const double* d_lf, cplx* wfn, int maxcyc,
           double thresh) {
  cudaStream_t st = c.st;
  int rc = h1_bufs(c);
  if (rc) return rc;
  H1Fac F;
  rc = h1_factor(c, fac, &F);
  if (rc) return rc;
  H1ElemArgs E{};
  E.fac = F; E.Nr = c.Nr; E.L1 = c.L1; E.nfun = c.nfun; E.nfcore = c.nfcore; E.mmax1 = c.mmax1; E.igauge = c.igauge;
  E.mval = c.d_mval; E.radk = c.radk; E.radk0 = c.radk0; E.radp = c.radp; E.tdiag = c.tdiag; E.xrad = c.xrad;
  E.alph = c.alph; E.lfield = d_lf; E.cb = c.h1_cb; E.xb = c.h1_xb; E.torb = wfn;
  E.thresh = thresh; E.norm_div = (double)c.nfun; E.partial = c.h1_partial; E.ticket = c.h1_ticket;
  E.done = c.h1_flags; E.ncyc = c.h1_flags + 1;
  E.iter = c.h1_flags + 2; E.zb0 = c.h1_z[0]; E.zb1 = c.h1_z[1]; E.iter_mode = 0;
  for (int f = 0; f < c.nfun && f < 16; ++f) E.mv[f] = c.mval[f];
  cudaMemsetAsync(c.h1_flags, 0, 3 * sizeof(int), st);
  int zb = 0;  // z buffer the next pass writes
  // h1itr also solves the frozen-core columns once: their first correction
  // enters the residual norm of the first cycle (h1itr_prop.F90:105-129)
  const int f_first = pade ? c.nfcore : 0;
  // first right-hand side: wfn (dpade) or wfn + zfac1 (T + zfield V) wfn (h1itr)
  E.finalize = 0; E.make_rhs = 1; E.check_skip = 0; E.f_rhs = f_first; E.f_fin = c.nfun; E.in = wfn;
  E.a = mkc(1, 0);
  E.b = pade ? mkc(0, 0) : zf0;
  E.cz0 = (!pade && c.isplit == 1) ? zf0 : mkc(0, 0);
  E.z_in = c.h1_z[1 - zb]; E.z_out = c.h1_z[zb];
  rc |= launch_h1elem(E, st);
  rc |= launch_h1bridge(E, st);
  c.launches += 2;
  zb = 1 - zb;
  const bool cycles = c.isplit == 1 && maxcyc > 0 && allow_cycles;
  cudaStreamCaptureStatus cst = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(st, &cst);
  if (cycles && cst == cudaStreamCaptureStatusActive) {
    // inside a graph capture: the correction cycles become a conditional
    // while-loop node whose body (element pass, bridge pass, loop control)
    // runs until the residual norm is below thresh or maxcyc cycles have run;
    // the control kernel advances the cycle counter every iteration, so the
    // loop ends after at most maxcyc iterations
    E.a = mkc(0, 0); E.b = mkc(0, 0); E.cz0 = zf0; E.in = nullptr;
    E.f_first = f_first;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndep = 0;
    cudaStreamCaptureStatus cs2;
    if (cudaStreamGetCaptureInfo(st, &cs2, nullptr, &g, &deps, &ndep) != cudaSuccess) return ST_CUDA;
    cudaGraphConditionalHandle hnd;
    if (cudaGraphConditionalHandleCreate(&hnd, g, 1, cudaGraphCondAssignDefault) != cudaSuccess) return ST_CUDA;
    cudaGraphNodeParams np{};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = hnd;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    if (cudaGraphAddNode(&node, g, deps, ndep, &np) != cudaSuccess) return ST_CUDA;
    cudaGraph_t body = np.conditional.phGraph_out[0];
    if (cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies) != cudaSuccess) return ST_CUDA;
    if (cudaStreamBeginCaptureToGraph(c.st4, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
      return ST_CUDA;
    E.finalize = 1; E.do_norm = 1; E.make_rhs = 1; E.check_skip = 1; E.f_rhs = c.nfcore; E.iter_mode = 1;
    rc |= launch_h1elem(E, c.st4);
    rc |= launch_h1bridge(E, c.st4);
    rc |= launch_h1loop_ctl(c.h1_flags + 2, c.h1_flags, maxcyc, hnd, c.st4);
    cudaGraph_t body_out = nullptr;
    if (cudaStreamEndCapture(c.st4, &body_out) != cudaSuccess) return ST_CUDA;
    c.launches += 3;
    E.finalize = 1; E.do_norm = 0; E.make_rhs = 0; E.f_fin = c.nfcore; E.f_rhs = c.nfun;
    E.accumulate = 1; E.check_skip = 1; E.iter_mode = 2;
    rc |= launch_h1elem(E, st);
    c.launches++;
    return rc ? ST_CUDA : 0;
  }
  if (cycles) {
    E.a = mkc(0, 0); E.b = mkc(0, 0); E.cz0 = zf0; E.in = nullptr;
    for (int k = 1; k <= maxcyc; ++k) {
      E.finalize = 1; E.do_norm = 1; E.make_rhs = 1; E.check_skip = 1;
      E.f_fin = k == 1 ? f_first : c.nfcore;
      E.accumulate = k > 1;
      E.f_rhs = c.nfcore;
      E.z_in = c.h1_z[1 - zb]; E.z_out = c.h1_z[zb];
      rc |= launch_h1elem(E, st);
      rc |= launch_h1bridge(E, st);
      c.launches += 2;
      zb = 1 - zb;
    }
  }
  // the last correction (or the only solve) into torb
  E.finalize = 1; E.do_norm = 0; E.make_rhs = 0; E.f_fin = c.nfcore; E.f_rhs = c.nfun;
  E.accumulate = cycles ? 1 : 0; E.check_skip = cycles ? 1 : 0;
  E.z_in = c.h1_z[1 - zb]; E.z_out = c.h1_z[zb];
  rc |= launch_h1elem(E, st);
  c.launches++;
  return rc ? ST_CUDA : 0;
}

// the four stages of clcrk::prop (clcrk.cpp:55-87, set_coeff_04 221-235)
// from the state (y_orb, y_cic), stage fields lf[0..35] on the device
int rk4_stages(Ctx& c, cplx* y_orb, cplx* y_cic, double dt, const double* lf) {
  cudaStream_t st = c.st;
  const size_t no = c.nbas * c.nfun, nc = c.lcic;
  RkBufs& b = c.rk;
  const double wts[4] = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0};
  const double anext[4] = {0.5, 0.5, 1.0, 0.0};
  cudaMemcpyAsync(b.y0, y_orb, no * sizeof(cplx), cudaMemcpyDeviceToDevice, st);
  cudaMemcpyAsync(b.y0 + no, y_cic, nc * sizeof(cplx), cudaMemcpyDeviceToDevice, st);
  int rc = 0;
  for (int is = 0; is < 4; ++is) {
    const cplx* in = (is == 0) ? b.y0 : b.yt;
    rc |= run_htot(c, lf + 9 * is, in, in + no, b.k, b.k + no, 1.0);
    const int nxt = is < 3 ? 1 : 0;
    rk_combine_kernel<<<(unsigned)((no + 255) / 256), 256, 0, st>>>(no, y_orb, b.y0, b.k, b.yt, dt * wts[is], dt * anext[is], nxt);
    rk_combine_kernel<<<(unsigned)((nc + 255) / 256), 256, 0, st>>>(nc, y_cic, b.y0 + no, b.k + no, b.yt + no, dt * wts[is],
                                                                  dt * anext[is], nxt);
    c.launches += 2;
  }
  return rc;
}

// step prologue (fields of the step, optional restart state) and epilogue
// (wfn_mask, step counter)
void step_begin(Ctx& c, cplx* y_orb, cplx* y_cic, int per) {
  cudaStream_t st = c.st;
  RkBufs& b = c.rk;
  field_select_kernel<<<1, 64, 0, st>>>(c.field_tab, b.counter, per, b.lf_cur);
  c.launches++;
  if (b.reset_orb) {
    cudaMemcpyAsync(y_orb, b.reset_orb, c.nbas * c.nfun * sizeof(cplx), cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(y_cic, b.reset_cic, c.lcic * sizeof(cplx), cudaMemcpyDeviceToDevice, st);
  }
}
int step_end(Ctx& c, cplx* y_orb, bool do_mask) {
  cudaStream_t st = c.st;
  const size_t no = c.nbas * c.nfun;
  if (do_mask) {
    int min_irad = 1;
    for (int ir = 1; ir <= c.Nr; ++ir) if (c.h_xrad[ir] > c.rmask) { min_irad = ir; break; }
    mask_kernel<<<(unsigned)((no + 255) / 256), 256, 0, st>>>(c.Nr, c.L1, c.nfun, c.nfcore, min_irad, c.d_mval, c.mask, y_orb);
    c.launches++;
  }
  counter_inc_kernel<<<1, 32, 0, st>>>(c.rk.counter);
  c.launches++;
  return (int)cudaGetLastError();
}

int rk_step(Ctx& c, cplx* y_orb, cplx* y_cic, double dt) {
  step_begin(c, y_orb, y_cic, 36);
  int rc = rk4_stages(c, y_orb, y_cic, dt, c.rk.lf_cur);
  rc |= step_end(c, y_orb, true);
  return rc;
}

// tdse_split2 (tdse.cpp:225-266) with H1P = clh1itr, H2P = clcrk: h1itr over
// dt/2 with the field at t + dt/4, RK4 over dt, h1itr over dt/2 with the
// field at t + 3 dt/4 (clh1itr.cpp:61-94), wfn_mask.  Step fields: the four
// RK4 stages, then the two h1itr fields.
int split2_step(Ctx& c, cplx* y_orb, cplx* y_cic, double dt, int maxcyc, double thresh, bool do_mask) {
  step_begin(c, y_orb, y_cic, 54);
  const bool doh1 = c.isplit != 0, doh2 = c.neltot > 1 || c.isplit != 1;
  const double* lf = c.rk.lf_cur;
  int rc = 0;
  if (doh1) rc |= h1_apply(c, false, lf + 36, y_orb, 0.5 * dt, mkc(0, 0), maxcyc, thresh);
  if (doh2) rc |= rk4_stages(c, y_orb, y_cic, dt, lf);
  if (doh1) rc |= h1_apply(c, false, lf + 45, y_orb, 0.5 * dt, mkc(0, 0), maxcyc, thresh);
  rc |= step_end(c, y_orb, do_mask);
  return rc;
}

// cletdrk2::prop (cletdrk2.cpp:36-61) with cldpade(alpha = 2) and wfn_mask
// (tdse_prop12, tdse.cpp:268-310; init_prop12 does not mask).  Step fields:
// t, t + dt.
int etdrk2_step(Ctx& c, cplx* y_orb, cplx* y_cic, double dt, int maxcyc, double thresh, bool do_mask) {
  cudaStream_t st = c.st;
  step_begin(c, y_orb, y_cic, 18);
  RkBufs& b = c.rk;
  const size_t no = c.nbas * c.nfun, nc = c.lcic, n = no + nc;
  const double* lf = b.lf_cur;
  const unsigned gn = (unsigned)((n + 255) / 256), go = (unsigned)((no + 255) / 256), gc = (unsigned)((nc + 255) / 256);
  cudaMemcpyAsync(b.y0, y_orb, no * sizeof(cplx), cudaMemcpyDeviceToDevice, st);
  cudaMemcpyAsync(b.y0 + no, y_cic, nc * sizeof(cplx), cudaMemcpyDeviceToDevice, st);
  int rc = run_htot(c, lf, b.y0, b.y0 + no, b.k, b.k + no, 1.0);  // hWfn0
  lincomb_kernel<<<gn, 256, 0, st>>>(n, b.yt, b.y0, b.k, 2.0, dt, 0);  // tWfn = 2 Wfn0 + dt hWfn0
  c.launches++;
  if (c.isplit != 0) rc |= h1_apply(c, true, lf, b.yt, dt, mkc(2, 0), maxcyc, thresh);
  lincomb_kernel<<<go, 256, 0, st>>>(no, y_orb, b.yt, b.y0, 1.0, -1.0, 0);  // Wfn1 = tWfn - Wfn0
  lincomb_kernel<<<gc, 256, 0, st>>>(nc, y_cic, b.yt + no, b.y0 + no, 1.0, -1.0, 0);
  c.launches += 2;
  rc |= run_htot(c, lf + 9, y_orb, y_cic, b.k2, b.k2 + no, 1.0);  // hWfn1
  lincomb_kernel<<<gn, 256, 0, st>>>(n, b.yt, b.k2, b.k, 0.5 * dt, 0.0, 1);  // tWfn = (hWfn1 - hWfn0) dt/2
  c.launches++;
  if (c.isplit != 0) rc |= h1_apply(c, true, lf + 9, b.yt, dt, mkc(2, 0), maxcyc, thresh);
  lincomb_kernel<<<go, 256, 0, st>>>(no, y_orb, y_orb, b.yt, 1.0, 1.0, 0);  // Wfn = Wfn1 + tWfn
  lincomb_kernel<<<gc, 256, 0, st>>>(nc, y_cic, y_cic, b.yt + no, 1.0, 1.0, 0);
  c.launches += 2;
  rc |= step_end(c, y_orb, do_mask);
  return rc;
}

// ETD-RK4 (cletdrk4.cpp) with clh1rat (clh1rat.cpp, h1rat_gen.F90,
// h1rat_prod.F90:2-95) at the default orders etd_dim_numer = etd_dim_denom
// = 2.  Each of the six functions is a Pade form n(x) / (dfac (x - r0)(x - r1))
// of x = tunit dt_f H (tunit = -i in real time, -1 in imaginary time), with
// the numerator times pref and the CI part times rk (cletdrk4::gen_exp,
// gen_gfun, gen_f0fun, gen_f1fun, gen_f2fun, cletdrk4.cpp:134-935).
struct Etd4Fun {
  cplx n[3], d0[2], d1[2], rk;
  double dt;
};
Etd4Fun etd4_fun(int which, double dt, int icomp) {
  const std::complex<double> I(0.0, 1.0), tunit = icomp == 0 ? std::complex<double>(-1.0) : -I;
  const double s3 = std::sqrt(3.0);
  double nn[3] = {0, 0, 0}, dfac = 1.0, dtf = dt, pref = 1.0, rk = 1.0;
  std::complex<double> r0, r1;
  switch (which) {
    case 0: case 1:  // exp(x) = (x^2 + 6x + 12) / (x^2 - 6x + 12): exp1 over dt, exp2 over dt/2
      nn[0] = 12; nn[1] = 6; nn[2] = 1; r0 = {3, -s3}; r1 = {3, s3}; dtf = which == 0 ? dt : 0.5 * dt;
      break;
    case 2:  // (exp(x) - 1)/x = (x^2 + 6x + 60) / (3x^2 - 24x + 60), times dt/2 over dt/2
      nn[0] = 60; nn[1] = 6; nn[2] = 1; dfac = 3; r0 = {4, -2}; r1 = {4, 2}; dtf = 0.5 * dt; pref = rk = 0.5 * dt;
      break;
    case 3:  // (-4 - x + e^x (4 - 3x + x^2))/x^3
      nn[0] = 34860; nn[1] = 19620; nn[2] = 2657; dfac = 13260;
      r0 = std::complex<double>(762.0, -std::sqrt(189762.0)) / 221.0; r1 = std::conj(r0); pref = dt; rk = dt / 6.0;
      break;
    case 4:  // 2 (2 + x + e^x (x - 2))/x^3
      nn[0] = 2940; nn[1] = 450; nn[2] = 41; dfac = 330;
      r0 = std::complex<double>(51.0, -std::sqrt(633.0)) / 11.0; r1 = std::conj(r0); pref = dt; rk = dt / 3.0;
      break;
    default:  // (-4 - 3x - x^2 + e^x (4 - x))/x^3
      nn[0] = 1260; nn[1] = -420; nn[2] = -13; dfac = 300;
      r0 = std::complex<double>(21.0, -3.0 * std::sqrt(21.0)) / 5.0; r1 = std::conj(r0); pref = dt; rk = dt / 6.0;
      break;
  }
  auto C = [](std::complex<double> z) { return mkc(z.real(), z.imag()); };
  Etd4Fun F;
  std::complex<double> tt = pref;
  for (int k = 0; k <= 2; ++k) { F.n[k] = C(nn[k] * tt); tt *= tunit; }
  F.d1[0] = C(dfac * tunit * dtf); F.d0[0] = C(-dfac * r0);
  F.d1[1] = C(tunit * dtf); F.d0[1] = C(-r1);
  F.rk = mkc(rk, 0);
  F.dt = dtf;
  return F;
}


void zaxpby(Ctx& c, size_t n, cplx* z, const cplx* x, const cplx* y, cplx a, cplx b) {
  if (!n) return;
  zaxpby_kernel<<<(unsigned)((n + 255) / 256), 256, 0, c.st>>>(n, z, x, y, a, b);
  c.launches++;
}

// clh1rat::prod on the orbitals w: numerator sum_k n_k (dt H1)^k, H1 = T + V
// + laser (hprod_h1tot: the one-body kernel's h0 + h1), then per denominator
// factor (d0 + d1 (T + V))^-1 as the shifted inverse with fac = d1/d0 of the
// input over d0 (laser by correction cycles in real time, isplit 1).  With
// isplit 0 the orbitals are scaled by the function's value at 0.
int h1rat_run(Ctx& c, const Etd4Fun& F, const double* d_lf, cplx* w, int maxcyc, double thresh) {
  const size_t nf = c.nbas * c.nfcore, nd = c.nbas * (c.nfun - c.nfcore), no = c.nbas * c.nfun;
  cudaStream_t st = c.st;
  if (c.isplit == 0) {
    cplx lim = F.n[0];
    for (int k = 0; k < 2; ++k) {
      const double den = F.d0[k].x * F.d0[k].x + F.d0[k].y * F.d0[k].y;
      lim = cmul(lim, mkc(F.d0[k].x / den, -F.d0[k].y / den));
    }
    zaxpby(c, nd, w + nf, w + nf, w + nf, lim, mkc(0, 0));
    return 0;
  }
  int rc = 0;
  cplx* t = c.e4.tmp;
  cudaMemcpyAsync(t, w, no * sizeof(cplx), cudaMemcpyDeviceToDevice, st);
  zaxpby(c, nd, w + nf, w + nf, w + nf, F.n[0], mkc(0, 0));
  OneBodyArgs ob{};
  ob.Nr = c.Nr; ob.L1 = c.L1; ob.nd = c.nd; ob.nfun = c.nfun; ob.nfcore = c.nfcore; ob.mmax1 = c.mmax1; ob.igauge = c.igauge;
  ob.radk = c.radk; ob.radk0 = c.radk0; ob.radp = c.radp; ob.tdiag = c.tdiag; ob.xrad = c.xrad; ob.alph = c.alph;
  ob.mval = c.d_mval; ob.orb = t; ob.h0orb = c.h0orb; ob.h1orb = c.h1orb; ob.lfield = d_lf;
  for (int k = 1; k <= 2; ++k) {
    rc |= launch_onebody(ob, st);
    c.launches++;
    zaxpby(c, nd, t + nf, c.h0orb + nf, c.h1orb + nf, mkc(F.dt, 0), mkc(F.dt, 0));  // t = dt H1 t
    zaxpby(c, nd, w + nf, w + nf, t + nf, mkc(1, 0), F.n[k]);
  }
  for (int k = 0; k < 2; ++k) {
    if (std::hypot(F.d1[k].x, F.d1[k].y) < 1e-10) continue;  // h1rat_thresh
    const double den = F.d0[k].x * F.d0[k].x + F.d0[k].y * F.d0[k].y;
    const cplx inv0 = mkc(F.d0[k].x / den, -F.d0[k].y / den);
    zaxpby(c, nd, w + nf, w + nf, w + nf, inv0, mkc(0, 0));
    const cplx fac = cmul(F.d1[k], inv0);
    rc |= h1_run(c, true, fac, mkc(-fac.x, -fac.y), c.icomp == 1, d_lf, w, maxcyc, thresh);
  }
  return rc ? ST_CUDA : 0;
}

// cletdrk4::prop (cletdrk4.cpp:53-114) and wfn_mask (tdse_prop12).  Step
// fields: t, t + dt/2, t + dt; every function product takes t + dt/2.
int etdrk4_step(Ctx& c, cplx* y_orb, cplx* y_cic, double dt, int maxcyc, double thresh, bool do_mask) {
  cudaStream_t st = c.st;
  step_begin(c, y_orb, y_cic, 27);
  RkBufs& b = c.rk;
  Etd4Bufs& e = c.e4;
  const size_t no = c.nbas * c.nfun, nc = c.lcic, n = no + nc;
  const double* lf = b.lf_cur;
  const double* lh = lf + 9;
  Etd4Fun fn[6];
  for (int k = 0; k < 6; ++k) fn[k] = etd4_fun(k, dt, c.icomp);
  const cplx one = mkc(1, 0), zero = mkc(0, 0);
  int rc = 0;
  // prod1: out = in, CI times rk, orbitals by the function
  auto prod1 = [&](const Etd4Fun& F, const cplx* in, cplx* out) {
    cudaMemcpyAsync(out, in, n * sizeof(cplx), cudaMemcpyDeviceToDevice, st);
    zaxpby(c, nc, out + no, out + no, out + no, F.rk, zero);
    rc |= h1rat_run(c, F, lh, out, maxcyc, thresh);
  };
  cplx *W0 = b.y0, *tW = b.yt, *H0 = b.k, *H1 = b.k2;
  cudaMemcpyAsync(W0, y_orb, no * sizeof(cplx), cudaMemcpyDeviceToDevice, st);
  cudaMemcpyAsync(W0 + no, y_cic, nc * sizeof(cplx), cudaMemcpyDeviceToDevice, st);
  rc |= run_htot(c, lf, W0, W0 + no, H0, H0 + no, 1.0);
  prod1(fn[2], H0, e.w1);
  prod1(fn[1], W0, tW);
  zaxpby(c, n, e.w1, e.w1, tW, one, one);
  rc |= run_htot(c, lf + 9, e.w1, e.w1 + no, H1, H1 + no, 1.0);
  prod1(fn[2], H1, e.w2);
  zaxpby(c, n, e.w2, e.w2, tW, one, one);
  rc |= run_htot(c, lf + 9, e.w2, e.w2 + no, e.h2, e.h2 + no, 1.0);
  zaxpby(c, n, tW, e.h2, H0, mkc(2, 0), mkc(-1, 0));
  prod1(fn[2], tW, e.w3);
  prod1(fn[1], e.w1, tW);
  zaxpby(c, n, e.w3, e.w3, tW, one, one);
  rc |= run_htot(c, lf + 18, e.w3, e.w3 + no, e.h3, e.h3 + no, 1.0);
  zaxpby(c, n, e.h2, e.h2, H1, one, one);
  // Wfn = exp1 Wfn0 + f0 hWfn0 + f1 (hWfn1 + hWfn2) + f2 hWfn3 (prod2 works in place on its input)
  prod1(fn[0], W0, tW);
  const int fi[3] = {3, 4, 5};
  cplx* hin[3] = {H0, e.h2, e.h3};
  for (int q = 0; q < 3; ++q) {
    zaxpby(c, nc, hin[q] + no, hin[q] + no, hin[q] + no, fn[fi[q]].rk, zero);
    rc |= h1rat_run(c, fn[fi[q]], lh, hin[q], maxcyc, thresh);
    zaxpby(c, n, tW, tW, hin[q], one, one);
  }
  cudaMemcpyAsync(y_orb, tW, no * sizeof(cplx), cudaMemcpyDeviceToDevice, st);
  cudaMemcpyAsync(y_cic, tW + no, nc * sizeof(cplx), cudaMemcpyDeviceToDevice, st);
  rc |= step_end(c, y_orb, do_mask);
  return rc;
}

// ---------------------------------------------------------------------------
// the learned form: split2 with the stage mean fields predicted from the
// history of exact step-start mean fields (predictor.cu)
// ---------------------------------------------------------------------------
int lp_setup(Ctx& c) {
  if (mlp_infer_prepare()) return ST_CUDA;
  if (c.lp_alloc) return 0;
  if (c.npair < 1 || c.nfe < 1) return ST_CONFIG;
  LpArgs& a = c.lp;
  a.nfe = c.nfe; a.nd = c.nd; a.Nr = c.Nr; a.nlat = c.nlat; a.npair = c.npair; a.nu = c.npair * c.nfe;
  a.ni = c.nact * c.nact * c.nact * c.nact;
  a.nw = c.ngrid * c.npair;
  a.W = c.W; a.int2e = c.int2e;
  a.ring = dalloc<cplx>(5 * a.nw);
  a.iring = dalloc<cplx>(5 * (size_t)std::max(a.ni, 1));
  a.gram = dalloc<cplx>((size_t)a.nu * 16);
  a.weights = dalloc<cplx>((size_t)a.nu * 4);
  a.err = dalloc<double>(a.nu); a.tnorm = dalloc<double>(a.nu);
  a.judge = dalloc<double>(2);
  a.counter = dalloc<int>(1);
  a.feat = dalloc<float>((size_t)a.nu * 32);
  c.lp_out = dalloc<float>((size_t)a.nu * 8);
  a.net_out = c.lp_out;
  c.lp_mi_status = dalloc<int>(1);
  std::vector<int> kind(c.npair);
  for (int p = 0; p < c.npair; ++p) kind[p] = c.pb[p] < c.nfcore ? 2 : (c.pa[p] == c.pb[p] ? 0 : 1);
  a.pair_kind = dupload(kind);
  a.record = nullptr; a.rec_count = dalloc<int>(1);
  c.lp_save = dalloc<cplx>(c.nbas * c.nfun + c.lcic);
  if (!a.ring || !a.iring || !c.lp_save) return ST_CUDA;
  c.lp_alloc = true;
  return 0;
}

// the exact mean field (W, int2e) of the orbitals wfn: the orbital transform
// with the frozen core's gauge phase of d_lf, the pair densities, Poisson,
// the l -> theta transform and int2e (hprod_htot.F90:44-140's mean-field part)
int run_meanfield(Ctx& c, const cplx* wfn, const double* d_lf) {
  cudaStream_t st = c.st;
  const size_t so = c.nbas * c.nfun;
  int rc = 0;
  cudaMemcpyAsync(c.orb + c.nfcore * c.nbas, wfn + c.nfcore * c.nbas, (so - c.nfcore * c.nbas) * sizeof(cplx),
                  cudaMemcpyDeviceToDevice, st);
  if (c.n_orbg) rc |= chk("orbg gemm", gemm(c, c.b_orbg, c.n_orbg, c.nlat, c.L1, false));
  if (c.nfcore > 0) {
    if (c.igauge == 0) {
      cudaMemcpyAsync(c.orbg, c.orbg0, c.nfcore * c.ngrid * sizeof(cplx), cudaMemcpyDeviceToDevice, st);
    } else {
      size_t nfc = c.ngrid * c.nfcore;
      fc_phase_kernel<<<(unsigned)((nfc + 255) / 256), 256, 0, st>>>(c.Nr, c.nlat, c.nfcore, c.xrad, c.cost, d_lf, c.orbg0, c.orbg);
      c.launches++;
    }
  }
  rc |= chk("rho gemm", gemm_mf(c, c.b_rho, c.npair, c.L2, c.nlat, true));
  rc |= chk("poisson", launch_ps_cond(ps_args(c), st));
  c.launches += 3;
  rc |= chk("W gemm", gemm_mf(c, c.b_W, c.npair, c.nlat, c.L2, false));
  if (c.nact > 0) {
    rc |= chk("int2e", int2e_run(c, st));
    c.launches += 3;
  }
  return rc;
}

// J: exact mean field of the step-start state y, pushed into the history; the
// judge of the last prediction; the network's weights for the next prediction
int lp_j(Ctx& c, const cplx* y, const double* d_lf) {
  cudaStream_t st = c.st;
  int rc = run_meanfield(c, y, d_lf);
  LpArgs a = c.lp;
  a.use_net = c.lp_use_net && c.lp_has_net;
  rc |= chk("lp push", launch_lp_push_judge(a, st));
  c.launches += 3;
  if (a.use_net) {
    rc |= chk("lp features", launch_lp_features(a, st));
    MlpInferArgs mi = c.lp_mi;
    rc |= chk("lp network", launch_mlp_infer_bf16(mi, st));
    c.launches += 2;
  }
  rc |= chk("lp weights", launch_lp_weights(a, st));
  c.launches++;
  return rc;
}

// RK4 of the two-body RHS with the predicted stage mean fields: stage 1 the
// exact W_n, int2e_n (the last J), stages 2 and 3 the c = 1/2 values, stage 4
// the c = 1 values
int lp_rk4_pred(Ctx& c, cplx* y_orb, cplx* y_cic, double dt, const double* lf) {
  cudaStream_t st = c.st;
  const size_t no = c.nbas * c.nfun, nc = c.lcic;
  RkBufs& b = c.rk;
  const double wts[4] = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0};
  const double anext[4] = {0.5, 0.5, 1.0, 0.0};
  cudaMemcpyAsync(b.y0, y_orb, no * sizeof(cplx), cudaMemcpyDeviceToDevice, st);
  cudaMemcpyAsync(b.y0 + no, y_cic, nc * sizeof(cplx), cudaMemcpyDeviceToDevice, st);
  int rc = 0;
  c.mf_external = 1;
  for (int is = 0; is < 4; ++is) {
    if (is == 1 || is == 3) {
      rc |= chk("lp stage", launch_lp_stage(c.lp, is == 1 ? 1 : 0, st));
      c.launches += 2;
    }
    const cplx* in = (is == 0) ? b.y0 : b.yt;
    rc |= run_htot(c, lf + 9 * is, in, in + no, b.k, b.k + no, 1.0);
    const int nxt = is < 3 ? 1 : 0;
    rk_combine_kernel<<<(unsigned)((no + 255) / 256), 256, 0, st>>>(no, y_orb, b.y0, b.k, b.yt, dt * wts[is], dt * anext[is], nxt);
    rk_combine_kernel<<<(unsigned)((nc + 255) / 256), 256, 0, st>>>(nc, y_cic, b.y0 + no, b.k + no, b.yt + no, dt * wts[is],
                                                                  dt * anext[is], nxt);
    c.launches += 2;
  }
  c.mf_external = 0;
  return rc;
}

// the three step kinds of the learned driver: E plain split2; H split2 then J
// of the new state; P split2 with predicted stage mean fields, then J
int lp_step(Ctx& c, int kind, cplx* y, cplx* yc, double dt, int maxcyc, double thresh) {
  if (kind == 0) return split2_step(c, y, yc, dt, maxcyc, thresh, true);
  int rc = 0;
  if (kind == 1) {
    rc |= split2_step(c, y, yc, dt, maxcyc, thresh, true);
  } else {
    step_begin(c, y, yc, 54);
    const double* lf = c.rk.lf_cur;
    rc |= h1_apply(c, false, lf + 36, y, 0.5 * dt, mkc(0, 0), maxcyc, thresh);
    rc |= lp_rk4_pred(c, y, yc, dt, lf);
    rc |= h1_apply(c, false, lf + 45, y, 0.5 * dt, mkc(0, 0), maxcyc, thresh);
    rc |= step_end(c, y, true);
  }
  rc |= lp_j(c, y, c.rk.lf_cur + 27);  // the field at t + dt (the step's last stage field)
  return rc;
}

// Propagation driver of td1c_gpu_rk4 / _split2 / _etdrk2 / _etdrk4 (kind 0 / 1 / 2 / 3):
// stages the fields of every step, then runs the steps eagerly or as one
// CUDA graph per step (captured after one eager step that does the first-call
// set-up: factor tables, scratch, kernel attributes).
int prop_run(int kind, void* d_wfn, void* d_cic, double t0, double dt, int nstep, double fint, double wlen, double numcyc,
             double cep, int maxcyc, double thresh, int use_graph, bool do_mask = true) {
  Ctx& c = ctx();
  if (!c.initialized) return ST_CONFIG;
  if (nstep <= 0) return 0;
  if (kind != 0 && (maxcyc < 0 || !(thresh >= 0.0))) return ST_CONFIG;
  cudaStream_t st = c.st;
  const size_t no = c.nbas * c.nfun, nc = c.lcic;
  RkBufs& b = c.rk;
  if (b.cap < no + nc) {
    b.y0 = dalloc<cplx>(no + nc); b.yt = dalloc<cplx>(no + nc); b.k = dalloc<cplx>(no + nc); b.k2 = dalloc<cplx>(no + nc);
    if (!b.lf_cur) { b.lf_cur = dalloc<double>(54); b.counter = dalloc<int>(2); }
    b.cap = no + nc;
  }
  if (kind == 3 && c.e4.cap < no + nc) {
    Etd4Bufs& e = c.e4;
    for (cplx** q : {&e.w1, &e.w2, &e.w3, &e.h2, &e.h3, &e.tmp}) *q = dalloc<cplx>(no + nc);
    e.cap = no + nc;
  }
  // fields of every step: RK4 stages t + dt c_s (clcrk.cpp:62-73); split2
  // adds the two h1itr fields; ETD-RK2 uses t and t + dt
  Pulse p;
  p.famp = std::sqrt(fint / 3.50944506E+16); p.freq = 1239.84190 / (wlen * 27.2113845);
  p.period = 2 * PI / p.freq; p.numcyc = numcyc; p.cep = cep / 180.0 * PI; p.igauge = c.igauge;
  static const double nodes_rk[4] = {0.0, 0.5, 0.5, 1.0};
  static const double nodes_s2[6] = {0.0, 0.5, 0.5, 1.0, 0.25, 0.75};
  static const double nodes_etd[2] = {0.0, 1.0};
  static const double nodes_etd4[3] = {0.0, 0.5, 1.0};
  const double* nodes = kind == 0 ? nodes_rk : (kind == 1 ? nodes_s2 : (kind == 2 ? nodes_etd : nodes_etd4));
  const int nf = kind == 0 ? 4 : (kind == 1 ? 6 : (kind == 2 ? 2 : 3)), per = 9 * nf;
  std::vector<double> tab((size_t)nstep * per);
  for (int s = 0; s < nstep; ++s)
    for (int is = 0; is < nf; ++is) pulse_lfield(p, t0 + dt * s + dt * nodes[is], &tab[(size_t)s * per + 9 * is]);
  const size_t need = (size_t)nstep * per;
  if ((size_t)c.field_cap < need) {
    const size_t cap = std::max(need, (size_t)65536 * 54);  // keep the table address stable across calls
    c.field_tab = dalloc<double>(cap);
    c.field_cap = (long)cap;
  }
  cudaMemcpyAsync(c.field_tab, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice, st);
  b.h_counter[0] = 0; b.h_counter[1] = nstep;
  cudaMemcpyAsync(b.counter, b.h_counter, 2 * sizeof(int), cudaMemcpyHostToDevice, st);
  c.launches = 0;
  cplx* y = (cplx*)d_wfn;
  cplx* yc = (cplx*)d_cic;
  auto step = [&]() -> int {
    if (kind == 0) return rk_step(c, y, yc, dt);
    if (kind == 1) return split2_step(c, y, yc, dt, maxcyc, thresh, do_mask);
    if (kind == 2) return etdrk2_step(c, y, yc, dt, maxcyc, thresh, do_mask);
    return etdrk4_step(c, y, yc, dt, maxcyc, thresh, do_mask);
  };
  int rc = 0;
  if (!use_graph) {
    for (int s = 0; s < nstep; ++s) rc |= step();
  } else {
    int s0 = 0;
    cudaGraphExec_t& ge = c.graph_exec[kind];
    bool cached;
    const int ctl = c.icomp * 2 + c.igauge + 4 * c.mixed + 8 * c.mf_external;
    if (kind == 0) {
      cached = ge && b.g_y == y && b.g_yc == yc && b.g_tab == c.field_tab && b.g_dt == dt && b.g_ro == b.reset_orb &&
               b.g_ctl == ctl;
    } else {
      const int q = kind - 1;
      cached = ge && b.s_y[q] == y && b.s_yc[q] == yc && b.s_tab[q] == c.field_tab && b.s_dt[q] == dt &&
               b.s_cyc[q] == maxcyc && b.s_thr[q] == thresh && b.s_split[q] == c.isplit &&
               b.s_mask[q] == (int)do_mask && b.s_ro[q] == b.reset_orb && b.s_ctl[q] == ctl;
    }
    if (!cached) {
      rc |= step();
      s0 = 1;
      if (ge) { cudaGraphExecDestroy(ge); ge = nullptr; }
      long l0 = c.launches;
      cudaGraph_t graph;
      if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return ST_CUDA;
      rc |= step();
      if (cudaStreamEndCapture(st, &graph) != cudaSuccess) return ST_CUDA;
      if (cudaGraphInstantiate(&ge, graph, cudaGraphInstantiateFlagUseNodePriority) != cudaSuccess) { cudaGraphDestroy(graph); return ST_CUDA; }
      cudaGraphDestroy(graph);
      const long per_step = c.launches - l0;
      c.launches = l0;
      if (kind == 0) {
        b.g_per = per_step; b.g_y = y; b.g_yc = yc; b.g_tab = c.field_tab; b.g_dt = dt; b.g_ro = b.reset_orb;
        b.g_ctl = ctl;
      } else {
        const int q = kind - 1;
        b.s_per[q] = per_step; b.s_y[q] = y; b.s_yc[q] = yc; b.s_tab[q] = c.field_tab; b.s_dt[q] = dt;
        b.s_cyc[q] = maxcyc; b.s_thr[q] = thresh; b.s_split[q] = c.isplit; b.s_mask[q] = (int)do_mask;
        b.s_ro[q] = b.reset_orb; b.s_ctl[q] = ctl;
      }
    }
    const long per_step = kind == 0 ? b.g_per : b.s_per[kind - 1];
    for (int s = s0; s < nstep; ++s) {
      if (cudaGraphLaunch(ge, st) != cudaSuccess) return ST_CUDA;
      c.launches += per_step;
    }
  }
  check_finite(c, y, 2 * no, st);
  check_finite(c, yc, 2 * nc, st);
  rc |= (int)cudaGetLastError();
  return rc ? ST_CUDA : 0;
}

// The learned split2 driver.  Windows of LP_WIN steps:
//   FILL  the exact mean field of the window's start state, then exact steps
//         that push the history (H), so predictions have four history values;
//   TRY   predicted steps (P); every step's J judges the prediction the last
//         one made; after the window the largest judge value decides: at or
//         below the bound the window stands, above it the state goes back to
//         the window's start and the window is recomputed with exact steps (H);
//   PLAIN exact steps without history (E), the back-off after a rejection
//         (1, 3, 7, ... up to 63 windows), followed by a FILL.
// With record != null only exact steps run (J0 then H), and every J writes its
// training records (nstep + 1 of them, the first four before the history is full).
// stats (10 doubles): windows accepted, rejected, plain, fill; largest judge
// value of an accepted window; smallest and largest window judge value seen;
// predicted steps kept; last window judge value; steps run.
constexpr int LP_WIN = 8;
// The streams of a context. The main stream (and the one-body correction loop's
// body stream) carry the critical path of a step: transforms, Poisson solve,
// mean-field action, integrals, one-body cycles. The side streams carry work that
// only has to be done by a later join (the CI chain, the one-body stencil, int2e
// and the CI T vectors, the sigma vector): they get the lowest priority, so their
// blocks take the SMs the main path leaves free. Captured graphs keep these
// priorities per node (instantiated with cudaGraphInstantiateFlagUseNodePriority).
void make_stream(cudaStream_t* q, bool main) {
  int least = 0, greatest = 0;
  if (cudaDeviceGetStreamPriorityRange(&least, &greatest) != cudaSuccess) least = greatest = 0;
  cudaStreamCreateWithPriority(q, cudaStreamNonBlocking, main ? greatest : least);
}

// windows of exact steps after a judge value above the bound: 1, 3, 7, ... 63, and 63 at
// once when the value is more than ten times the bound (predictions that far off are not
// worth screening again soon)
int lp_next_backoff(int backoff, double judge, double bound) {
  if (!(judge <= 10.0 * bound)) return 63;
  return std::min(2 * backoff + 1, 63);
}

int learned_run(void* d_wfn, void* d_cic, double t0, double dt, int nstep, double fint, double wlen, double numcyc, double cep,
                int maxcyc, double thresh, double* record, double* stats) {
  Ctx& c = ctx();
  if (!c.initialized || c.isplit != 1 || c.npair < 1 || nstep < 0 || maxcyc < 0 || !(thresh >= 0.0)) return ST_CONFIG;
  int rc = lp_setup(c);
  if (rc) return rc;
  cudaStream_t st = c.st;
  const size_t no = c.nbas * c.nfun, nc = c.lcic;
  RkBufs& b = c.rk;
  if (b.cap < no + nc) {
    b.y0 = dalloc<cplx>(no + nc); b.yt = dalloc<cplx>(no + nc); b.k = dalloc<cplx>(no + nc); b.k2 = dalloc<cplx>(no + nc);
    if (!b.lf_cur) { b.lf_cur = dalloc<double>(54); b.counter = dalloc<int>(2); }
    b.cap = no + nc;
  }
  b.reset_orb = nullptr; b.reset_cic = nullptr;
  Pulse pl;
  pl.famp = std::sqrt(fint / 3.50944506E+16); pl.freq = 1239.84190 / (wlen * 27.2113845);
  pl.period = 2 * PI / pl.freq; pl.numcyc = numcyc; pl.cep = cep / 180.0 * PI; pl.igauge = c.igauge;
  static const double nodes[6] = {0.0, 0.5, 0.5, 1.0, 0.25, 0.75};
  const int per = 54;
  std::vector<double> tab((size_t)std::max(nstep, 1) * per);
  for (int s = 0; s < nstep; ++s)
    for (int is = 0; is < 6; ++is) pulse_lfield(pl, t0 + dt * s + dt * nodes[is], &tab[(size_t)s * per + 9 * is]);
  if ((size_t)c.field_cap < tab.size()) {
    const size_t cap = std::max(tab.size(), (size_t)65536 * 54);
    c.field_tab = dalloc<double>(cap);
    c.field_cap = (long)cap;
  }
  cudaMemcpyAsync(c.field_tab, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice, st);
  auto set_step = [&](int s) {
    b.h_counter[0] = s; b.h_counter[1] = nstep;
    cudaMemcpyAsync(b.counter, b.h_counter, 2 * sizeof(int), cudaMemcpyHostToDevice, st);
  };
  set_step(0);
  c.launches = 0;
  cplx* y = (cplx*)d_wfn;
  cplx* yc = (cplx*)d_cic;
  c.lp.record = record;
  cudaMemsetAsync(c.lp.rec_count, 0, sizeof(int), st);
  // captured steps are reused while their inputs are the same; a call that continues the last one
  // (same buffers and pulse, t0 = its end time) keeps the history and the window schedule
  const double key[8] = {dt, fint, wlen, numcyc, cep, (double)maxcyc, thresh,
                         (double)(c.icomp * 2 + c.igauge + 4 * c.mixed + 16 * (c.lp_use_net && c.lp_has_net))};
  bool same = c.lp_key_y == y && c.lp_key_yc == yc && c.lp_key_tab == c.field_tab && !record;
  for (int i = 0; i < 8 && same; ++i) same = c.lp_key[i] == key[i];
  const bool cont = same && std::fabs(t0 - c.lp_t_end) <= 1e-9 * std::max(1.0, std::fabs(t0));
  if (!same || record) {
    for (auto& ge : c.lp_exec) if (ge) { cudaGraphExecDestroy(ge); ge = nullptr; }
    c.lp_key_y = record ? nullptr : y; c.lp_key_yc = record ? nullptr : yc; c.lp_key_tab = c.field_tab;
    for (int i = 0; i < 8; ++i) c.lp_key[i] = key[i];
  }
  if (!cont) {
    cudaMemsetAsync(c.lp.gram, 0, (size_t)c.lp.nu * 16 * sizeof(cplx), st);
    c.lp_mode = 0; c.lp_backoff = 0; c.lp_plain_left = 0;
  }
  // J of the state at step s (the window's start state)
  auto j0 = [&](int s) -> int {
    double lf[9];
    pulse_lfield(pl, t0 + dt * s, lf);
    cudaMemcpyAsync(c.lfield, lf, 9 * sizeof(double), cudaMemcpyHostToDevice, st);
    cudaStreamSynchronize(st);  // lf lives on this frame
    return lp_j(c, y, c.lfield);
  };
  // one step of the given kind: the first step after the graphs were dropped runs eagerly (the
  // first-call set-up: one-body factors, scratch, kernel attributes); the next one captures every
  // kind the call can use (exact, exact + judge, predicted), so that no capture falls inside a
  // later window. The graphs are kept for later calls with the same inputs.
  bool warm = c.lp_exec[0] || c.lp_exec[1] || c.lp_exec[2];
  auto capture = [&](int kind) -> int {
    cudaGraphExec_t& ge = c.lp_exec[kind];
    const long l0 = c.launches;
    cudaGraph_t graph;
    if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return ST_CUDA;
    int r = lp_step(c, kind, y, yc, dt, maxcyc, thresh);
    if (cudaStreamEndCapture(st, &graph) != cudaSuccess || r) return ST_CUDA;
    if (cudaGraphInstantiate(&ge, graph, cudaGraphInstantiateFlagUseNodePriority) != cudaSuccess) { cudaGraphDestroy(graph); return ST_CUDA; }
    cudaGraphDestroy(graph);
    c.lp_exec_launch[kind] = c.launches - l0;
    c.launches = l0;
    return 0;
  };
  auto step = [&](int kind) -> int {
    cudaGraphExec_t& ge = c.lp_exec[kind];
    if (!ge && !warm) {
      warm = true;
      return lp_step(c, kind, y, yc, dt, maxcyc, thresh);
    }
    if (!ge) {
      for (int k = record ? kind : 0; k <= (record ? kind : 2); ++k)
        if (!c.lp_exec[k] && capture(k)) return ST_CUDA;
    }
    if (cudaGraphLaunch(ge, st) != cudaSuccess) return ST_CUDA;
    c.launches += c.lp_exec_launch[kind];
    return 0;
  };
  double stt[10] = {0, 0, 0, 0, 0, 1e300, 0, 0, 0, 0};
  int s = 0;
  if (record) {
    rc |= j0(0);
    for (; s < nstep && !rc; ++s) rc |= step(1);
  } else {
    int mode = c.lp_mode;  // 0 FILL, 1 TRY, 2 PLAIN (continued from the last call when it continues it)
    int backoff = c.lp_backoff, plain_left = c.lp_plain_left;
    const bool can_predict = true;
    while (s < nstep && !rc) {
      const int w = std::min(LP_WIN, nstep - s);
      if (mode == 0) {
        // the exact steps judge every step's prediction as well (their J): once the history
        // is full, the window's judge values decide whether predicted steps are tried at all
        rc |= j0(s);
        for (int k = 0; k < w && !rc; ++k) {
          if (k == 4) cudaMemsetAsync(c.lp.judge, 0, 2 * sizeof(double), st);
          rc |= step(1);
        }
        s += w;
        stt[3] += 1;
        double jd[2] = {0, 0};
        cudaMemcpyAsync(jd, c.lp.judge, 2 * sizeof(double), cudaMemcpyDeviceToHost, st);
        if (cudaStreamSynchronize(st) != cudaSuccess) { rc |= ST_CUDA; break; }
        if (w > 4) { stt[5] = std::min(stt[5], jd[1]); stt[6] = std::max(stt[6], jd[1]); stt[8] = jd[1]; }
        if (w > 4 && can_predict && (!c.lp_screen || (jd[1] <= c.lp_bound && std::isfinite(jd[1])))) {
          mode = 1;
        } else {
          backoff = lp_next_backoff(backoff, w > 4 ? jd[1] : 0.0, c.lp_bound);
          plain_left = backoff;
          mode = w > 4 ? 2 : 0;
        }
      } else if (mode == 1) {
        cudaMemcpyAsync(c.lp_save, y, no * sizeof(cplx), cudaMemcpyDeviceToDevice, st);
        cudaMemcpyAsync(c.lp_save + no, yc, nc * sizeof(cplx), cudaMemcpyDeviceToDevice, st);
        cudaMemsetAsync(c.lp.judge, 0, 2 * sizeof(double), st);
        for (int k = 0; k < w && !rc; ++k) rc |= step(2);
        double jd[2] = {0, 0};
        cudaMemcpyAsync(jd, c.lp.judge, 2 * sizeof(double), cudaMemcpyDeviceToHost, st);
        if (cudaStreamSynchronize(st) != cudaSuccess) { rc |= ST_CUDA; break; }
        const double wj = jd[1];
        stt[8] = wj;
        stt[5] = std::min(stt[5], wj);
        stt[6] = std::max(stt[6], wj);
        if (wj <= c.lp_bound && std::isfinite(wj)) {
          stt[0] += 1; stt[4] = std::max(stt[4], wj); stt[7] += w;
          s += w;
          backoff = 0;
        } else {
          // the window's predictions are rejected: back to its start, recompute it exactly
          stt[1] += 1;
          cudaMemcpyAsync(y, c.lp_save, no * sizeof(cplx), cudaMemcpyDeviceToDevice, st);
          cudaMemcpyAsync(yc, c.lp_save + no, nc * sizeof(cplx), cudaMemcpyDeviceToDevice, st);
          set_step(s);
          rc |= j0(s);
          for (int k = 0; k < w && !rc; ++k) rc |= step(1);
          s += w;
          backoff = lp_next_backoff(backoff, wj, c.lp_bound);
          plain_left = backoff;
          mode = 2;
        }
      } else {
        for (int k = 0; k < w && !rc; ++k) rc |= step(0);
        s += w;
        stt[2] += 1;
        if (--plain_left <= 0) mode = 0;
      }
    }
    c.lp_mode = mode; c.lp_backoff = backoff; c.lp_plain_left = plain_left;
  }
  c.lp_t_end = t0 + dt * s;
  stt[9] = s;
  check_finite(c, y, 2 * no, st);
  check_finite(c, yc, 2 * nc, st);
  c.lp.record = nullptr;
  if (cudaStreamSynchronize(st) != cudaSuccess) rc |= ST_CUDA;
  if (stats) for (int i = 0; i < 10; ++i) stats[i] = stt[i];
  rc |= (int)cudaGetLastError();
  return rc ? ST_CUDA : 0;
}

}  // namespace

// ===========================================================================
// C-ABI
// ===========================================================================
extern "C" {

int td1c_gpu_bind_rad(int nfe, int ndvr, int nrad, const double* xrad, const double* wrad, const double* radp,
                      const double* radk, const double* radk0, double rmask, const double* mask) {
  Ctx& c = ctx();
  c.nfe = nfe; c.nd = ndvr; c.nrad = nrad; c.Nr = nrad - 1; c.rmask = rmask;
  const size_t n1 = nrad + 1, nb = (size_t)(2 * ndvr + 1) * n1;
  c.h_xrad.assign(xrad, xrad + n1); c.h_wrad.assign(wrad, wrad + n1); c.h_mask.assign(mask, mask + n1);
  c.h_radp.assign(radp, radp + nb); c.h_radk.assign(radk, radk + nb); c.h_radk0.assign(radk0, radk0 + nb);
  c.have_rad = true;
  return 0;
}

int td1c_gpu_bind_sph(int lmax1, int lmax2, int mmax1, int mmax2, int nlat, const double* wlat, const double* cost,
                      const double* legf1, const double* legb1, const double* legf2, const double* legb2) {
  Ctx& c = ctx();
  c.lmax1 = lmax1; c.lmax2 = lmax2; c.mmax1 = mmax1; c.mmax2 = mmax2; c.nlat = nlat; c.L1 = lmax1 + 1; c.L2 = lmax2 + 1;
  c.h_wlat.assign(wlat, wlat + nlat); c.h_cost.assign(cost, cost + nlat);
  size_t s1 = (size_t)nlat * c.L1 * (2 * mmax1 + 1), s2 = (size_t)nlat * c.L2 * (2 * mmax2 + 1);
  c.h_legf1.assign(legf1, legf1 + s1); c.h_legb1.assign(legb1, legb1 + s1);
  c.h_legf2.assign(legf2, legf2 + s2); c.h_legb2.assign(legb2, legb2 + s2);
  c.have_sph = true;
  return 0;
}

int td1c_gpu_bind_bas(double znuc, int smul, int mtot, int nfun, const int* otype, const int* mval, const int* lval,
                      int nela, int nelb) {
  Ctx& c = ctx();
  c.znuc = znuc; c.smul = smul; c.mtot = mtot; c.nfun = nfun; c.nela = nela; c.nelb = nelb;
  c.otype.assign(otype, otype + nfun); c.mval.assign(mval, mval + nfun); c.lval.assign(lval, lval + nfun);
  c.nfcore = c.ndcore = c.nact = 0;
  for (int i = 0; i < nfun; ++i) {
    if (otype[i] == -1) c.nfcore++;
    else if (otype[i] == 0) c.ndcore++;
    else if (otype[i] == 1) c.nact++;
    else return ST_CONFIG;
    if (i > 0 && otype[i] < otype[i - 1]) return ST_CONFIG;
  }
  c.ncore = c.nfcore + c.ndcore;
  c.neltot = nela + nelb;
  c.nelact = nela + nelb - 2 * c.ncore;
  c.have_bas = true;
  return 0;
}

int td1c_gpu_bind_ormas(int nsub) {
  Ctx& c = ctx();
  c.nsub = nsub;
  return nsub == 1 ? 0 : ST_CONFIG;
}

int td1c_gpu_bind_control(int icomp, int igauge) {
  Ctx& c = ctx();
  c.icomp = icomp; c.igauge = igauge;
  return 0;
}

int td1c_gpu_bind_split(int split_type) {
  if (split_type < 0 || split_type > 2) return ST_CONFIG;
  ctx().isplit = split_type;
  return 0;
}

void hprod_bind_(double* ene_fcore, double* ene_dcore, double* ene_core, double* ene_act, double* ene_tot, double* dip_exp,
                 double* vel_exp, double* acc_exp, const bool* projhigh, const double* cutoff) {
  Ctx& c = ctx();
  c.p_ene_fcore = ene_fcore; c.p_ene_dcore = ene_dcore; c.p_ene_core = ene_core; c.p_ene_act = ene_act; c.p_ene_tot = ene_tot;
  (void)dip_exp; (void)vel_exp; (void)acc_exp; (void)projhigh; (void)cutoff;
}

void hprod_init_(void) {
  Ctx& c = ctx();
  if (!c.have_rad || !c.have_sph || !c.have_bas) { c.status |= ST_CONFIG; return; }
  if (c.nfun > 16) { c.status |= ST_CONFIG; return; }
  // the active-active rotations of ORMAS with several subspaces
  // (ormas_xact2.F90:46,82) are not built: only CAS (nsub = 1) is accepted
  if (c.nsub != 1) { c.status |= ST_CONFIG; return; }
  // one library stream for the process lifetime: callers may hold it
  // (td1c_gpu_stream) beyond hprod_final_
  static cudaStream_t lib_stream = nullptr, lib_stream2 = nullptr, lib_stream3 = nullptr, lib_stream4 = nullptr;
  if (g_cur == 0) {
    if (!lib_stream4) make_stream(&lib_stream4, true);
    if (!lib_stream) make_stream(&lib_stream, true);
    if (!lib_stream2) make_stream(&lib_stream2, false);
    if (!lib_stream3) make_stream(&lib_stream3, false);
    c.st = lib_stream; c.st2 = lib_stream2; c.st3 = lib_stream3; c.st4 = lib_stream4;
  } else if (!c.st) {
    // an ensemble job: its own streams, so that a graph captured over several
    // jobs (forked from one stream) has no edges between them
    make_stream(&c.st, true); make_stream(&c.st2, false); make_stream(&c.st3, false); make_stream(&c.st4, true);
    c.own_streams = true;
  }
  for (cudaEvent_t* e : {&c.ev_fork, &c.ev_join, &c.ev_ob_fork, &c.ev_ob_join, &c.ev_i2_fork, &c.ev_i2_join,
                         &c.ev_sig_fork, &c.ev_sig_join})
    cudaEventCreateWithFlags(e, cudaEventDisableTiming);
  int rc = build_tables(c);
  rc |= build_pairs(c);
  rc |= build_state(c);
  rc |= build_ci(c);
  rc |= build_batches(c);
  rc |= build_reductions(c);
  cudaDeviceSynchronize();
  rc |= (int)cudaGetLastError();
  if (rc) { c.status |= ST_CUDA; return; }
  c.initialized = true;
}

void hprod_set_wfn0_(const double* wfn, const double* cic, const char* v2xfc_type, int len) {
  Ctx& c = ctx();
  (void)cic; (void)v2xfc_type; (void)len;
  if (!c.initialized) { c.status |= ST_CONFIG; return; }
  cudaStream_t st = c.st;
  const size_t so = c.nbas * c.nfun;
  cudaMemcpyAsync(c.orb0, wfn, so * sizeof(cplx), cudaMemcpyHostToDevice, st);
  c.ene_fcore = 0;
  if (c.nfcore == 0 || c.neltot < 2) {
    cudaMemsetAsync(c.v2jfc, 0, c.Nr * sizeof(double), st);
    cudaStreamSynchronize(st);
    return;
  }
  // sph2ang1 of the stored frozen core (lfield = 0: no gauge phase)
  launch_legendre_gemm(c.b_orbg0, c.nfcore, c.nlat, c.L1, 2 * c.Nr, false, st);
  // frozen-core Hartree potential (hprod_mkrhofc, hprod_mkv2jfc)
  int* d_lval = dupload(c.lval);
  v2jfc_kernel<<<1, 1, 0, st>>>(c.Nr, c.nd, c.L1, c.nfcore, c.d_mval, d_lval, c.orb0, c.d2ll, c.d2rinv, c.rpl0, c.rpl1, c.invr,
                                c.fac2, c.h_xrad[c.Nr + 1], c.v2jfc);
  // frozen-core pair potentials and energy (hprod_v2fc_enefc): orb(fc) = orb0 projected,
  // orbg(fc) = orbg0; fcfc pair densities, Poisson, l->theta
  cudaMemcpyAsync(c.orbg, c.orbg0, c.nfcore * c.ngrid * sizeof(cplx), cudaMemcpyDeviceToDevice, st);
  if (c.igauge == 0) cudaMemcpyAsync(c.orb, c.orb0, c.nfcore * c.nbas * sizeof(cplx), cudaMemcpyDeviceToDevice, st);
  else launch_legendre_gemm(c.b_orbfc, c.nfcore, c.L1, c.nlat, 2 * c.Nr, false, st);  // orb(fc) = ang2sph1(orbg(fc))
  launch_legendre_gemm(c.b_rho_fcfc, c.nfcfc, c.L2, c.nlat, 2 * c.Nr, true, st);
  launch_poisson(c.ps_fcfc, st);
  launch_legendre_gemm(c.b_W_fcfc, c.nfcfc, c.nlat, c.L2, 2 * c.Nr, false, st);
  // frozen-core energy: enefc = 2 Re <phi|h0|phi> + Re <phi| v2jfc - sum_j W(j,i) phi_j >
  // with h0 from the bare kinetic table (before v2jfc is added)
  OneBodyArgs ob{};
  ob.Nr = c.Nr; ob.L1 = c.L1; ob.nd = c.nd; ob.nfun = c.nfcore; ob.nfcore = c.nfcore; ob.mmax1 = c.mmax1; ob.igauge = 0;
  ob.radk = c.radk; ob.radk0 = c.radk0; ob.radp = c.radp; ob.tdiag = c.tdiag; ob.xrad = c.xrad; ob.alph = c.alph;
  ob.mval = c.d_mval; ob.orb = c.orb; ob.h0orb = c.h0orb; ob.h1orb = c.h1orb; ob.lfield = c.lfield;
  cudaMemsetAsync(c.lfield, 0, 9 * sizeof(double), st);
  launch_onebody(ob, st);
  dot_re_kernel<<<1, 256, 0, st>>>(c.orb, c.h0orb, c.nfcore * c.nbas, c.d_scalar);
  const size_t nfcg = c.nfcore * c.ngrid;
  fc_g_kernel<<<(unsigned)((nfcg + 255) / 256), 256, 0, st>>>(c.Nr, c.nlat, c.nfcore, c.nfun, c.orbg, c.W, c.pair_of,
                                                              c.pair_cj, c.v2jfc, c.gorbg);
  launch_legendre_gemm(c.b_gorbfc, c.nfcore, c.L1, c.nlat, 2 * c.Nr, false, st);
  dot_re_kernel<<<1, 256, 0, st>>>(c.orb, c.gorb, c.nfcore * c.nbas, c.d_scalar + 1);
  double es[2] = {0, 0};
  cudaMemcpyAsync(es, c.d_scalar, 2 * sizeof(double), cudaMemcpyDeviceToHost, st);
  cudaStreamSynchronize(st);
  c.ene_fcore = 2.0 * es[0] + es[1];
  cudaMemsetAsync(c.gorbg, 0, c.nfcore * c.ngrid * sizeof(cplx), st);  // scratch of the energy only
  // hprod_addfc_tmat: add v2jfc to the kinetic diagonal; the one-body
  // propagator factors of the old T are stale
  tdiag_kernel<<<(c.Nr * c.L1 + 255) / 256, 256, 0, st>>>(c.Nr, c.L1, c.nd, c.znuc, c.xrad, c.radk, c.radk0, c.v2jfc, c.tdiag);
  for (int i = 0; i < c.n_h1; ++i) c.h1slot[i].cre = c.h1slot[i].cim = std::nan("");
  cudaStreamSynchronize(st);
  if (cudaGetLastError() != cudaSuccess) c.status |= ST_CUDA;
}

void hprod_htot_(const double* dtime, const double* lfield, const double* wfn, const double* cic, double* hwfn, double* hcic) {
  Ctx& c = ctx();
  if (!c.initialized) { c.status |= ST_CONFIG; return; }
  cudaStream_t st = c.st;
  const size_t so = c.nbas * c.nfun;
  cudaMemcpyAsync(c.lfield, lfield, 9 * sizeof(double), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(c.wfn_io, wfn, so * sizeof(cplx), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(c.cic_io, cic, c.lcic * sizeof(cplx), cudaMemcpyHostToDevice, st);
  int rc = run_htot(c, c.lfield, c.wfn_io, c.cic_io, c.hwfn_io, c.hcic_io, *dtime);
  // the reference stops on a failed solve (hprod_mkv2mf.F90:167-170); here a
  // non-finite output (a NaN in the input, a diverged state) is reported in
  // the status word instead
  check_finite(c, c.hwfn_io, 2 * so, st);
  check_finite(c, c.hcic_io, 2 * (size_t)c.lcic, st);
  check_finite(c, c.ene, 5, st);
  cudaMemcpyAsync(hwfn, c.hwfn_io, so * sizeof(cplx), cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(hcic, c.hcic_io, c.lcic * sizeof(cplx), cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(c.h_ene, c.ene, 5 * sizeof(double), cudaMemcpyDeviceToHost, st);
  int dst = 0;
  cudaMemcpyAsync(&dst, c.d_status, sizeof(int), cudaMemcpyDeviceToHost, st);
  cudaError_t e = cudaStreamSynchronize(st);
  if (rc || e != cudaSuccess) c.status |= ST_CUDA;
  c.status |= dst;
  if (c.p_ene_fcore) *c.p_ene_fcore = c.h_ene[0];
  if (c.p_ene_dcore) *c.p_ene_dcore = c.h_ene[1];
  if (c.p_ene_core) *c.p_ene_core = c.h_ene[2];
  if (c.p_ene_act) *c.p_ene_act = c.h_ene[3];
  if (c.p_ene_tot) *c.p_ene_tot = c.h_ene[4];
}

void hprod_final_(void) {
  if (!g) return;
  Ctx& c = *g;
  for (auto& ge : c.graph_exec) if (ge) { cudaGraphExecDestroy(ge); ge = nullptr; }
  for (auto& ge : c.lp_exec) if (ge) { cudaGraphExecDestroy(ge); ge = nullptr; }
  if (c.st) cudaStreamSynchronize(c.st);
  if (c.st2) cudaStreamSynchronize(c.st2);
  if (c.st3) cudaStreamSynchronize(c.st3);
  for (cudaEvent_t e : {c.ev_fork, c.ev_join, c.ev_ob_fork, c.ev_ob_join, c.ev_i2_fork, c.ev_i2_join, c.ev_sig_fork,
                        c.ev_sig_join})
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t& e : c.ev) if (e) { cudaEventDestroy(e); e = nullptr; }
  for (void* p : c.allocs) cudaFree(p);
  c.allocs.clear();
  if (c.own_streams)
    for (cudaStream_t q : {c.st, c.st2, c.st3, c.st4}) if (q) cudaStreamDestroy(q);
  delete g;
  g = nullptr;
  g_ctxs[g_cur] = nullptr;
}

int td1c_gpu_last_status(void) { return g ? g->status : 0; }

int td1c_gpu_dims(int* d) {
  Ctx& c = ctx();
  int v[16] = {c.nrad, (int)c.nbas, (int)c.nbas2, (int)c.ngrid, c.nlat, c.lcic, c.nfcore, c.ndcore, c.nact, c.ncore,
               c.nstr_a, c.nstr_b, c.npair, c.nd, c.lmax1, c.lmax2};
  memcpy(d, v, sizeof(v));
  return 0;
}

int td1c_gpu_ci_tables(unsigned* stra, unsigned* strb, int* detoff, int* afirst, int* acount) {
  Ctx& c = ctx();
  if (stra) std::copy(c.h_stra.begin(), c.h_stra.end(), stra);
  if (strb) std::copy(c.h_strb.begin(), c.h_strb.end(), strb);
  if (detoff) std::copy(c.h_detoff.begin(), c.h_detoff.end(), detoff);
  if (afirst) std::copy(c.h_afirst.begin(), c.h_afirst.end(), afirst);
  if (acount) std::copy(c.h_acount.begin(), c.h_acount.end(), acount);
  return 0;
}

int td1c_gpu_energies(double* e) {
  Ctx& c = ctx();
  if (c.st) cudaStreamSynchronize(c.st);
  cudaMemcpy(c.h_ene, c.ene, 5 * sizeof(double), cudaMemcpyDeviceToHost);
  memcpy(e, c.h_ene, sizeof(c.h_ene));
  return 0;
}

int td1c_gpu_htot_dev(double dtime, const double* lfield, const void* d_wfn, const void* d_cic, void* d_hwfn, void* d_hcic) {
  Ctx& c = ctx();
  if (!c.initialized) return ST_CONFIG;
  cudaMemcpyAsync(c.lfield, lfield, 9 * sizeof(double), cudaMemcpyHostToDevice, c.st);
  int rc = run_htot(c, c.lfield, (const cplx*)d_wfn, (const cplx*)d_cic, (cplx*)d_hwfn, (cplx*)d_hcic, dtime);
  return rc ? ST_CUDA : 0;
}

// length-form dipole <z> of a device-resident state (hprod_dipole.F90, dip(1));
// uses the context's 1-RDM buffers and its stream, synchronous
static void dipole_entries(Ctx& c) {
  if (!c.dip_ent) {
    std::vector<int2> ent;
    for (int f = 0; f < c.ncore; ++f) ent.push_back(make_int2(f, f));
    for (int ia = 0; ia < c.nact; ++ia)
      for (int ja = 0; ja < c.nact; ++ja)
        if (c.mval[c.ncore + ia] == c.mval[c.ncore + ja]) ent.push_back(make_int2(c.ncore + ia, c.ncore + ja));
    c.dip_nent = (int)ent.size();
    c.dip_ent = dupload(ent);
    c.dip_partial = dalloc<cplx>((size_t)std::max(1, dipole_partial_size(c.Nr, c.dip_nent)));
  }
}

int td1c_gpu_dipole(const void* d_wfn, const void* d_cic, double* out) {
  Ctx& c = ctx();
  if (!c.initialized || !out) return ST_CONFIG;
  cudaStream_t st = c.st;
  dipole_entries(c);
  int rc = 0;
  if (c.nact > 0) {
    CiArgs ca{};
    ca.t = c.cit; ca.cic = (const cplx*)d_cic; ca.Da = c.Da; ca.Db = c.Db; ca.T = c.T; ca.den1 = c.den1; ca.den2 = c.den2;
    rc |= chk("ci dvec", launch_ci_dvec(ca, c.maxsec, st));
    rc |= chk("ci rdm", launch_ci_rdm(ca, st));
  }
  DipoleArgs da{};
  da.Nr = c.Nr; da.L1 = c.L1; da.mmax1 = c.mmax1; da.ncore = c.ncore; da.nact = c.nact; da.nent = c.dip_nent;
  da.xrad = c.xrad; da.alph = c.alph; da.mval = c.d_mval; da.ent = c.dip_ent; da.wfn = (const cplx*)d_wfn;
  da.den1 = c.den1; da.partial = c.dip_partial; da.out = c.d_scalar + 2;
  rc |= chk("dipole", launch_dipole(da, st));
  cudaMemcpyAsync(out, c.d_scalar + 2, sizeof(double), cudaMemcpyDeviceToHost, st);
  cudaError_t e = cudaStreamSynchronize(st);
  return (rc || e != cudaSuccess) ? ST_CUDA : 0;
}

// the index maps of the frozen-core dipole's overlaps (rowdot entries):
// buffers 0 orb, 1 z phi, 2 p_z phi, 3 generalized-Fock vectors
static void dipole_fc_entries(Ctx& c) {
  if (c.dip_rd_ent) return;
  const int nf = c.nfun, nfc = c.nfcore;
  std::vector<int4> ent;
  auto add = [&](int ba, int ra, int bb, int rb) { ent.push_back(make_int4(ba, ra, bb, rb)); return (int)ent.size() - 1; };
  c.dip_ia.assign(nfc, -1); c.dip_ib.assign(nfc, -1);
  c.dip_if.assign((size_t)nfc * nf, -1); c.dip_isz.assign((size_t)nf * nfc, -1); c.dip_isp.assign((size_t)nf * nfc, -1);
  for (int f = 0; f < nfc; ++f) { c.dip_ia[f] = add(1, f, 3, f); c.dip_ib[f] = add(2, f, 3, f); }
  for (int j = 0; j < nfc; ++j)
    for (int b = 0; b < nf; ++b)
      if (c.mval[b] == c.mval[j]) c.dip_if[(size_t)j * nf + b] = add(0, j, 3, b);
  for (int a = 0; a < nf; ++a)
    for (int j = 0; j < nfc; ++j)
      if (c.mval[a] == c.mval[j]) {
        c.dip_isz[(size_t)a * nfc + j] = add(1, a, 0, j);
        c.dip_isp[(size_t)a * nfc + j] = add(2, a, 0, j);
      }
  c.dip_rd_n = (int)ent.size();
  c.dip_rd_ent = dupload(ent);
  c.dip_rd = dalloc<cplx>(ent.size());
  const size_t so = c.nbas * c.nfun;
  c.dip_z = dalloc<cplx>(so); c.dip_p = dalloc<cplx>(so); c.dip_g = dalloc<cplx>(so);
  if (!c.dip_lfd) c.dip_lfd = dalloc<double>(9);
}

// hprod_dipole (hprod_dipole.F90:2-146; no pseudopotential, do_op1tr off):
// the length, velocity and acceleration forms as 1-RDM traces of z, p_z (the
// one-body kernel's velocity coupling at unit field) and the acceleration
// operator, plus A_z N (velocity gauge) and -E_z N.  With frozen-core
// orbitals the velocity and acceleration forms add the generalized-Fock
// corrections: the generalized-Fock vectors g (hprod_gfock: the RHS's
// orbital phase, one-body and mean-field passes, then the mean field on the
// frozen-core rows), and
//   vel(2) = -4 Im sum_{f < nfcore} <z phi_f|g_f> - 2 Im trace1(z phi, P_fc g),
//   acc(2) the same with p_z phi,
// P_fc g_b = sum_{j < nfcore, m_j = m_b} phi_j <phi_j|g_b> (hprod_projfc).
// The overlaps are reduced on the device; their few scalars are combined here.
// out = dip(1:3), vel(1:3), acc(1:3).
int td1c_gpu_dipole3(const void* d_wfn, const void* d_cic, const double* lfield, double* out) {
  Ctx& c = ctx();
  if (!c.initialized || !out || !lfield) return ST_CONFIG;
  cudaStream_t st = c.st;
  dipole_entries(c);
  int rc = 0;
  if (!c.dip_lf) {
    const double unit[9] = {0, 0, 1, 0, 0, 0, 0, 0, 0};  // lfield(3,1) = 1: the operator at unit field
    c.dip_lf = dupload(std::vector<double>(unit, unit + 9));
    c.dip_out = dalloc<double>(3);
  }
  const bool fc = c.nfcore > 0;
  const cplx* w = (const cplx*)d_wfn;
  if (fc) {
    // generalized-Fock vectors: the RHS passes leave the orbitals (frozen cores with their gauge
    // phase), den1, every pair potential and the dynamic rows' g and v2 in place
    dipole_fc_entries(c);
    cudaMemcpyAsync(c.dip_lfd, lfield, 9 * sizeof(double), cudaMemcpyHostToDevice, st);
    rc |= run_htot(c, c.dip_lfd, (const cplx*)d_wfn, (const cplx*)d_cic, c.hwfn_io, c.hcic_io, 1.0);
    if (c.neltot >= 2) {
      const size_t nfcg = c.nfcore * c.ngrid;
      fc_gfock_kernel<<<(unsigned)((nfcg + 255) / 256), 256, 0, st>>>(c.Nr, c.nlat, c.nfcore, c.ncore, c.nact, c.nfun, c.d_mval,
                                                                      c.orbg, c.W, c.pair_of, c.pair_cj, c.den1, c.gorbg);
      rc |= chk("fc gorb gemm", gemm(c, c.b_gorbfc, c.nfcore, c.L1, c.nlat, false));
    }
    w = c.orb;
  } else if (c.nact > 0) {
    CiArgs ca{};
    ca.t = c.cit; ca.cic = (const cplx*)d_cic; ca.Da = c.Da; ca.Db = c.Db; ca.T = c.T; ca.den1 = c.den1; ca.den2 = c.den2;
    rc |= chk("ci dvec", launch_ci_dvec(ca, c.maxsec, st));
    rc |= chk("ci rdm", launch_ci_rdm(ca, st));
  }
  // p_z phi: the velocity coupling of the one-body kernel (igauge 1, unit field); z phi (igauge 0)
  OneBodyArgs ob{};
  ob.Nr = c.Nr; ob.L1 = c.L1; ob.nd = c.nd; ob.nfun = c.nfun; ob.nfcore = 0; ob.mmax1 = c.mmax1; ob.igauge = 1;
  ob.radk = c.radk; ob.radk0 = c.radk0; ob.radp = c.radp; ob.tdiag = c.tdiag; ob.xrad = c.xrad; ob.alph = c.alph;
  ob.mval = c.d_mval; ob.orb = w; ob.h0orb = fc ? c.dip_g : c.h0orb; ob.h1orb = fc ? c.dip_p : c.h1orb; ob.lfield = c.dip_lf;
  rc |= chk("onebody", launch_onebody(ob, st));
  const cplx* po = fc ? c.dip_p : c.h1orb;
  if (fc) {
    ob.igauge = 0; ob.h1orb = c.dip_z;
    rc |= chk("onebody", launch_onebody(ob, st));
    const size_t so = c.nbas * c.nfun;
    const double ef = c.igauge == 1 ? lfield[5] : 0.0;
    gfock_sum_kernel<<<(unsigned)((so + 255) / 256), 256, 0, st>>>(so, c.nfcore * c.nbas, ef, c.gorb, c.v2orb, c.h0orb, c.h1orb,
                                                                   c.dip_z, c.dip_g);
    RowDotBufs bufs{{c.orb, c.dip_z, c.dip_p, c.dip_g}};
    rowdot_kernel<<<c.dip_rd_n, 256, 0, st>>>(c.nbas, bufs, c.dip_rd_ent, c.dip_rd);
    rc |= chk("gfock overlaps", (int)cudaGetLastError());
  }
  DipoleArgs da{};
  da.Nr = c.Nr; da.L1 = c.L1; da.mmax1 = c.mmax1; da.ncore = c.ncore; da.nact = c.nact; da.nent = c.dip_nent;
  da.xrad = c.xrad; da.alph = c.alph; da.mval = c.d_mval; da.ent = c.dip_ent; da.wfn = w;
  da.den1 = c.den1; da.partial = c.dip_partial; da.znuc = c.znuc;
  for (int k = 0; k < 3; ++k) {  // z, p_z, acceleration
    da.mode = k == 0 ? 0 : (k == 1 ? 2 : 1);
    da.pv = k == 1 ? po : nullptr;
    da.out = c.dip_out + k;
    rc |= chk("dipole", launch_dipole(da, st));
  }
  double tr[3];
  std::vector<std::complex<double>> rd(fc ? c.dip_rd_n : 0), den1(fc ? (size_t)c.nact * c.nact : 0);
  cudaMemcpyAsync(tr, c.dip_out, 3 * sizeof(double), cudaMemcpyDeviceToHost, st);
  if (fc) {
    cudaMemcpyAsync(rd.data(), c.dip_rd, rd.size() * sizeof(cplx), cudaMemcpyDeviceToHost, st);
    if (!den1.empty()) cudaMemcpyAsync(den1.data(), c.den1, den1.size() * sizeof(cplx), cudaMemcpyDeviceToHost, st);
  }
  cudaError_t e = cudaStreamSynchronize(st);
  if (rc || e != cudaSuccess) return ST_CUDA;
  const double v = tr[1] + (c.igauge == 1 ? lfield[8] * c.neltot : 0.0), a = tr[2] - lfield[5] * c.neltot;
  double vc = 0.0, ac = 0.0;
  if (fc) {
    const int nf = c.nfun, nfc = c.nfcore;
    // <X phi_a | P_fc g_b> = sum_{j < nfcore, m_j = m_b} <X phi_a|phi_j> <phi_j|g_b>
    auto xpg = [&](const std::vector<int>& isx, int a_, int b_) {
      std::complex<double> s = 0.0;
      for (int j = 0; j < nfc; ++j) {
        const int i1 = isx[(size_t)a_ * nfc + j], i2 = c.dip_if[(size_t)j * nf + b_];
        if (i1 >= 0 && i2 >= 0) s += rd[i1] * rd[i2];
      }
      return s;
    };
    auto trace1 = [&](const std::vector<int>& isx) {  // hprod_trace1(.true., den1, X phi, P_fc g)
      std::complex<double> s = 0.0;
      for (int f = 0; f < c.ncore; ++f) s += 2.0 * xpg(isx, f, f);
      for (int ia = 0; ia < c.nact; ++ia)
        for (int ja = 0; ja < c.nact; ++ja)
          if (c.mval[c.ncore + ia] == c.mval[c.ncore + ja]) s += xpg(isx, c.ncore + ia, c.ncore + ja) * den1[ja + c.nact * ia];
      return s;
    };
    std::complex<double> v1 = 0.0, a1 = 0.0;
    for (int f = 0; f < nfc; ++f) { v1 += rd[c.dip_ia[f]]; a1 += rd[c.dip_ib[f]]; }
    vc = -4.0 * v1.imag() - 2.0 * trace1(c.dip_isz).imag();
    ac = -4.0 * a1.imag() - 2.0 * trace1(c.dip_isp).imag();
  }
  const double r[9] = {tr[0], 0.0, tr[0], v, vc, v + vc, a, ac, a + ac};
  for (int k = 0; k < 9; ++k) out[k] = r[k];
  return 0;
}

// hprod_dipole_ (include/wrapper.hpp:114; clhprod::dipole, clhprod.cpp:218-222)
// with host buffers: the state is copied in and dip, vel, acc (3 each) are
// written back; errors go to the status word.
void hprod_dipole_(const double* lfield, const double* wfn, const double* cic, double* dip, double* vel, double* acc) {
  Ctx& c = ctx();
  if (!c.initialized) { c.status |= ST_CONFIG; return; }
  cudaStream_t st = c.st;
  cudaMemcpyAsync(c.wfn_io, wfn, c.nbas * c.nfun * sizeof(cplx), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(c.cic_io, cic, c.lcic * sizeof(cplx), cudaMemcpyHostToDevice, st);
  double out[9];
  const int rc = td1c_gpu_dipole3(c.wfn_io, c.cic_io, lfield, out);
  if (rc) {
    const double nan = std::numeric_limits<double>::quiet_NaN();
    for (int k = 0; k < 9; ++k) out[k] = nan;
  }
  c.status |= rc;
  for (int k = 0; k < 3; ++k) { dip[k] = out[k]; vel[k] = out[3 + k]; acc[k] = out[6 + k]; }
}

// wfn_orth_cic + wfn_orth_orb on a device-resident state (in place)
int td1c_gpu_orth(void* d_wfn, void* d_cic) {
  Ctx& c = ctx();
  if (!c.initialized) return ST_CONFIG;
  int rc = launch_orth(c.Nr, c.L1, c.nfun, c.nfcore, c.lcic, c.d_mval, (cplx*)d_wfn, (cplx*)d_cic, c.st);
  return rc ? ST_CUDA : 0;
}

int td1c_gpu_rk4(void* d_wfn, void* d_cic, double t0, double dt, int nstep, double fint, double wlen, double numcyc,
                 double cep, int use_graph);

// imaginary-time relaxation in the form of init_prop12 (init.cpp:250-319):
// per cycle the total energy of the current state (ene[s], host), one
// zero-field RK4 step of dt (wfn_mask included) and wfn_orth; needs a
// context bound with icomp = 0
int td1c_gpu_relax(void* d_wfn, void* d_cic, double dt, int ncyc, double* ene) {
  Ctx& c = ctx();
  if (!c.initialized || c.icomp != 0 || ncyc < 0) return ST_CONFIG;
  cudaStream_t st = c.st;
  const size_t so = c.nbas * c.nfun;
  if (!c.relax_hw) { c.relax_hw = dalloc<cplx>(so); c.relax_hc = dalloc<cplx>(std::max(1, c.lcic)); }
  double* d_trace = nullptr;
  if (cudaMalloc(&d_trace, sizeof(double) * std::max(1, ncyc)) != cudaSuccess) return ST_CUDA;
  const double lf0[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  cudaMemcpyAsync(c.lfield, lf0, 9 * sizeof(double), cudaMemcpyHostToDevice, st);
  int rc = 0;
  for (int s = 0; s < ncyc && !rc; ++s) {
    rc |= run_htot(c, c.lfield, (const cplx*)d_wfn, (const cplx*)d_cic, c.relax_hw, c.relax_hc, 1.0);
    cudaMemcpyAsync(d_trace + s, c.ene + 4, sizeof(double), cudaMemcpyDeviceToDevice, st);
    rc |= td1c_gpu_rk4(d_wfn, d_cic, 0.0, dt, 1, 0.0, 800.0, 1.0, 0.0, 1);
    rc |= launch_orth(c.Nr, c.L1, c.nfun, c.nfcore, c.lcic, c.d_mval, (cplx*)d_wfn, (cplx*)d_cic, st);
  }
  if (ene && ncyc > 0) cudaMemcpyAsync(ene, d_trace, ncyc * sizeof(double), cudaMemcpyDeviceToHost, st);
  cudaError_t e = cudaStreamSynchronize(st);
  cudaFree(d_trace);
  int dst = 0;
  cudaMemcpy(&dst, c.d_status, sizeof(int), cudaMemcpyDeviceToHost);
  return (rc || e != cudaSuccess) ? ST_CUDA : dst;
}

int td1c_gpu_rk4(void* d_wfn, void* d_cic, double t0, double dt, int nstep, double fint, double wlen, double numcyc,
                 double cep, int use_graph) {
  return prop_run(0, d_wfn, d_cic, t0, dt, nstep, fint, wlen, numcyc, cep, 0, 0.0, use_graph);
}

int td1c_gpu_split2(void* d_wfn, void* d_cic, double t0, double dt, int nstep, double fint, double wlen, double numcyc,
                    double cep, int maxcyc, double thresh, int use_graph) {
  return prop_run(1, d_wfn, d_cic, t0, dt, nstep, fint, wlen, numcyc, cep, maxcyc, thresh, use_graph);
}

int td1c_gpu_etdrk2(void* d_wfn, void* d_cic, double t0, double dt, int nstep, double fint, double wlen, double numcyc,
                    double cep, int maxcyc, double thresh, int use_graph) {
  return prop_run(2, d_wfn, d_cic, t0, dt, nstep, fint, wlen, numcyc, cep, maxcyc, thresh, use_graph);
}

int td1c_gpu_etdrk4(void* d_wfn, void* d_cic, double t0, double dt, int nstep, double fint, double wlen, double numcyc,
                    double cep, int maxcyc, double thresh, int use_graph) {
  return prop_run(3, d_wfn, d_cic, t0, dt, nstep, fint, wlen, numcyc, cep, maxcyc, thresh, use_graph);
}

// one h1itr_prop / dpade_prod on a device-resident state; cycles = correction
// cycles applied
static int h1_call(bool pade, void* d_wfn, const double* lfield, double dtime, cplx alpha, int maxcyc, double thresh,
                   int* cycles) {
  Ctx& c = ctx();
  if (!c.initialized || !d_wfn || !lfield || maxcyc < 0 || !(thresh >= 0.0)) return ST_CONFIG;
  cudaStream_t st = c.st;
  cudaMemcpyAsync(c.lfield, lfield, 9 * sizeof(double), cudaMemcpyHostToDevice, st);
  int rc = h1_apply(c, pade, c.lfield, (cplx*)d_wfn, dtime, alpha, maxcyc, thresh);
  if (rc) return rc;
  int flags[2] = {0, 0}, dst = 0;
  cudaMemcpyAsync(flags, c.h1_flags, 2 * sizeof(int), cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(&dst, c.d_status, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) return ST_CUDA;
  if (cycles) *cycles = flags[1];
  return dst;
}

int td1c_gpu_h1itr(void* d_wfn, const double* lfield, double dtime, int maxcyc, double thresh, int* cycles) {
  return h1_call(false, d_wfn, lfield, dtime, mkc(0, 0), maxcyc, thresh, cycles);
}

int td1c_gpu_dpade(void* d_wfn, const double* lfield, double dtime, double alpha_re, double alpha_im, int maxcyc,
                   double thresh, int* cycles) {
  if (alpha_re == 0.0 && alpha_im == 0.0) return ST_CONFIG;
  return h1_call(true, d_wfn, lfield, dtime, mkc(alpha_re, alpha_im), maxcyc, thresh, cycles);
}

// imaginary-time relaxation in the form of init_prop12 (init.cpp:250-319)
// with H2P = cletdrk2: per cycle the total energy (ene[s], host), one
// zero-field ETD-RK2 step of dt without mask, wfn_orth; icomp = 0
int td1c_gpu_relax_etdrk2(void* d_wfn, void* d_cic, double dt, int ncyc, int maxcyc, double thresh, double* ene) {
  Ctx& c = ctx();
  if (!c.initialized || c.icomp != 0 || ncyc < 0) return ST_CONFIG;
  cudaStream_t st = c.st;
  const size_t so = c.nbas * c.nfun;
  if (!c.relax_hw) { c.relax_hw = dalloc<cplx>(so); c.relax_hc = dalloc<cplx>(std::max(1, c.lcic)); }
  double* d_trace = nullptr;
  if (cudaMalloc(&d_trace, sizeof(double) * std::max(1, ncyc)) != cudaSuccess) return ST_CUDA;
  const double lf0[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  int rc = 0;
  for (int s = 0; s < ncyc && !rc; ++s) {
    cudaMemcpyAsync(c.lfield, lf0, 9 * sizeof(double), cudaMemcpyHostToDevice, st);
    rc |= run_htot(c, c.lfield, (const cplx*)d_wfn, (const cplx*)d_cic, c.relax_hw, c.relax_hc, 1.0);
    cudaMemcpyAsync(d_trace + s, c.ene + 4, sizeof(double), cudaMemcpyDeviceToDevice, st);
    rc |= prop_run(2, d_wfn, d_cic, 0.0, dt, 1, 0.0, 800.0, 1.0, 0.0, maxcyc, thresh, 1, false);
    rc |= launch_orth(c.Nr, c.L1, c.nfun, c.nfcore, c.lcic, c.d_mval, (cplx*)d_wfn, (cplx*)d_cic, st);
  }
  if (ene && ncyc > 0) cudaMemcpyAsync(ene, d_trace, ncyc * sizeof(double), cudaMemcpyDeviceToHost, st);
  cudaError_t e = cudaStreamSynchronize(st);
  cudaFree(d_trace);
  int dst = 0;
  cudaMemcpy(&dst, c.d_status, sizeof(int), cudaMemcpyDeviceToHost);
  return (rc || e != cudaSuccess) ? ST_CUDA : dst;
}

// ---- drop-in one-body propagator entries (host buffers) -------------------
// The factor calls build the condensed factors on the device and write a
// handle into the caller's pivot array (the band array is not touched); the
// product calls check the handle and the bound control flags.
static const int kH1Magic = 0x7D1C0B1;

static int h1_dropin_factor(int icomp, double dtime, cplx alpha, bool pade, int* piv) {
  Ctx& c = ctx();
  if (!c.initialized || icomp != c.icomp || !piv) return ST_CONFIG;
  const bool rt = icomp == 1;
  cplx fac;
  if (pade) {
    const double den = alpha.x * alpha.x + alpha.y * alpha.y;
    if (den == 0.0) return ST_CONFIG;
    const cplx ia = mkc(alpha.x / den, -alpha.y / den);
    fac = rt ? cmul(mkc(0, dtime), ia) : cmul(mkc(dtime, 0), ia);
  } else {
    fac = rt ? mkc(0, dtime * 0.5) : mkc(dtime * 0.5, 0);
  }
  H1Fac F;
  int rc = h1_bufs(c);
  rc |= h1_factor(c, fac, &F);
  if (cudaStreamSynchronize(c.st) != cudaSuccess) rc |= ST_CUDA;
  int dst = 0;
  cudaMemcpy(&dst, c.d_status, sizeof(int), cudaMemcpyDeviceToHost);
  piv[0] = kH1Magic;
  piv[1] = pade ? 1 : 0;
  return rc | dst;
}

static int h1_dropin_prod(bool pade, int isplit, int igauge, int icomp, int iprojfc, const double* lfield, double dtime,
                          cplx alpha, int maxcyc, double thresh, const int* piv, double* wfn) {
  Ctx& c = ctx();
  if (!c.initialized || !piv || piv[0] != kH1Magic || piv[1] != (pade ? 1 : 0)) return ST_CONFIG;
  if (isplit != c.isplit || igauge != c.igauge || icomp != c.icomp || iprojfc != 0) return ST_CONFIG;
  cudaStream_t st = c.st;
  const size_t so = c.nbas * c.nfun;
  cudaMemcpyAsync(c.wfn_io, wfn, so * sizeof(cplx), cudaMemcpyHostToDevice, st);
  int rc = h1_call(pade, c.wfn_io, lfield, dtime, alpha, maxcyc, thresh, nullptr);
  cudaMemcpyAsync(wfn, c.wfn_io, so * sizeof(cplx), cudaMemcpyDeviceToHost, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) rc |= ST_CUDA;
  return rc;
}

void h1itr_gen_cninv_(const int* icomp, const double* dtime, int* cnpiv, double* cninv) {
  (void)cninv;
  Ctx& c = ctx();
  c.status |= h1_dropin_factor(*icomp, *dtime, mkc(0, 0), false, cnpiv);
}

void h1itr_prop_(const int* icomp, const int* isplit, const int* igauge, const int* iprojfc, const double* lfield,
                 const double* dtime, const int* maxcyc, const double* thresh, const int* cnpiv, const double* cninv,
                 double* wfn) {
  (void)cninv;
  Ctx& c = ctx();
  c.status |= h1_dropin_prod(false, *isplit, *igauge, *icomp, *iprojfc, lfield, *dtime, mkc(0, 0), *maxcyc, *thresh,
                             cnpiv, wfn);
}

void dpade_gen_(const int* icomp, const double* dtime, const double* alpha, double* tinv, int* tpiv) {
  (void)tinv;
  Ctx& c = ctx();
  c.status |= h1_dropin_factor(*icomp, *dtime, mkc(alpha[0], alpha[1]), true, tpiv);
}

void dpade_prod_(const int* isplit, const int* igauge, const int* icomp, const int* iprojfc, const double* lfield,
                 const double* dtime, const double* alpha, const int* maxcyc, const double* thresh, const int* tpiv,
                 const double* tinv, double* wfn) {
  (void)tinv;
  Ctx& c = ctx();
  c.status |= h1_dropin_prod(true, *isplit, *igauge, *icomp, *iprojfc, lfield, *dtime, mkc(alpha[0], alpha[1]), *maxcyc,
                             *thresh, tpiv, wfn);
}

long td1c_gpu_launch_count(void) { return g ? g->launches : 0; }

int td1c_gpu_rk4_reset(const void* d_wfn0, const void* d_cic0) {
  ctx().rk.reset_orb = (const cplx*)d_wfn0;
  ctx().rk.reset_cic = (const cplx*)d_cic0;
  return 0;
}

void* td1c_gpu_stream(void) { return g ? (void*)g->st : nullptr; }

// the mixed-precision form of the RHS: on = 1 runs the mean field's pair-density
// multipoles and pair potentials on the grid (the two theta <-> l transforms of
// the pair fields) in split TF32 on the tensor cores, FP32 accumulation, FP64
// everywhere else; on = 0 restores the plain FP64 path.  Captured step graphs
// are recaptured on their next use.
int td1c_gpu_set_mixed(int on) {
  Ctx& c = ctx();
  if (!c.initialized) return ST_CONFIG;
  if (on < 0 || on > 3) return ST_CONFIG;
  c.mixed = on;
  if (c.mixed) build_tc_plans(c);
  return 0;
}

// the deviation of the mixed-precision form from FP64 on one RHS of a device
// state: out[0] = max |d rho2| / max |rho2| (pair-density multipoles),
// out[1] = the same for the pair potentials on the grid W, out[2] for hwfn.
// Runs the RHS twice (lfield: host lfield(3,3)); the mode is restored.
int td1c_gpu_mixed_selftest(const void* d_wfn, const void* d_cic, const double* lfield, double* out) {
  Ctx& c = ctx();
  if (!c.initialized || !out || !lfield) return ST_CONFIG;
  cudaStream_t st = c.st;
  if (!c.dip_lfd) c.dip_lfd = dalloc<double>(9);
  cudaMemcpyAsync(c.dip_lfd, lfield, 9 * sizeof(double), cudaMemcpyHostToDevice, st);
  const size_t nr = c.nbas2 * c.npair, nw = c.ngrid * c.npair, nh = c.nbas * c.nfun;
  std::vector<std::complex<double>> r[2], w[2], h[2];
  const int keep = c.mixed;
  build_tc_plans(c);
  int rc = 0;
  for (int mode = 0; mode < 2; ++mode) {
    c.mixed = mode ? std::max(keep, 1) : 0;
    rc |= run_htot(c, c.dip_lfd, (const cplx*)d_wfn, (const cplx*)d_cic, c.hwfn_io, c.hcic_io, 1.0);
    r[mode].resize(nr); w[mode].resize(nw); h[mode].resize(nh);
    cudaMemcpyAsync(r[mode].data(), c.rho2, nr * sizeof(cplx), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(w[mode].data(), c.W, nw * sizeof(cplx), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(h[mode].data(), c.hwfn_io, nh * sizeof(cplx), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) rc |= ST_CUDA;
  }
  c.mixed = keep;
  if (rc) return ST_CUDA;
  int dst = 0;
  cudaMemcpy(&dst, c.d_status, sizeof(int), cudaMemcpyDeviceToHost);
  c.status |= dst;
  if (dst & ST_TIMEOUT) return ST_TIMEOUT;
  auto rel = [](const std::vector<std::complex<double>>& a, const std::vector<std::complex<double>>& b) {
    double d = 0.0, m = 0.0;
    for (size_t k = 0; k < a.size(); ++k) { d = std::max(d, std::abs(b[k] - a[k])); m = std::max(m, std::abs(a[k])); }
    return m > 0.0 ? d / m : d;
  };
  out[0] = rel(r[0], r[1]); out[1] = rel(w[0], w[1]); out[2] = rel(h[0], h[1]);
  return 0;
}

int td1c_gpu_mixed_int2e_selftest(const void* d_wfn, const void* d_cic, const double* lfield, double* out2) {
  Ctx& c = ctx();
  if (!c.initialized || !out2 || !lfield) return ST_CONFIG;
  out2[0] = out2[1] = -1.0;
  if (!c.i2_tc || c.nact == 0) return ST_CONFIG;
  cudaStream_t st = c.st;
  if (!c.dip_lfd) c.dip_lfd = dalloc<double>(9);
  cudaMemcpyAsync(c.dip_lfd, lfield, 9 * sizeof(double), cudaMemcpyHostToDevice, st);
  const size_t n4 = (size_t)c.nact * c.nact * c.nact * c.nact;
  std::vector<std::complex<double>> i2[3];
  const int keep = c.mixed;
  build_tc_plans(c);
  int rc = 0;
  for (int k = 0; k < 3; ++k) {
    if (k < 2) {
      c.mixed = k ? 3 : 0;
      rc |= run_htot(c, c.dip_lfd, (const cplx*)d_wfn, (const cplx*)d_cic, c.hwfn_io, c.hcic_io, 1.0);
    } else {
      // the FP64 DMMA kernel on the mixed RHS's own pair densities and potentials
      rc |= launch_int2e_dmma(c.i2d, c.i2, i2_split(c), st);
    }
    i2[k].resize(n4);
    cudaMemcpyAsync(i2[k].data(), c.int2e, n4 * sizeof(cplx), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) rc |= ST_CUDA;
  }
  c.mixed = keep;
  if (rc) return ST_CUDA;
  int dst = 0;
  cudaMemcpy(&dst, c.d_status, sizeof(int), cudaMemcpyDeviceToHost);
  c.status |= dst;
  if (dst & ST_TIMEOUT) return ST_TIMEOUT;
  auto rel = [](const std::vector<std::complex<double>>& a, const std::vector<std::complex<double>>& b) {
    double d = 0.0, m = 0.0;
    for (size_t k = 0; k < a.size(); ++k) { d = std::max(d, std::abs(b[k] - a[k])); m = std::max(m, std::abs(a[k])); }
    return m > 0.0 ? d / m : d;
  };
  out2[0] = rel(i2[2], i2[1]);  // tensor-core kernel against DMMA on the same inputs
  out2[1] = rel(i2[0], i2[1]);  // mixed RHS against the FP64 RHS
  return 0;
}

int td1c_gpu_profile(int reps, double dtime, const double* lfield, const void* d_wfn, const void* d_cic, void* d_hwfn,
                     void* d_hcic, double* ms, char* names, int names_cap) {
  Ctx& c = ctx();
  if (!c.initialized) return ST_CONFIG;
  for (int i = 0; i < 16; ++i) if (!c.ev[i]) cudaEventCreate(&c.ev[i]);
  cudaMemcpyAsync(c.lfield, lfield, 9 * sizeof(double), cudaMemcpyHostToDevice, c.st);
  std::vector<double> acc(kNumPhases, 0.0);
  c.profile = true;
  int rc = 0;
  for (int r = 0; r < reps; ++r) {
    rc |= run_htot(c, c.lfield, (const cplx*)d_wfn, (const cplx*)d_cic, (cplx*)d_hwfn, (cplx*)d_hcic, dtime);
    cudaStreamSynchronize(c.st);
    for (int k = 0; k + 1 < c.nev && k < kNumPhases; ++k) {
      float t = 0;
      cudaError_t e = cudaEventElapsedTime(&t, c.ev[k], c.ev[k + 1]);
      if (e != cudaSuccess) {
        fprintf(stderr, "td1c_b200: phase timing %d failed: %s (nev %d)\n", k, cudaGetErrorString(e), c.nev);
        rc |= ST_CUDA;
      }
      acc[k] += t;
    }
  }
  c.profile = false;
  for (int k = 0; k < kNumPhases; ++k) ms[k] = acc[k] / std::max(reps, 1);
  if (names) {
    std::string all;
    for (int k = 0; k < kNumPhases; ++k) { all += kPhaseNames[k]; all += (k + 1 < kNumPhases) ? "," : ""; }
    strncpy(names, all.c_str(), names_cap - 1);
    names[names_cap - 1] = 0;
  }
  return rc ? -ST_CUDA : kNumPhases;
}

int td1c_gpu_set_learned(int depth, const int* sizes, const float* const* W, const float* const* b, void* pack, int use_net,
                         double bound) {
  Ctx& c = ctx();
  if (!c.initialized || bound < 0.0) return ST_CONFIG;
  int rc = lp_setup(c);
  if (rc) return rc;
  c.lp_bound = bound;
  c.lp_use_net = use_net ? 1 : 0;
  c.lp_key_y = nullptr;
  if (depth <= 0) { c.lp_has_net = false; return 0; }
  if (depth > MLP_MAXDEPTH || !sizes || !W || !b || !pack || sizes[0] != 32 || sizes[depth] != 8) return ST_CONFIG;
  MlpInferArgs& a = c.lp_mi;
  a = MlpInferArgs{};
  a.depth = depth; a.rows = c.lp.nu; a.nin = sizes[0]; a.x = c.lp.feat; a.ldx = 32; a.y = c.lp_out; a.ldy = 8;
  a.status = c.lp_mi_status;
  unsigned short* p = (unsigned short*)pack;
  for (int k = 0; k < depth; ++k) {
    if (sizes[k + 1] < 1 || sizes[k + 1] > 256) return ST_CONFIG;
    const int np = (sizes[k + 1] + 15) / 16 * 16, kp = (sizes[k] + 15) / 16 * 16;
    a.n[k] = sizes[k + 1]; a.np[k] = np; a.kp[k] = kp; a.b[k] = b[k]; a.wbf16[k] = p;
    p += (long)np * kp;
  }
  c.lp_has_net = true;
  for (auto& ge : c.lp_exec) if (ge) { cudaGraphExecDestroy(ge); ge = nullptr; }
  c.lp_key_y = nullptr;  // the next call starts afresh
  return 0;
}

int td1c_gpu_set_learned_policy(int screen) {
  Ctx& c = ctx();
  c.lp_screen = screen ? 1 : 0;
  c.lp_key_y = nullptr;
  return 0;
}

int td1c_gpu_split2_learned(void* d_wfn, void* d_cic, double t0, double dt, int nstep, double fint, double wlen, double numcyc,
                            double cep, int maxcyc, double thresh, double* stats) {
  return learned_run(d_wfn, d_cic, t0, dt, nstep, fint, wlen, numcyc, cep, maxcyc, thresh, nullptr, stats);
}

int td1c_gpu_learned_record(void* d_wfn, void* d_cic, double t0, double dt, int nstep, double fint, double wlen, double numcyc,
                            double cep, int maxcyc, double thresh, double* d_record) {
  if (!d_record) return ST_CONFIG;
  return learned_run(d_wfn, d_cic, t0, dt, nstep, fint, wlen, numcyc, cep, maxcyc, thresh, d_record, nullptr);
}

int td1c_gpu_learned_dims(int* out4) {
  Ctx& c = ctx();
  if (!c.initialized || !out4) return ST_CONFIG;
  out4[0] = c.npair * c.nfe; out4[1] = c.nfe; out4[2] = c.npair; out4[3] = LP_REC;
  return 0;
}

// pair kind of each stored pair (0 diagonal, 1 off-diagonal, 2 with the frozen core) as the predictor uses it
int td1c_gpu_learned_pair_kind(int* out) {
  Ctx& c = ctx();
  if (!c.initialized || !out) return ST_CONFIG;
  for (int p = 0; p < c.npair; ++p) out[p] = c.pb[p] < c.nfcore ? 2 : (c.pa[p] == c.pb[p] ? 0 : 1);
  return 0;
}

// ---- contexts of an ensemble and their launch shapes ------------------------
int td1c_gpu_ctx_create(void) {
  int id = -1;
  for (int i = 1; i < (int)g_ctxs.size(); ++i)
    if (!g_ctxs[i]) { id = i; break; }
  if (id < 0) { id = (int)g_ctxs.size(); g_ctxs.push_back(nullptr); }
  g_cur = id;
  g = new Ctx();
  g_ctxs[id] = g;
  return id;
}

int td1c_gpu_ctx_select(int id) {
  if (id < 0 || id >= (int)g_ctxs.size()) return ST_CONFIG;
  g_cur = id;
  g = g_ctxs[id];
  return 0;
}

int td1c_gpu_ctx_current(void) { return g_cur; }

int td1c_gpu_ctx_destroy(int id) {
  if (id <= 0 || id >= (int)g_ctxs.size()) return ST_CONFIG;
  const int keep = g_cur;
  td1c_gpu_ctx_select(id);
  hprod_final_();
  td1c_gpu_ctx_select(keep == id ? 0 : keep);
  return 0;
}

int td1c_gpu_set_tuning(int mt, int mf_cap, int i2_split_) {
  Ctx& c = ctx();
  if ((mt != 0 && mt != 3 && mt != 6) || mf_cap < 0) return ST_CONFIG;
  c.tune_mt = mt; c.tune_mf_cap = mf_cap; c.tune_i2_split = i2_split_;
  for (auto& ge : c.graph_exec) if (ge) { cudaGraphExecDestroy(ge); ge = nullptr; }  // recaptured with the new shapes
  c.lp_key_y = nullptr;  // and so are the learned form's steps
  return 0;
}

int td1c_gpu_get_tuning(int* out4) {
  Ctx& c = ctx();
  if (!out4) return ST_CONFIG;
  out4[0] = c.tune_mt; out4[1] = c.tune_mf_cap; out4[2] = c.tune_i2_split; out4[3] = c.i2_nsplit;
  return 0;
}

// nstep split2 steps of every job of an ensemble in one CUDA graph per step:
// the step of job j is captured on job j's own streams, forked from one
// stream and joined back, so the jobs' kernels have no order between them and
// the GPU runs them side by side.  *ms = device time of the nstep replays.
int td1c_gpu_ensemble_split2(int njob, const int* ids, void* const* d_wfn, void* const* d_cic, const double* t0,
                             const double* dt, int nstep, const double* fint, const double* wlen, const double* numcyc,
                             const double* cep, int maxcyc, double thresh, double* ms) {
  if (njob < 1 || !ids || !d_wfn || !d_cic || !t0 || !dt || !fint || !wlen || !numcyc || !cep || nstep < 0 || maxcyc < 0)
    return ST_CONFIG;
  const int keep = g_cur;
  static cudaStream_t master = nullptr;
  static std::vector<cudaEvent_t> evs;
  if (!master) make_stream(&master, true);
  while ((int)evs.size() < 2 * njob + 2) {
    cudaEvent_t e;
    cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    evs.push_back(e);
  }
  int rc = 0;
  // per job: the field table, buffers and first-call set-up (outside any capture)
  for (int j = 0; j < njob && !rc; ++j) {
    if (td1c_gpu_ctx_select(ids[j]) || !g || !g->initialized || g->isplit != 1) { rc = ST_CONFIG; break; }
    Ctx& c = *g;
    const size_t no = c.nbas * c.nfun, nc = c.lcic;
    RkBufs& b = c.rk;
    if (b.cap < no + nc) {
      b.y0 = dalloc<cplx>(no + nc); b.yt = dalloc<cplx>(no + nc); b.k = dalloc<cplx>(no + nc); b.k2 = dalloc<cplx>(no + nc);
      if (!b.lf_cur) { b.lf_cur = dalloc<double>(54); b.counter = dalloc<int>(2); }
      b.cap = no + nc;
    }
    b.reset_orb = nullptr; b.reset_cic = nullptr;
    Pulse pl;
    pl.famp = std::sqrt(fint[j] / 3.50944506E+16); pl.freq = 1239.84190 / (wlen[j] * 27.2113845);
    pl.period = 2 * PI / pl.freq; pl.numcyc = numcyc[j]; pl.cep = cep[j] / 180.0 * PI; pl.igauge = c.igauge;
    static const double nodes[6] = {0.0, 0.5, 0.5, 1.0, 0.25, 0.75};
    std::vector<double> tab((size_t)std::max(nstep, 1) * 54);
    for (int s = 0; s < nstep; ++s)
      for (int is = 0; is < 6; ++is) pulse_lfield(pl, t0[j] + dt[j] * s + dt[j] * nodes[is], &tab[(size_t)s * 54 + 9 * is]);
    if ((size_t)c.field_cap < tab.size()) {
      const size_t cap = std::max(tab.size(), (size_t)4096 * 54);
      c.field_tab = dalloc<double>(cap);
      c.field_cap = (long)cap;
    }
    cudaMemcpyAsync(c.field_tab, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice, c.st);
    b.h_counter[0] = 0; b.h_counter[1] = nstep;
    cudaMemcpyAsync(b.counter, b.h_counter, 2 * sizeof(int), cudaMemcpyHostToDevice, c.st);
    // warm-up on a copy of the state: the one-body factors, scratch and kernel attributes
    cudaMemcpyAsync(b.yt, d_wfn[j], no * sizeof(cplx), cudaMemcpyDeviceToDevice, c.st);
    cudaMemcpyAsync(b.yt + no, d_cic[j], nc * sizeof(cplx), cudaMemcpyDeviceToDevice, c.st);
    cudaMemcpyAsync(c.lfield, tab.data(), 9 * sizeof(double), cudaMemcpyHostToDevice, c.st);
    rc |= h1_apply(c, false, c.lfield, b.yt, 0.5 * dt[j], mkc(0, 0), maxcyc, thresh);
    rc |= run_htot(c, c.lfield, b.yt, b.yt + no, b.k, b.k + no, 1.0);
    if (cudaStreamSynchronize(c.st) != cudaSuccess) rc |= ST_CUDA;
  }
  cudaGraphExec_t exec = nullptr;
  if (!rc && nstep > 0) {
    cudaGraph_t graph = nullptr;
    if (cudaStreamBeginCapture(master, cudaStreamCaptureModeThreadLocal) != cudaSuccess) rc = ST_CUDA;
    for (int j = 0; j < njob && !rc; ++j) {
      td1c_gpu_ctx_select(ids[j]);
      Ctx& c = *g;
      cudaEventRecord(evs[2 * j], master);
      cudaStreamWaitEvent(c.st, evs[2 * j], 0);
      rc |= split2_step(c, (cplx*)d_wfn[j], (cplx*)d_cic[j], dt[j], maxcyc, thresh, true);
      cudaEventRecord(evs[2 * j + 1], c.st);
      cudaStreamWaitEvent(master, evs[2 * j + 1], 0);
    }
    if (cudaStreamEndCapture(master, &graph) != cudaSuccess) rc |= ST_CUDA;
    if (!rc && cudaGraphInstantiate(&exec, graph, cudaGraphInstantiateFlagUseNodePriority) != cudaSuccess) rc |= ST_CUDA;
    if (graph) cudaGraphDestroy(graph);
  }
  if (!rc && exec) {
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, master);
    for (int s = 0; s < nstep && !rc; ++s)
      if (cudaGraphLaunch(exec, master) != cudaSuccess) rc |= ST_CUDA;
    cudaEventRecord(e1, master);
    if (cudaEventSynchronize(e1) != cudaSuccess) rc |= ST_CUDA;
    float t = 0;
    cudaEventElapsedTime(&t, e0, e1);
    if (ms) *ms = t;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }
  if (exec) cudaGraphExecDestroy(exec);
  for (int j = 0; j < njob; ++j) {
    td1c_gpu_ctx_select(ids[j]);
    if (!g) continue;
    Ctx& c = *g;
    const size_t no = c.nbas * c.nfun, nc = c.lcic;
    check_finite(c, d_wfn[j], 2 * no, c.st);
    check_finite(c, d_cic[j], 2 * nc, c.st);
    int dst = 0;
    cudaMemcpyAsync(&dst, c.d_status, sizeof(int), cudaMemcpyDeviceToHost, c.st);
    if (cudaStreamSynchronize(c.st) != cudaSuccess) rc |= ST_CUDA;
    c.status |= dst;
    rc |= dst;
  }
  td1c_gpu_ctx_select(keep);
  return rc;
}

int td1c_gpu_wait_selftest(void) {
  Ctx& c = ctx();
  if (!c.initialized) return ST_CONFIG;
  static int* d_word = nullptr;
  if (!d_word && cudaMalloc(&d_word, sizeof(int)) != cudaSuccess) return ST_CUDA;
  int word = 0;
  cudaMemsetAsync(d_word, 0, sizeof(int), c.st);
  wait_selftest_kernel<<<1, 32, 0, c.st>>>(d_word);
  cudaMemcpyAsync(&word, d_word, sizeof(int), cudaMemcpyDeviceToHost, c.st);
  if (cudaStreamSynchronize(c.st) != cudaSuccess) return ST_CUDA;
  return word;
}

int td1c_gpu_sync(void) {
  Ctx& c = ctx();
  cudaError_t e = cudaStreamSynchronize(c.st);
  return e == cudaSuccess ? 0 : (int)e;
}

// device address of a named buffer of the context (for callers that stage
// their own mean field with td1c_gpu_set_mf_external), or NULL
void* td1c_gpu_debug_ptr(const char* name) {
  Ctx& c = ctx();
  std::string n(name);
  if (n == "W") return c.W;
  if (n == "int2e") return c.int2e;
  if (n == "rho2") return c.rho2;
  if (n == "v2sph") return c.v2sph;
  return nullptr;
}

// copy a named buffer of the context to (to_ctx = 0) or from (to_ctx = 1) the
// device buffer d_other, queued on the library stream; returns the bytes or -1
long td1c_gpu_debug_xfer(const char* name, void* d_other, int to_ctx) {
  Ctx& c = ctx();
  std::string n(name);
  void* p = nullptr;
  size_t bytes = 0;
  if (n == "W") { p = c.W; bytes = c.ngrid * c.npair * sizeof(cplx); }
  else if (n == "int2e") { p = c.int2e; bytes = (size_t)c.nact * c.nact * c.nact * c.nact * sizeof(cplx); }
  else if (n == "rho2") { p = c.rho2; bytes = c.nbas2 * c.npair * sizeof(cplx); }
  else if (n == "v2sph") { p = c.v2sph; bytes = c.nbas2 * c.npair * sizeof(cplx); }
  else return -1;
  if (!d_other || !p) return -1;
  if (cudaMemcpyAsync(to_ctx ? p : d_other, to_ctx ? d_other : p, bytes, cudaMemcpyDeviceToDevice, c.st) != cudaSuccess)
    return -1;
  return (long)bytes;
}

// on = 1: every following RHS skips the pair densities, the Poisson solve, the
// l -> theta transform of the pair potentials and int2e, and uses W and int2e
// as they stand in the context's buffers; 0 restores the full RHS
int td1c_gpu_set_mf_external(int on) {
  Ctx& c = ctx();
  if (!c.initialized) return ST_CONFIG;
  c.mf_external = on ? 1 : 0;
  return 0;
}

// lfield(3,3) of the sin^2 pulse at time t in the bound gauge, as the
// propagators stage it (clfield1 velocity1 / length1)
int td1c_gpu_pulse_lfield(double t, double fint, double wlen, double numcyc, double cep, double* out9) {
  Ctx& c = ctx();
  Pulse p;
  p.famp = std::sqrt(fint / 3.50944506E+16); p.freq = 1239.84190 / (wlen * 27.2113845);
  p.period = 2 * PI / p.freq; p.numcyc = numcyc; p.cep = cep / 180.0 * PI; p.igauge = c.igauge;
  pulse_lfield(p, t, out9);
  return 0;
}

long td1c_gpu_debug_get(const char* name, double* out, long cap) {
  Ctx& c = ctx();
  std::string n(name);
  const void* src = nullptr;
  size_t bytes = 0;
  const size_t so = c.nbas * c.nfun * sizeof(cplx), sg = c.ngrid * c.nfun * sizeof(cplx);
  if (n == "orb") { src = c.orb; bytes = so; }
  else if (n == "orbg") { src = c.orbg; bytes = sg; }
  else if (n == "h0orb") { src = c.h0orb; bytes = so; }
  else if (n == "h1orb") { src = c.h1orb; bytes = so; }
  else if (n == "gorb") { src = c.gorb; bytes = so; }
  else if (n == "v2orb") { src = c.v2orb; bytes = so; }
  else if (n == "gorbg") { src = c.gorbg; bytes = sg; }
  else if (n == "v2orbg") { src = c.v2orbg; bytes = sg; }
  else if (n == "rho2") { src = c.rho2; bytes = c.nbas2 * c.npair * sizeof(cplx); }
  else if (n == "v2sph") { src = c.v2sph; bytes = c.nbas2 * c.npair * sizeof(cplx); }
  else if (n == "W") { src = c.W; bytes = c.ngrid * c.npair * sizeof(cplx); }
  else if (n == "den1") { src = c.den1; bytes = (size_t)c.nact * c.nact * sizeof(cplx); }
  else if (n == "den2") { src = c.den2; bytes = (size_t)c.nact * c.nact * c.nact * c.nact * sizeof(cplx); }
  else if (n == "rden") { src = c.rden; bytes = (size_t)c.nact * c.nact * sizeof(cplx); }
  else if (n == "rrden") { src = c.rrden; bytes = (size_t)c.nact * c.nact * sizeof(cplx); }
  else if (n == "int1e") { src = c.int1e; bytes = (size_t)c.nact * c.nact * sizeof(cplx); }
  else if (n == "int2e") { src = c.int2e; bytes = (size_t)c.nact * c.nact * c.nact * c.nact * sizeof(cplx); }
  else if (n == "xmat") { src = c.xmat; bytes = (size_t)c.nfun * c.nfun * sizeof(cplx); }
  else if (n == "v2jfc") { src = c.v2jfc; bytes = c.Nr * sizeof(double); }
  else if (n == "tdiag") { src = c.tdiag; bytes = (size_t)c.Nr * c.L1 * sizeof(double); }
  else if (n == "d2ll") { src = c.d2ll; bytes = (size_t)c.Nr * c.L2 * (c.nd + 1) * sizeof(double); }
  else return -1;
  long nd = (long)(bytes / sizeof(double));
  if (!out) return nd;
  if (nd > cap) return -2;
  cudaStreamSynchronize(c.st);
  if (bytes) cudaMemcpy(out, src, bytes, cudaMemcpyDeviceToHost);
  return nd;
}

}  // extern "C"
