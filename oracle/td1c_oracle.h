/*
 * td1c_oracle.h -- C API of the CPU oracle.
 *
 * TEST INFRASTRUCTURE ONLY.  The oracle is a plain C++17/OpenMP restatement of
 * the td1c orbital-equation right-hand side (hprod_htot and what it calls) and
 * of the grid/operator-table setup it depends on.  It exists to check the CUDA
 * product path and to serve as the timed CPU baseline.  Nothing in the product
 * (the td1c_b200 package and its shared library) may link, load or call it.
 *
 * Parity status: the reference (Fortran 2018 + MKL + SHTOOLS + GSL) cannot be
 * built in this environment and ships no tests or golden outputs, so this
 * restatement is "parity unpinned" against the reference binary.  It is pinned
 * instead by analytic known-answer checks (hydrogenic spectra, Legendre
 * orthonormality, Poisson of Slater densities, Hermiticity, conservation laws)
 * and by scipy/LAPACK cross-checks of its banded Cholesky and eigen solvers.
 *
 * Every array crossing this API is a flat float64 buffer; complex arrays are
 * interleaved (re, im) and use the reference's Fortran column-major layouts:
 *   wfn/hwfn : orb(1:nrad-1, 0:lmax1, 1:nfun)
 *   cic/hcic : cic(1:lcic)   (determinant order documented in td1c_oracle.cpp)
 *   lfield   : lfield(1:3, 1:3) column-major (gauge field, E, A), z at [2],[5],[8]
 */
#ifndef TD1C_ORACLE_H
#define TD1C_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  double znuc;            /* nuclear charge                                  */
  double rmin, rmax;      /* one uniform FEDVR segment "grid: rmin rmax ndvr nfe" */
  int ndvr;               /* Lobatto points per element minus one            */
  int nfe;                /* number of finite elements                       */
  int lmax1, lmax2, nlat; /* orbital / pair l cut-offs, Gauss-Legendre theta points */
  int nfun;               /* number of orbitals                              */
  const int* otype;       /* per orbital: -1 frozen core, 0 dynamic core, 1 active */
  const int* mval;        /* per orbital magnetic quantum number             */
  const int* lval;        /* per orbital nominal l (used for the frozen-core density) */
  int nela, nelb;         /* total alpha / beta electrons                    */
  int mtot;               /* total M of the CI space                         */
  int smul;               /* spin multiplicity (1 enables the singlet RDM shortcut) */
  int igauge;             /* 0 length gauge, 1 velocity gauge                */
  int icomp;              /* 1 real time, 0 imaginary time                   */
  double rmask;           /* mask radius                                     */
  double mask_cos_order;  /* cos^(1/order) mask                              */
} orc_config;

void* orc_create(const orc_config* cfg);
void  orc_destroy(void* h);
/* dims[0..15]: nrad, nbas, nbas2, ngrid, nlat, lcic, nfcore, ndcore, nact,
 * ncore, nstr_alpha, nstr_beta, ndvr, lmax1, lmax2, nfun                    */
void  orc_dims(void* h, int* dims);
/* Copy a named internal array into out (may be NULL to query the length);
 * returns the number of float64 values, or -1 for an unknown name.         */
long  orc_get(void* h, const char* name, double* out);
/* Frozen-core set-up (hprod_set_wfn0): stores orb0, builds v2jfc, adds it to
 * the kinetic table and computes the frozen-core energy.                   */
void  orc_set_wfn0(void* h, const double* wfn, const double* cic);
/* The RHS: hprod_htot(dtime, lfield, wfn, cic, hwfn, hcic).                 */
void  orc_htot(void* h, double dtime, const double* lfield,
               const double* wfn, const double* cic, double* hwfn, double* hcic);
/* energies[0..4]: ene_fcore, ene_dcore, ene_core, ene_act, ene_tot of the last htot */
void  orc_energies(void* h, double* energies);
/* Standard RK4 (clcrk) + mask over nstep steps with the sin^2 pulse below;
 * wfn/cic are updated in place.  dip[nstep] (may be NULL) receives the
 * length-form dipole <z> after each step.                                   */
typedef struct {
  double fint;    /* peak intensity W/cm^2                          */
  double wlen;    /* wavelength nm                                  */
  double numcyc;  /* cycles of the sin^2 envelope                   */
  double cep;     /* carrier-envelope phase, degrees                */
  int igauge;     /* 0 length1, 1 velocity1                         */
} orc_pulse;
void  orc_field(const orc_pulse* p, double t, double* lfield9);
void  orc_rk4(void* h, const orc_pulse* p, double t0, double dt, int nstep,
              double* wfn, double* cic, double* dip);
/* wfn_orth_cic + wfn_orth_orb (Gram-Schmidt within each m), in place        */
void  orc_orth(void* h, double* wfn, double* cic);
/* Imaginary-time relaxation (init_prop12 form; needs icomp = 0): per cycle
 * ene[s] = total energy of the current state, one zero-field RK4 step of dt,
 * then orc_orth.  wfn/cic are updated in place.                              */
void  orc_relax(void* h, double dt, int ncyc, double* wfn, double* cic, double* ene);
/* split_type (0 full H in the RHS, 1 two-body part only, 2 h0 left out);
 * only hprod_htot_dtorb and the one-body propagators below read it.         */
void  orc_set_split(void* h, int isplit);
/* h1itr_prop: one Crank-Nicolson step over dtime of the one-body part of the
 * non-frozen orbitals (laser coupling by correction cycles when isplit = 1,
 * at most maxcyc, stopping below thresh); returns the corrections added.   */
int   orc_h1itr_prop(void* h, const double* lfield9, double dtime, int maxcyc, double thresh, double* wfn);
/* dpade_prod: non-frozen orbitals <- (1 + c (T + V))^-1 wfn, c = i dtime /
 * alpha (dtime / alpha in imaginary time); returns the corrections added.  */
int   orc_dpade_prod(void* h, const double* lfield9, double dtime, double alpha_re, double alpha_im,
                     int maxcyc, double thresh, double* wfn);
/* tdse_split2 with clh1itr + clcrk: per step h1itr over dt/2, RK4 over dt,
 * h1itr over dt/2, wfn_mask; dip[nstep] as in orc_rk4.                      */
void  orc_split2(void* h, const orc_pulse* p, double t0, double dt, int nstep, int maxcyc, double thresh,
                 double* wfn, double* cic, double* dip);
/* tdse_prop12 with cletdrk2 (+ cldpade, alpha = 2) and wfn_mask per step.   */
void  orc_etdrk2(void* h, const orc_pulse* p, double t0, double dt, int nstep, int maxcyc, double thresh,
                 double* wfn, double* cic, double* dip);
/* tdse_prop12 with cletdrk4 (+ clh1rat, default orders 2/2) and wfn_mask
 * per step; orc_etd4_fun: the coefficients of function `which` (exp1, exp2,
 * gfun, f0, f1, f2): n0..n2, d0[2], d1[2], rk as (re, im) pairs, then dt.  */
void  orc_etdrk4(void* h, const orc_pulse* p, double t0, double dt, int nstep, int maxcyc, double thresh,
                 double* wfn, double* cic, double* dip);
void  orc_etd4_fun(int which, double dt, int icomp, double* out);
/* hprod_dipole: out = dip(1:3), vel(1:3), acc(1:3) (length, velocity,
 * acceleration forms); with frozen-core orbitals vel(2), acc(2) carry the
 * generalized-Fock corrections (hprod_gfock, hprod_projfc). Returns 0.     */
int   orc_dipole3(void* h, const double* wfn, const double* cic, const double* lfield, double* out);
/* init_prop12 with cletdrk2: per cycle ene[s], one zero-field ETD-RK2 step
 * (no mask), orc_orth (needs icomp = 0).                                     */
void  orc_relax_etdrk2(void* h, double dt, int ncyc, int maxcyc, double thresh, double* wfn, double* cic,
                       double* ene);
/* Observable: length-form dipole <z> of the full state (orbitals + CI)      */
double orc_dipole(void* h, const double* wfn, const double* cic);
int   orc_num_threads(void);
/* v2sph of the last RHS for the 'dyn' pairs: out [npair][lmax2 + 1][nrad - 1]
 * complex; returns npair (test data for the learned mean-field predictor).  */
int   orc_v2sph(void* h, double* out);

#ifdef __cplusplus
}
#endif
#endif
