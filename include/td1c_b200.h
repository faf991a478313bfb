/*
 * td1c_b200.h -- C-ABI of the B200 (sm_100a) implementation of td1c's
 * orbital-equation right-hand side.  Plain C types only.
 *
 * Drop-in entry points keep the reference's Fortran-to-C symbol names and
 * argument meaning (include/wrapper.hpp in the td1c tree):
 *   hprod_bind_      include/wrapper.hpp:110   (src/hprod/hprod_bind.F90)
 *   hprod_init_      include/wrapper.hpp:185   (src/hprod/hprod_init.F90:2-103)
 *   hprod_set_wfn0_  include/wrapper.hpp:400   (src/hprod/hprod_set_wfn0.F90:2-130)
 *   hprod_htot_      include/wrapper.hpp:159   (src/hprod/hprod_htot.F90:2-42)
 *   hprod_final_     include/wrapper.hpp:132   (src/hprod/hprod_final.F90)
 * The geometry, tables and flags that the reference hands to Fortran through
 * bas_rad_bind_, bas_sph_bind_, bas_bas_bind_, ormas_bind_ and control_bind_
 * (include/wrapper.hpp:773-806; called from src/bas/clbas.cpp:59-146 and
 * src/control/clcontrol.cpp:185-189) arrive through the td1c_gpu_bind_*
 * calls below, restricted to the fields the RHS reads.  Operator tables the
 * reference derives in bas_gen_* (tmat, pmat, d2ll, zfac, pzfac, d2fac) are
 * derived by the library itself on the device.
 *
 * Complex arrays are interleaved (re, im) float64, Fortran column-major:
 *   wfn, hwfn : orb(1:nrad-1, 0:lmax1, 1:nfun)
 *   cic, hcic : cic(1:lcic), determinants ordered by beta string, then by the
 *               alpha strings of matching M; string lists sorted by (M, mask)
 *   lfield    : lfield(1:3, 1:3) column-major (gauge field, E, A)
 * Errors: the void drop-in calls record a status readable with
 * td1c_gpu_last_status() (0 = ok); the td1c_gpu_* calls return it directly.
 * Status bits: 1 Poisson band factor not positive definite, 2 Jacobi
 * eigensolver not converged, 4 non-finite value in an output (hprod_htot_'s
 * hwfn, hcic and energies; the state at the end of every propagation call),
 * 8 CUDA call failed, 16 unsupported configuration, 32 a bounded device
 * wait ran out, 64 singular one-body factor.  The reference stops the
 * program in these cases (e.g. src/hprod/hprod_mkv2mf.F90:167-170,
 * src/bas/bas_gen_d2ll.F90:120-123).
 */
#ifndef TD1C_B200_H
#define TD1C_B200_H

#include <stddef.h>

#ifdef __cplusplus
#define TD1C_BOOL bool
extern "C" {
#else
#define TD1C_BOOL _Bool
#endif

/* ---- binding of geometry, tables and flags --------------------------- */

/* bas_rad_bind_ (src/bas/bas_bind.F90:2-74): FEDVR radial grid.  Arrays are
 * indexed 0..nrad; band arrays are (2*ndvr+1) x (nrad+1), band index fastest. */
int td1c_gpu_bind_rad(int nfe, int ndvr, int nrad, const double* xrad, const double* wrad,
                      const double* radp, const double* radk, const double* radk0,
                      double rmask, const double* mask);

/* bas_sph_bind_ (src/bas/bas_bind.F90:76-120): Gauss-Legendre theta grid and
 * normalised associated Legendre tables, reference layouts
 * legf1(0:lmax1, 1:nlat, -mmax1:mmax1), legb1(1:nlat, 0:lmax1, -mmax1:mmax1),
 * legf2(0:lmax2, 1:nlat, -mmax2:mmax2), legb2(1:nlat, 0:lmax2, -mmax2:mmax2). */
int td1c_gpu_bind_sph(int lmax1, int lmax2, int mmax1, int mmax2, int nlat,
                      const double* wlat, const double* cost,
                      const double* legf1, const double* legb1,
                      const double* legf2, const double* legb2);

/* bas_bas_bind_ + ormas_bind_ (src/bas/bas_bind.F90:122-194,
 * src/ormas/ormas_bind.F90:1-70): nuclear charge and orbital classes.
 * otype: -1 frozen core (fc1), 0 dynamic core, 1 active; orbitals ordered
 * frozen, dynamic core, active.  lval is the nominal l of each orbital. */
int td1c_gpu_bind_bas(double znuc, int smul, int mtot, int nfun, const int* otype,
                      const int* mval, const int* lval, int nela, int nelb);

/* ormas_bind_'s subspace count nsub (src/ormas/ormas_bind.F90:2-75).  Only
 * CAS (nsub = 1) is supported: other values are recorded and hprod_init_
 * then fails with ST_CONFIG (16), where the reference would run the
 * active-active rotation solve of ormas_xact2 (src/ormas/ormas_xact2.F90:
 * 46,82).  Returns 16 for nsub != 1.  Default 1. */
int td1c_gpu_bind_ormas(int nsub);

/* control_bind_ (src/control/control_bind.F90:2-61): icomp 1 real time,
 * 0 imaginary time; igauge 0 length, 1 velocity. */
int td1c_gpu_bind_control(int icomp, int igauge);
/* split_type of control_bind_ (isplit; src/control/clcontrol.cpp:98): 0 the
 * orbital RHS holds h0 + h1 + g + v2, 2 it leaves out h0, 1 it leaves out h0
 * and the laser coupling h1 (src/hprod/hprod_htot_dtorb.F90:58-84), which the
 * one-body propagators below then apply.  Default 0. */
int td1c_gpu_bind_split(int split_type);

/* ---- drop-in hprod entry points -------------------------------------- */
void hprod_bind_(double* ene_fcore, double* ene_dcore, double* ene_core, double* ene_act,
                 double* ene_tot, double* dip_exp, double* vel_exp, double* acc_exp,
                 const TD1C_BOOL* projhigh, const double* cutoff);
void hprod_init_(void);
void hprod_set_wfn0_(const double* wfn, const double* cic, const char* v2xfc_type, int len);
void hprod_htot_(const double* dtime, const double* lfield, const double* wfn, const double* cic,
                 double* hwfn, double* hcic);
void hprod_final_(void);

/* ---- drop-in one-body propagators (src/prop) --------------------------
 * The reference factors 1 + c T_l (c = i dtime/2, or i dtime/alpha) per l
 * with ZGBTRF into the caller's band array and solves with ZGBTRS.  Here the
 * factor calls build the factors on the device and write a handle into the
 * caller's pivot array (at least 2 ints); the band array is not touched and
 * may be any buffer.  The product calls take host orbitals
 * orb(1:nrad-1, 0:lmax1, 1:nfun) and replace the non-frozen ones.  The flags
 * passed must equal the bound ones (icomp, igauge, split_type) and iprojfc
 * must be 0; violations, a missing handle or a singular factor are recorded
 * in td1c_gpu_last_status().
 *   h1itr_gen_cninv_  include/wrapper.hpp:668 (src/prop/h1itr_gen_cninv.F90:2-63)
 *   h1itr_prop_       include/wrapper.hpp:670 (src/prop/h1itr_prop.F90:2-175):
 *       (1 + i dtime/2 H1)^-1 (1 - i dtime/2 H1), H1 = T + V (split_type 1,
 *       V by correction cycles until their rms norm < thresh, at most maxcyc)
 *   dpade_gen_        include/wrapper.hpp:650 (src/prop/dpade_gen.F90:2-63)
 *   dpade_prod_       include/wrapper.hpp:653 (src/prop/dpade_prod.F90:2-124):
 *       (1 + i dtime/alpha (T + V))^-1, alpha complex (2 doubles) */
void h1itr_gen_cninv_(const int* icomp, const double* dtime, int* cnpiv, double* cninv);
void h1itr_prop_(const int* icomp, const int* isplit, const int* igauge, const int* iprojfc, const double* lfield,
                 const double* dtime, const int* maxcyc, const double* thresh, const int* cnpiv, const double* cninv,
                 double* wfn);
void dpade_gen_(const int* icomp, const double* dtime, const double* alpha, double* tinv, int* tpiv);
void dpade_prod_(const int* isplit, const int* igauge, const int* icomp, const int* iprojfc, const double* lfield,
                 const double* dtime, const double* alpha, const int* maxcyc, const double* thresh, const int* tpiv,
                 const double* tinv, double* wfn);

/* ---- extensions ------------------------------------------------------- */
int td1c_gpu_last_status(void);
/* sizes: [nrad, nbas, nbas2, ngrid, nlat, lcic, nfcore, ndcore, nact, ncore,
 *         nstr_alpha, nstr_beta, npair, ndvr, lmax1, lmax2] */
int td1c_gpu_dims(int* dims16);
/* CI tables (for building CI vectors in the library's determinant order):
 * stra[nstr_a], strb[nstr_b] bit strings; detoff/afirst/acount[nstr_b]. */
int td1c_gpu_ci_tables(unsigned* stra, unsigned* strb, int* detoff, int* afirst, int* acount);
/* energies of the last htot: ene_fcore, ene_dcore, ene_core, ene_act, ene_tot */
int td1c_gpu_energies(double* ene5);
/* RHS on device-resident buffers (no host copies), on the library stream.
 * lfield is a host array of 9 doubles. */
int td1c_gpu_htot_dev(double dtime, const double* lfield, const void* d_wfn, const void* d_cic,
                      void* d_hwfn, void* d_hcic);
/* Copy a named device intermediate of the last htot to host memory
 * (complex arrays as interleaved doubles); returns doubles copied or -1. */
long td1c_gpu_debug_get(const char* name, double* out, long capacity);

/* Device address of a named buffer of the context: "W" (pair potentials on
 * the grid, [pair][nlat][Nr] complex), "int2e" ([nact^4] complex), "rho2",
 * "v2sph" ([pair][lmax2+1][Nr] complex); NULL for other names. */
void* td1c_gpu_debug_ptr(const char* name);
/* Queue a device copy of a named buffer (names as above) to (to_ctx = 0) or
 * from (to_ctx = 1) the device buffer d_other on the library stream; returns
 * the bytes copied or -1. */
long td1c_gpu_debug_xfer(const char* name, void* d_other, int to_ctx);
/* on = 1: every following RHS takes the pair potentials W and int2e as they
 * stand in the context instead of forming them from the stage's orbitals
 * (no pair densities, Poisson solve, l -> theta transform or int2e); the
 * rest of hprod_htot (src/hprod/hprod_htot.F90:44-208) is unchanged.  This
 * is the stage RHS of the learned form, whose predictor writes W and int2e;
 * 0 restores the full RHS. */
int td1c_gpu_set_mf_external(int on);
/* lfield(3,3) (9 doubles, host) of the sin^2 pulse at time t in the bound
 * gauge, as the propagators stage it (clfield1 velocity1 / length1,
 * src/field/clfield1.cpp:253-300,472-500,573-620). */
int td1c_gpu_pulse_lfield(double t, double fint, double wlen, double numcyc, double cep, double* out9);

/* Length-form dipole <z> of a device-resident state, written to *out (host):
 * dip(1) of hprod_dipole (src/hprod/hprod_dipole.F90:2-70), i.e.
 * Re[2 sum_core <phi|z phi> + sum_{ij} <phi_i|z phi_j> den1(j,i)] with z
 * applied as the unit-field length-gauge coupling.  Uses the library stream
 * and its 1-RDM buffers; returns when the value is on the host. */
int td1c_gpu_dipole(const void* d_wfn, const void* d_cic, double* out);
/* hprod_dipole (src/hprod/hprod_dipole.F90:2-146) of a device state:
 * out[9] = dip(1:3), vel(1:3), acc(1:3) (length, velocity and acceleration
 * forms by the Ehrenfest traces hprod_trace1 of z, p_z and the nuclear
 * acceleration operator, plus A_z N in the velocity gauge and -E_z N).
 * Without frozen-core orbitals the second components are 0; with them
 * vel(2), acc(2) are the generalized-Fock corrections (hprod_gfock,
 * src/hprod/hprod_gfock.F90:2-230; hprod_projfc, src/hprod/hprod_projfc.F90)
 * and the call also runs the RHS passes (the library's RHS scratch is
 * overwritten).  lfield: host lfield(3,3). */
int td1c_gpu_dipole3(const void* d_wfn, const void* d_cic, const double* lfield, double* out);
/* The mixed-precision form of the RHS (no counterpart in the reference; the
 * precision variant of hprod_htot, src/hprod/hprod_htot.F90:2-208): on = 1
 * runs the mean field's pair-density multipoles (bas_ang2sph2.F90:330-482)
 * and pair potentials on the grid (bas_sph2ang2.F90:334-463) in split TF32
 * on the tensor cores with FP32 accumulation, FP64 everywhere else; 0 restores
 * the plain FP64 path.  Every later RHS and step uses the mode.  on = 2 is the
 * same arithmetic on the per-tile split-TF32 kernel instead of the persistent
 * one (for comparisons); on = 3 is mode 1 with the Poisson solve's interior
 * products (the pair densities times the element Poisson inverses,
 * hprod_mkv2mf.F90:143-178) and the MO two-electron integrals
 * (hprod_mkint2_sph.F90:2-100) in split TF32 on the tensor cores as well
 * (FP64 int2e where that plan does not apply); other values return 16. */
int td1c_gpu_set_mixed(int on);
/* Deviation of the mixed form from FP64 on one RHS of a device state:
 * out[0..2] = max |delta| / max |FP64 value| of the pair-density multipoles,
 * the pair potentials on the grid and hwfn.  lfield: host lfield(3,3). */
int td1c_gpu_mixed_selftest(const void* d_wfn, const void* d_cic, const double* lfield, double* out);
/* The split-TF32 int2e of mixed mode 3 on one RHS of a device state:
 * out2[0] = max |delta| / max |value| between the tensor-core int2e and the
 * FP64 DMMA int2e on the same (mixed) pair densities and potentials; out2[1]
 * = the same between the mode-3 RHS's int2e and the FP64 RHS's.  16 (and
 * out2 = -1) where the tensor-core plan does not apply (no active orbitals,
 * more than 64 stored active pairs). */
int td1c_gpu_mixed_int2e_selftest(const void* d_wfn, const void* d_cic, const double* lfield, double* out2);
/* Drop-in for hprod_dipole_ (include/wrapper.hpp:114, called by
 * clhprod::dipole, src/hprod/clhprod.cpp:218-222): host lfield(3,3), wfn,
 * cic; writes dip[3], vel[3], acc[3] (td1c_gpu_dipole3 on the library's
 * staging buffers; on an error all nine are NaN and the status word holds
 * the error). */
void hprod_dipole_(const double* lfield, const double* wfn, const double* cic, double* dip, double* vel, double* acc);

/* wfn_orth_cic + wfn_orth_orb (src/wfn/wfn_orth.F90:2-110): normalise the CI
 * vector and Gram-Schmidt the non-frozen orbitals against all earlier
 * orbitals of equal m, in place on device buffers (library stream). */
int td1c_gpu_orth(void* d_wfn, void* d_cic);
/* Imaginary-time relaxation in the form of init_prop12 (src/main/init.cpp:250-319):
 * per cycle ene[s] (host, ncyc values) = total energy of the current state,
 * one zero-field RK4 step of dt (with the absorbing mask) and td1c_gpu_orth.
 * Needs a context bound with icomp = 0 (returns 16 otherwise).  The full-H
 * RK4 step is explicit: dt must respect its stability limit on the grid's
 * largest one-body eigenvalue. */
int td1c_gpu_relax(void* d_wfn, void* d_cic, double dt, int ncyc, double* ene);

/* Device-resident RK4 propagation (clcrk::prop with the standard tableau,
 * src/prop/clcrk.cpp:55-87,221-235, plus wfn_mask after every step).
 * d_wfn / d_cic are device buffers updated in place.  The sin^2 pulse is
 * evaluated on the host at every stage time (clfield1 velocity1/length1)
 * and staged in device memory once per call; steps run as one CUDA graph
 * per step when use_graph != 0. */
int td1c_gpu_rk4(void* d_wfn, void* d_cic, double t0, double dt, int nstep,
                 double fint, double wlen, double numcyc, double cep, int use_graph);
/* The one-body propagators on a device-resident state, in place (library
 * stream, synchronous); *cycles (may be NULL) = correction cycles added.
 * lfield is a host array of 9 doubles. */
int td1c_gpu_h1itr(void* d_wfn, const double* lfield, double dtime, int maxcyc, double thresh, int* cycles);
int td1c_gpu_dpade(void* d_wfn, const double* lfield, double dtime, double alpha_re, double alpha_im, int maxcyc,
                   double thresh, int* cycles);
/* Device-resident split-operator propagation, tdse_split2 with clh1itr +
 * clcrk (src/main/tdse.cpp:225-266, src/prop/clh1itr.cpp:61-94): per step
 * the one-body Crank-Nicolson over dt/2 (field at t + dt/4), RK4 over dt on
 * the RHS of the bound split_type, one-body over dt/2 (field at t + 3dt/4),
 * wfn_mask.  The one-body steps are skipped for split_type 0 (then this is
 * td1c_gpu_rk4).  One CUDA graph per step when use_graph != 0. */
int td1c_gpu_split2(void* d_wfn, void* d_cic, double t0, double dt, int nstep, double fint, double wlen, double numcyc,
                    double cep, int maxcyc, double thresh, int use_graph);
/* ETD-RK2 with the Pade one-body inverse (cletdrk2::prop + cldpade with
 * alpha = 2, src/prop/cletdrk2.cpp:36-61; tdse_prop12 mask per step). */
int td1c_gpu_etdrk2(void* d_wfn, void* d_cic, double t0, double dt, int nstep, double fint, double wlen, double numcyc,
                    double cep, int maxcyc, double thresh, int use_graph);
/* ETD-RK4 (cletdrk4::prop, src/prop/cletdrk4.cpp:53-114) with the rational
 * one-body functions of clh1rat at the default orders 2/2 (clh1rat.cpp:15-47,
 * h1rat_prod.F90:2-95: numerator by one-body products, each denominator
 * factor a banded solve with the laser by correction cycles); tdse_prop12
 * mask per step.  Twelve factor sets are built on the first step. */
int td1c_gpu_etdrk4(void* d_wfn, void* d_cic, double t0, double dt, int nstep, double fint, double wlen, double numcyc,
                    double cep, int maxcyc, double thresh, int use_graph);
/* init_prop12 with cletdrk2 (src/main/init.cpp:250-319): per cycle ene[s] =
 * total energy, one zero-field ETD-RK2 step of dt (no mask), td1c_gpu_orth;
 * needs icomp = 0. */
int td1c_gpu_relax_etdrk2(void* d_wfn, void* d_cic, double dt, int ncyc, int maxcyc, double thresh, double* ene);
/* Make every following td1c_gpu_rk4 step start from the given device state
 * (NULL, NULL to switch off): each step then performs the complete update on
 * the same input, for throughput measurement of a fixed synthetic state. */
int td1c_gpu_rk4_reset(const void* d_wfn0, const void* d_cic0);
/* Self-test of the bounded wait that every staged kernel uses on its
 * mbarriers (a copy or tensor-core commit that never completes): one kernel
 * waits on a barrier that nothing arrives on, gives up after the bound (1 s)
 * and records ST_TIMEOUT in a word of its own (not the context's status).
 * Returns the bits that word holds, ST_TIMEOUT (32) when the bound works;
 * no copy or MMA is in flight, and the context stays usable.  No counterpart
 * in the reference, which has no device waits. */
int td1c_gpu_wait_selftest(void);
/* Synchronise the library stream. */
int td1c_gpu_sync(void);
/* Number of kernel launches issued by the last td1c_gpu_rk4 call. */
long td1c_gpu_launch_count(void);
/* The library's CUDA stream (a cudaStream_t), for callers that time or
 * order their own work against it. */
void* td1c_gpu_stream(void);
/* Run the RHS reps times with CUDA events between its phases and return the
 * mean phase durations in ms[] (phase names comma-separated in names);
 * returns the number of phases or a status > 0 on failure. */
int td1c_gpu_profile(int reps, double dtime, const double* lfield, const void* d_wfn, const void* d_cic,
                     void* d_hwfn, void* d_hcic, double* ms, char* names, int names_cap);

/* MO two-electron integrals for callers that cannot allocate GPU memory.
 * No counterpart in the reference.
 *
 * Computes int2e(i,j,k,l) = sum_x rho2_ij[x] v2sph_kl[x] (x over K complex
 * basis values, m_i + m_k = m_j + m_l, int2e(i,j,k,l) = conj(int2e(j,i,l,k)))
 * like the integrals of hprod_htot_, and needs no bound context and no
 * device allocation.  It is meant for hosts whose GPU memory belongs to
 * their own pool allocator, real-time loops that must not call cudaMalloc
 * (which synchronises the device and can fail), and frameworks that lend
 * only their own buffers.
 *
 *   nact        active orbitals, 1..16
 *   mval        host array [nact], m of each active orbital
 *   K           complex values per pair (Nr (lmax2 + 1) in the RHS)
 *   d_rho2      device [nact(nact+1)/2][K] complex: pair densities of
 *               (a, b), a >= b, in the packed lower triangle stored by
 *               columns, (0,0) (1,0) .. (n-1,0) (1,1) (2,1) ..
 *   d_v2sph     device, same layout: pair potentials
 *   d_int2e     device [nact^4] complex output, int2e(i,j,k,l) at
 *               i + n (j + n (k + n l)); cleared by the call
 *   stream      cudaStream_t the work is queued on (NULL: legacy stream)
 *
 * Scratch (block tables and split-K partial sums) lives in one 8 MiB device
 * array built into the library.  The call uses the current device and its
 * primary context: make it with the device that owns d_rho2, d_v2sph and
 * d_int2e current.  The array is reserved when CUDA loads this file's
 * module on a device: at the first call on that device under CUDA's default
 * lazy module loading (CUDA_MODULE_LOADING=EAGER reserves it when the
 * library is loaded), after which the device holds it until the process
 * exits.  So make the first call on each device during set-up, before a
 * pool allocator takes the device's memory and before any stream capture;
 * that first call also looks up the array's device address, which later
 * calls reuse (after cudaDeviceReset on that device, do not call it again
 * in the same process).  All calls on a device share the array, and it
 * keeps the last call's contents: calls whose GPU work overlaps (different
 * streams or unordered host threads) race and give wrong results, and so do
 * replays of a CUDA graph that holds the call, whichever graph or stream
 * they run on: order every direct call and replay like calls on one stream.
 * Returns 0 on success, 16 with a message on stderr when a size exceeds
 * these limits or an argument is null, 8 when a CUDA call fails.  The work
 * is asynchronous on the stream. */
int td1c_gpu_int2e_static(int nact, const int* mval, long K, const double* d_rho2, const double* d_v2sph,
                          double* d_int2e, void* stream);

/* ---- ensembles of independent jobs --------------------------------------
 * No counterpart in the reference, whose clhprod is a process singleton
 * (src/hprod/clhprod.cpp:32-34).  Every entry point above acts on the
 * current context; context 0 is the default one (the drop-in calls' context,
 * also current after loading).  A new context holds one job: bind, init and
 * set_wfn0 it like the default one; it gets streams of its own. */
int td1c_gpu_ctx_create(void);   /* new context, made current; returns its id (>= 1) */
int td1c_gpu_ctx_select(int id); /* make context id current; 16 for an unknown id */
int td1c_gpu_ctx_current(void);
int td1c_gpu_ctx_destroy(int id); /* hprod_final_ of context id (>= 1); the default context becomes current */
/* launch shapes of the current context (0 = the built-in choice): mt the
 * FP64 Legendre GEMM's m-tiles per CTA (3 or 6), mf_cap the cap of the
 * persistent mean-field action grid, i2_split the K split of int2e (at most
 * the allocated split, get_tuning's out4[3]); a negative i2_split runs int2e
 * with split -i2_split (-1: the built-in split) on the main stream after the
 * mean-field action instead of beside it on a side stream */
int td1c_gpu_set_tuning(int mt, int mf_cap, int i2_split);
int td1c_gpu_get_tuning(int* out4);
/* nstep split2 steps (td1c_gpu_split2 with its mask) of njob jobs at once:
 * job j is context ids[j] (bound with split_type 1) with state d_wfn[j],
 * d_cic[j] and its own pulse (t0, dt, fint, wlen, numcyc, cep per job).  One
 * CUDA graph holds one step of every job, each job's kernels on its own
 * streams forked from one stream, so the jobs run side by side; it is
 * replayed nstep times.  *ms (host, may be NULL) = device time of the
 * replays.  Returns 0 or the status bits of the jobs. */
int td1c_gpu_ensemble_split2(int njob, const int* ids, void* const* d_wfn, void* const* d_cic, const double* t0,
                             const double* dt, int nstep, const double* fint, const double* wlen, const double* numcyc,
                             const double* cep, int maxcyc, double thresh, double* ms);

/* ---- the learned form of the propagation -------------------------------
 * No counterpart in the reference.  td1c_gpu_split2 (tdse_split2) with the
 * mean field of the RK4 stages predicted instead of formed from the stage
 * orbitals: once per step the exact pair potentials W and integrals int2e of
 * the step's start state are formed (the pair densities, Poisson, the
 * l -> theta transform) and kept in a history of five; the stages take
 * W(c) at c = 0 (the exact value), 1/2 and 1 from it, per unit (a stored
 * pair and one FEDVR element) with weights = the cubic extrapolation through
 * the last four steps + a correction from the registered network.  The exact
 * value of every step judges the previous step's prediction (relative error
 * over all units).  Windows of 8 steps: a window of exact steps that fills
 * the history also judges the predictions it would have made; only when
 * their largest judge value is at most the bound are predicted steps tried.
 * A window of predicted steps stands if its largest judge value is at most
 * the bound, else the state returns to the window's start and the window
 * is recomputed exactly.  After a judge value above the bound, exact steps
 * without history run for a back-off of 1, 3, 7, ... (at most 63) windows
 * (63 at once when the judge value is more than ten times the bound).
 * Needs a context bound with split_type 1 (the RHS without h0 and laser). */
/* Register the network (device pointers, FP32 weights as td1c_mlp_forward
 * takes them, widths 32 .. 8; pack: td1c_mlp_pack_size bytes, the BF16
 * copy the steps read: pack it with td1c_mlp_infer_bf16(repack = 1) after
 * every weight update); use_net = 0 runs the cubic weights alone (the
 * method without the network); depth = 0 unregisters.  bound: the judge's
 * largest accepted relative error (1e-6 by default). */
int td1c_gpu_set_learned(int depth, const int* sizes, const float* const* W, const float* const* b, void* pack, int use_net,
                         double bound);
/* screen = 1 (default): predicted windows only after a history-filling window
 * whose judge values pass the bound; 0: after every history-filling window
 * (each predicted window is then judged and, above the bound, rolled back). */
int td1c_gpu_set_learned_policy(int screen);
/* learned split2 steps on device buffers (arguments as td1c_gpu_split2);
 * stats (host, 10 doubles, may be NULL): windows accepted, rejected, exact
 * (back-off), history fills; largest judge value of an accepted window;
 * smallest and largest window judge value; predicted steps kept; the last
 * window's judge value; steps run. */
int td1c_gpu_split2_learned(void* d_wfn, void* d_cic, double t0, double dt, int nstep, double fint, double wlen, double numcyc,
                            double cep, int maxcyc, double thresh, double* stats);
/* exact split2 steps that write the predictor's training records into
 * d_record (device, (nstep + 1) * nunit * 41 doubles): per step and unit the
 * Gram matrix of the previous four history values (4 x 4 complex), their
 * products with the new value (4 complex) and its squared norm; the first
 * four steps' records precede a full history. */
int td1c_gpu_learned_record(void* d_wfn, void* d_cic, double t0, double dt, int nstep, double fint, double wlen, double numcyc,
                            double cep, int maxcyc, double thresh, double* d_record);
/* out4 = units, FEDVR elements, stored pairs, doubles per record */
int td1c_gpu_learned_dims(int* out4);
/* the kind of each stored pair (0 diagonal, 1 off-diagonal, 2 with the frozen core) */
int td1c_gpu_learned_pair_kind(int* out);
/* network inputs (n x 32 floats) of training records (idx: record index of
 * each sample, NULL: 0..n-1; unit = record index mod nu), computed as the
 * steps compute them */
int td1c_lp_features(int n, const double* rec, const int* idx, int nu, int nfe, const int* pair_kind, float* x, void* stream);
/* relative squared error of each sample's prediction with weights cubic +
 * out (n x 8: re, im of the four corrections) into loss[n] (FP64), and the
 * gradient of their mean with respect to out into dy (NULL: none); use_net = 0
 * evaluates the cubic alone */
int td1c_lp_loss(int n, const double* rec, const int* idx, const float* out, float* dy, double* loss, int use_net, void* stream);

/* ---- the learned mean-field predictor's network ------------------------
 * No counterpart in the reference (td1c has no learned component).  A stack
 * of depth linear layers with tanh between them, widths sizes[0] (input) ..
 * sizes[depth] (output), depth <= 8; W[k], b[k] device pointers to layer
 * k+1's FP32 weights [sizes[k+1] x sizes[k]] (row-major) and bias.  All
 * buffers are device pointers; work is queued on stream (NULL: legacy).
 * Return 0, 16 for bad arguments, 8 when a launch fails. */
/* forward in FP32: acts receives every layer's output (sum_k rows * sizes[k]
 * floats, k = 1..depth; the network output is the last block) */
int td1c_mlp_forward(int depth, const int* sizes, const float* const* W, const float* const* b, const float* x, int rows,
                     float* acts, void* stream);
/* the hand-written backward pass for the output gradient dy [rows x
 * sizes[depth]]: dW[k], db[k] overwritten; work: 2 * rows * max(sizes) floats */
int td1c_mlp_backward(int depth, const int* sizes, const float* const* W, const float* x, int rows, const float* acts,
                      const float* dy, float* const* dW, float* const* db, float* work, void* stream);
/* one Adam step (Kingma and Ba) on n parameters; step = 1-based step count */
int td1c_mlp_adam(long n, float* p, const float* g, float* m, float* v, float lr, float beta1, float beta2, float eps, int step,
                  void* stream);
/* BF16 inference on the tensor cores (tcgen05.mma kind::f16, FP32
 * accumulation): widths <= 256; pack is a device buffer of
 * td1c_mlp_pack_size bytes that holds the BF16 weights, rebuilt from W when
 * repack != 0; y [rows x sizes[depth]] FP32; a bounded wait that runs out
 * sets ST_TIMEOUT (32) in *status (device). */
long td1c_mlp_pack_size(int depth, const int* sizes);
int td1c_mlp_infer_bf16(int depth, const int* sizes, const float* const* W, const float* const* b, void* pack, int repack,
                        const float* x, int rows, float* y, int* status, void* stream);

#ifdef __cplusplus
}
#endif
#endif
