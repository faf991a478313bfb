"""Python host mirror of td1c's clhprod (src/hprod/clhprod.cpp) over the C-ABI.

clhprod::gen binds the energy outputs and calls hprod_init_; set_wfn0 calls
hprod_set_wfn0_; htot calls hprod_htot_ (clhprod.cpp:29-82).  The grid and
tables are bound first, as clbas::gen does through bas_rad_bind_ /
bas_sph_bind_ / bas_bas_bind_ (clbas.cpp:52-146).  All arithmetic happens in
libtd1c_b200.so on the GPU; this module only moves host buffers.
"""
import ctypes

import numpy as np

from . import _lib as _libmod

_DP = ctypes.POINTER(ctypes.c_double)


def _dp(a):
    return a.ctypes.data_as(_DP)


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


class StatusError(RuntimeError):
    pass


class _CtxLib:
    """The library with a context selected before every call (the library's entry points act on its
    current context; an ensemble holds one context per job)."""

    def __init__(self, lib, ctx_id):
        self._lib, self._id = lib, ctx_id

    def __getattr__(self, name):
        f = getattr(self._lib, name)
        if name.startswith(("td1c_gpu_ctx_", "td1c_mlp_", "td1c_lp_", "td1c_gpu_ensemble")):
            return f
        lib, cid = self._lib, self._id

        def call(*a):
            lib.td1c_gpu_ctx_select(cid)
            return f(*a)
        return call


class HProd:
    """One GPU RHS instance.  The default one lives in the library's default context (the
    drop-in entry points' context, like td1c's clhprod singleton, clhprod.cpp:32-34);
    new_context=True gives it a context of its own (a job of an ensemble)."""

    def __init__(self, wl, rad, ang, new_context=False):
        raw = _libmod.load()
        if new_context:
            self.ctx_id = int(raw.td1c_gpu_ctx_create())
        else:
            self.ctx_id = 0
            raw.td1c_gpu_ctx_select(0)
        self.lib = _CtxLib(raw, self.ctx_id)
        self.wl = wl
        lib = self.lib
        orbs = wl["orbitals"]
        self.nfun = len(orbs)
        self._keep = []

        def keep(a):
            a = np.ascontiguousarray(a, dtype=np.float64)
            self._keep.append(a)
            return a

        xrad, wrad, mask = keep(rad["xrad"]), keep(rad["wrad"]), keep(rad["mask"])
        radk, radk0, radp = keep(rad["radk"]), keep(rad["radk0"]), keep(rad["radp"])
        self._check(lib.td1c_gpu_bind_rad(rad["nfe"], rad["ndvr"], rad["nrad"], _dp(xrad), _dp(wrad), _dp(radp),
                                          _dp(radk), _dp(radk0), float(rad["rmask"]), _dp(mask)))
        wlat, cost = keep(ang["wlat"]), keep(ang["cost"])
        lf1, lb1, lf2, lb2 = keep(ang["legf1"]), keep(ang["legb1"]), keep(ang["legf2"]), keep(ang["legb2"])
        self._check(lib.td1c_gpu_bind_sph(ang["lmax1"], ang["lmax2"], ang["mmax1"], ang["mmax2"], ang["nlat"],
                                          _dp(wlat), _dp(cost), _dp(lf1), _dp(lb1), _dp(lf2), _dp(lb2)))
        ot = np.array([o[3] for o in orbs], dtype=np.int32)
        mv = np.array([o[2] for o in orbs], dtype=np.int32)
        lv = np.array([o[1] for o in orbs], dtype=np.int32)
        self._keep += [ot, mv, lv]
        self._check(lib.td1c_gpu_bind_bas(float(wl["znuc"]), int(wl.get("smul", 1)), int(wl.get("mtot", 0)),
                                          self.nfun, _ip(ot), _ip(mv), _ip(lv), int(wl["nela"]), int(wl["nelb"])))
        self._check(lib.td1c_gpu_bind_ormas(int(wl.get("nsub", 1))))
        self._check(lib.td1c_gpu_bind_control(int(wl.get("icomp", 1)), int(wl["igauge"])))
        self._check(lib.td1c_gpu_bind_split(int(wl.get("split_type", 0))))
        self.ene = np.zeros(8)
        projhigh = ctypes.c_bool(False)
        cutoff = ctypes.c_double(0.0)
        e = self.ene
        lib.hprod_bind_(*[e[i:].ctypes.data_as(_DP) for i in range(8)], ctypes.byref(projhigh), ctypes.byref(cutoff))
        self._projhigh, self._cutoff = projhigh, cutoff
        lib.hprod_init_()
        self._status()
        d = (ctypes.c_int * 16)()
        lib.td1c_gpu_dims(d)
        names = ["nrad", "nbas", "nbas2", "ngrid", "nlat", "lcic", "nfcore", "ndcore", "nact", "ncore",
                 "nstr_a", "nstr_b", "npair", "ndvr", "lmax1", "lmax2"]
        self.dims = dict(zip(names, list(d)))

    def _check(self, rc):
        if rc != 0:
            raise StatusError("td1c_b200 call failed with status %d" % rc)

    def _status(self):
        st = self.lib.td1c_gpu_last_status()
        if st != 0:
            raise StatusError("td1c_b200 status %d" % st)

    def ci_tables(self):
        d = self.dims
        na, nb = max(d["nstr_a"], 1), max(d["nstr_b"], 1)
        stra = np.zeros(na, dtype=np.uint32)
        strb = np.zeros(nb, dtype=np.uint32)
        detoff = np.zeros(nb, dtype=np.int32)
        afirst = np.zeros(nb, dtype=np.int32)
        acount = np.zeros(nb, dtype=np.int32)
        up = ctypes.POINTER(ctypes.c_uint)
        self.lib.td1c_gpu_ci_tables(stra.ctypes.data_as(up), strb.ctypes.data_as(up), _ip(detoff), _ip(afirst),
                                    _ip(acount))
        return dict(stra=stra[:d["nstr_a"]], strb=strb[:d["nstr_b"]], detoff=detoff[:d["nstr_b"]],
                    afirst=afirst[:d["nstr_b"]], acount=acount[:d["nstr_b"]])

    def set_wfn0(self, wfn, cic):
        wfn = np.ascontiguousarray(wfn, dtype=np.complex128)
        cic = np.ascontiguousarray(cic, dtype=np.complex128)
        t = b"read"
        self.lib.hprod_set_wfn0_(_dp(wfn.view(np.float64)), _dp(cic.view(np.float64)), t, len(t))
        self._status()

    def htot(self, dtime, lfield, wfn, cic):
        """hprod_htot_ on host buffers; returns (hwfn, hcic)."""
        wfn = np.ascontiguousarray(wfn, dtype=np.complex128)
        cic = np.ascontiguousarray(cic, dtype=np.complex128)
        lf = np.ascontiguousarray(lfield, dtype=np.float64)
        hw = np.zeros_like(wfn)
        hc = np.zeros_like(cic)
        dt = ctypes.c_double(dtime)
        self.lib.hprod_htot_(ctypes.byref(dt), _dp(lf), _dp(wfn.view(np.float64)), _dp(cic.view(np.float64)),
                             _dp(hw.view(np.float64)), _dp(hc.view(np.float64)))
        self._status()
        return hw, hc

    def energies(self):
        """ene_fcore, ene_dcore, ene_core, ene_act, ene_tot bound by hprod_bind_."""
        return dict(zip(["ene_fcore", "ene_dcore", "ene_core", "ene_act", "ene_tot"], self.ene[:5].tolist()))

    def debug(self, name, complex_=True):
        n = self.lib.td1c_gpu_debug_get(name.encode(), None, 0)
        if n < 0:
            raise KeyError(name)
        out = np.zeros(n)
        self.lib.td1c_gpu_debug_get(name.encode(), _dp(out), n)
        return out.view(np.complex128) if complex_ else out

    # device-resident paths (pointers are CUDA device addresses, e.g. torch tensors' data_ptr())
    def htot_dev(self, dtime, lfield, d_wfn, d_cic, d_hwfn, d_hcic):
        lf = np.ascontiguousarray(lfield, dtype=np.float64)
        self._check(self.lib.td1c_gpu_htot_dev(float(dtime), _dp(lf), ctypes.c_void_p(d_wfn), ctypes.c_void_p(d_cic),
                                               ctypes.c_void_p(d_hwfn), ctypes.c_void_p(d_hcic)))

    def rk4_dev(self, d_wfn, d_cic, t0, dt, nstep, use_graph=True):
        wl = self.wl
        self._check(self.lib.td1c_gpu_rk4(ctypes.c_void_p(d_wfn), ctypes.c_void_p(d_cic), float(t0), float(dt),
                                          int(nstep), float(wl["fint"]), float(wl["wlen"]), float(wl["numcyc"]),
                                          float(wl.get("cep", 0.0)), 1 if use_graph else 0))

    def dipole_dev(self, d_wfn, d_cic):
        """Length-form dipole <z> of a device-resident state (hprod_dipole.F90, dip(1))."""
        out = np.zeros(1)
        self._check(self.lib.td1c_gpu_dipole(ctypes.c_void_p(d_wfn), ctypes.c_void_p(d_cic), _dp(out)))
        return float(out[0])

    def dipole3_dev(self, d_wfn, d_cic, lfield):
        """hprod_dipole of a device state: (dip[3], vel[3], acc[3]), the length, velocity and
        acceleration forms (with frozen-core orbitals vel[1], acc[1] are the generalized-Fock
        corrections)."""
        out = np.zeros(9)
        lf = np.ascontiguousarray(lfield, dtype=np.float64)
        self._check(self.lib.td1c_gpu_dipole3(ctypes.c_void_p(d_wfn), ctypes.c_void_p(d_cic), _dp(lf), _dp(out)))
        return out[0:3], out[3:6], out[6:9]

    def set_mixed(self, on):
        """Mixed-precision form of every later RHS: the mean field's pair-density multipoles and pair
        potentials in split TF32 on the tensor cores (on=True or 1; 2 = the same arithmetic on the
        per-tile kernel; 3 = mode 1 with the Poisson interior products and int2e in split TF32 too),
        or plain FP64 (on=False or 0)."""
        self._check(self.lib.td1c_gpu_set_mixed(int(on) if not isinstance(on, bool) else (1 if on else 0)))

    def mixed_selftest(self, d_wfn, d_cic, lfield):
        """Relative deviation of the mixed form from FP64 on one RHS: (pair-density multipoles,
        pair potentials on the grid, hwfn)."""
        out = np.zeros(3)
        lf = np.ascontiguousarray(lfield, dtype=np.float64)
        self._check(self.lib.td1c_gpu_mixed_selftest(ctypes.c_void_p(d_wfn), ctypes.c_void_p(d_cic), _dp(lf), _dp(out)))
        return out

    def mixed_int2e_selftest(self, d_wfn, d_cic, lfield):
        """The mixed form's tensor-core int2e on one RHS: (relative deviation from the FP64 DMMA
        int2e on the same pair densities and potentials, from the FP64 RHS's int2e), or None where
        the tensor-core plan does not apply."""
        out = np.zeros(2)
        lf = np.ascontiguousarray(lfield, dtype=np.float64)
        rc = self.lib.td1c_gpu_mixed_int2e_selftest(ctypes.c_void_p(d_wfn), ctypes.c_void_p(d_cic), _dp(lf), _dp(out))
        if rc == 16:
            return None
        self._check(rc)
        return out

    def orth_dev(self, d_wfn, d_cic):
        """wfn_orth_cic + wfn_orth_orb in place on device buffers."""
        self._check(self.lib.td1c_gpu_orth(ctypes.c_void_p(d_wfn), ctypes.c_void_p(d_cic)))

    def relax_dev(self, d_wfn, d_cic, dt, ncyc):
        """Imaginary-time relaxation in place (context bound with icomp = 0); returns the energy per cycle."""
        ene = np.zeros(max(1, int(ncyc)))
        self._check(self.lib.td1c_gpu_relax(ctypes.c_void_p(d_wfn), ctypes.c_void_p(d_cic), float(dt), int(ncyc), _dp(ene)))
        return ene[: int(ncyc)]

    def set_time_kind(self, icomp):
        """icomp of control_bind_ (1 real time, 0 imaginary time), keeping the context."""
        self.wl = dict(self.wl, icomp=int(icomp))
        self._check(self.lib.td1c_gpu_bind_control(int(icomp), int(self.wl["igauge"])))

    # ---- one-body propagators of the split schemes (src/prop: clh1itr, cldpade)
    def set_split(self, split_type):
        """split_type of control_bind_: 0 full H in the RHS, 1 two-body part only, 2 h0 left out."""
        self._check(self.lib.td1c_gpu_bind_split(int(split_type)))

    def h1itr_dev(self, d_wfn, lfield, dtime, maxcyc=20, thresh=1e-10):
        """h1itr_prop on a device state in place; returns the corrections added."""
        lf = np.ascontiguousarray(lfield, dtype=np.float64)
        n = ctypes.c_int(0)
        self._check(self.lib.td1c_gpu_h1itr(ctypes.c_void_p(d_wfn), _dp(lf), float(dtime), int(maxcyc), float(thresh),
                                            ctypes.byref(n)))
        return n.value

    def dpade_dev(self, d_wfn, lfield, dtime, alpha=2.0, maxcyc=20, thresh=1e-10):
        """dpade_prod on a device state in place; returns the corrections added."""
        lf = np.ascontiguousarray(lfield, dtype=np.float64)
        a = complex(alpha)
        n = ctypes.c_int(0)
        self._check(self.lib.td1c_gpu_dpade(ctypes.c_void_p(d_wfn), _dp(lf), float(dtime), a.real, a.imag, int(maxcyc),
                                            float(thresh), ctypes.byref(n)))
        return n.value

    def _prop_dev(self, fn, d_wfn, d_cic, t0, dt, nstep, maxcyc, thresh, use_graph):
        wl = self.wl
        self._check(fn(ctypes.c_void_p(d_wfn), ctypes.c_void_p(d_cic), float(t0), float(dt), int(nstep), float(wl["fint"]),
                       float(wl["wlen"]), float(wl["numcyc"]), float(wl.get("cep", 0.0)), int(maxcyc), float(thresh),
                       1 if use_graph else 0))

    def split2_dev(self, d_wfn, d_cic, t0, dt, nstep, maxcyc=20, thresh=1e-10, use_graph=True):
        """tdse_split2 steps (h1itr over dt/2, RK4 over dt, h1itr over dt/2, mask) in place."""
        self._prop_dev(self.lib.td1c_gpu_split2, d_wfn, d_cic, t0, dt, nstep, maxcyc, thresh, use_graph)

    def etdrk2_dev(self, d_wfn, d_cic, t0, dt, nstep, maxcyc=20, thresh=1e-10, use_graph=True):
        """ETD-RK2 steps with the Pade one-body inverse (cletdrk2 + cldpade, mask) in place."""
        self._prop_dev(self.lib.td1c_gpu_etdrk2, d_wfn, d_cic, t0, dt, nstep, maxcyc, thresh, use_graph)

    def etdrk4_dev(self, d_wfn, d_cic, t0, dt, nstep, maxcyc=20, thresh=1e-10, use_graph=True):
        """ETD-RK4 steps with the rational one-body functions (cletdrk4 + clh1rat, orders 2/2, mask) in place."""
        self._prop_dev(self.lib.td1c_gpu_etdrk4, d_wfn, d_cic, t0, dt, nstep, maxcyc, thresh, use_graph)

    def relax_etdrk2_dev(self, d_wfn, d_cic, dt, ncyc, maxcyc=20, thresh=1e-10):
        """Imaginary-time relaxation with ETD-RK2 steps (icomp = 0); returns the energy per cycle."""
        ene = np.zeros(max(1, int(ncyc)))
        self._check(self.lib.td1c_gpu_relax_etdrk2(ctypes.c_void_p(d_wfn), ctypes.c_void_p(d_cic), float(dt), int(ncyc),
                                                   int(maxcyc), float(thresh), _dp(ene)))
        return ene[: int(ncyc)]

    def h1itr_host(self, lfield, dtime, wfn, maxcyc=20, thresh=1e-10, split_type=1):
        """clh1itr's Fortran calls through the drop-in symbols: h1itr_gen_cninv_ then
        h1itr_prop_ on a host copy of wfn (returned)."""
        wfn = np.ascontiguousarray(wfn, dtype=np.complex128).copy()
        lf = np.ascontiguousarray(lfield, dtype=np.float64)
        icomp, isplit, igauge, iprojfc = (ctypes.c_int(v) for v in (self.wl.get("icomp", 1), split_type,
                                                                     self.wl["igauge"], 0))
        dt, thr, mc = ctypes.c_double(dtime), ctypes.c_double(thresh), ctypes.c_int(maxcyc)
        piv = np.zeros(4, dtype=np.int32)
        band = np.zeros(2)
        self.lib.h1itr_gen_cninv_(ctypes.byref(icomp), ctypes.byref(dt), _ip(piv), _dp(band))
        self._status()
        self.lib.h1itr_prop_(ctypes.byref(icomp), ctypes.byref(isplit), ctypes.byref(igauge), ctypes.byref(iprojfc),
                             _dp(lf), ctypes.byref(dt), ctypes.byref(mc), ctypes.byref(thr), _ip(piv), _dp(band),
                             _dp(wfn.view(np.float64)))
        self._status()
        return wfn

    def dpade_host(self, lfield, dtime, wfn, alpha=2.0, maxcyc=20, thresh=1e-10, split_type=1):
        """cldpade's Fortran calls through the drop-in symbols: dpade_gen_ then dpade_prod_
        on a host copy of wfn (returned)."""
        wfn = np.ascontiguousarray(wfn, dtype=np.complex128).copy()
        lf = np.ascontiguousarray(lfield, dtype=np.float64)
        icomp, isplit, igauge, iprojfc = (ctypes.c_int(v) for v in (self.wl.get("icomp", 1), split_type,
                                                                     self.wl["igauge"], 0))
        dt, thr, mc = ctypes.c_double(dtime), ctypes.c_double(thresh), ctypes.c_int(maxcyc)
        al = np.array([complex(alpha).real, complex(alpha).imag])
        piv = np.zeros(4, dtype=np.int32)
        band = np.zeros(2)
        self.lib.dpade_gen_(ctypes.byref(icomp), ctypes.byref(dt), _dp(al), _dp(band), _ip(piv))
        self._status()
        self.lib.dpade_prod_(ctypes.byref(isplit), ctypes.byref(igauge), ctypes.byref(icomp), ctypes.byref(iprojfc),
                             _dp(lf), ctypes.byref(dt), _dp(al), ctypes.byref(mc), ctypes.byref(thr), _ip(piv), _dp(band),
                             _dp(wfn.view(np.float64)))
        self._status()
        return wfn

    def rk4_reset(self, d_wfn0, d_cic0):
        self._check(self.lib.td1c_gpu_rk4_reset(ctypes.c_void_p(d_wfn0) if d_wfn0 else None,
                                                ctypes.c_void_p(d_cic0) if d_cic0 else None))

    def stream(self):
        return int(self.lib.td1c_gpu_stream() or 0)

    def profile(self, reps, lfield, d_wfn, d_cic, d_hwfn, d_hcic, dtime=1.0):
        lf = np.ascontiguousarray(lfield, dtype=np.float64)
        ms = np.zeros(16)
        names = ctypes.create_string_buffer(512)
        n = self.lib.td1c_gpu_profile(int(reps), float(dtime), _dp(lf), ctypes.c_void_p(d_wfn), ctypes.c_void_p(d_cic),
                                      ctypes.c_void_p(d_hwfn), ctypes.c_void_p(d_hcic), _dp(ms), names, 512)
        if n <= 0 or n > 16:
            raise StatusError("td1c_gpu_profile failed (%d)" % n)
        return dict(zip(names.value.decode().split(","), ms[:n].tolist()))

    def debug_ptr(self, name):
        """Device address of a named context buffer ("W", "int2e", "rho2", "v2sph")."""
        p = self.lib.td1c_gpu_debug_ptr(name.encode())
        if not p:
            raise KeyError(name)
        return int(p)

    def debug_xfer(self, name, d_other, to_ctx):
        """Queue a device copy of a named context buffer to (to_ctx=False) or from (to_ctx=True) the
        device buffer d_other on the library stream; returns the bytes copied."""
        n = self.lib.td1c_gpu_debug_xfer(name.encode(), ctypes.c_void_p(d_other), 1 if to_ctx else 0)
        if n < 0:
            raise KeyError(name)
        return n

    def set_mf_external(self, on):
        """on=True: later RHS evaluations take the pair potentials W and int2e as they stand in the
        context (see debug_ptr) instead of computing them from the stage's orbitals."""
        self._check(self.lib.td1c_gpu_set_mf_external(1 if on else 0))

    def pulse_lfield(self, t):
        """lfield(3,3) of the workload's sin^2 pulse at time t, as the propagators stage it."""
        wl = self.wl
        out = np.zeros(9)
        self._check(self.lib.td1c_gpu_pulse_lfield(float(t), float(wl["fint"]), float(wl["wlen"]), float(wl["numcyc"]),
                                                   float(wl.get("cep", 0.0)), _dp(out)))
        return out

    # ---- the learned form (predicted stage mean fields, judge and fallback)
    def learned_dims(self):
        d = (ctypes.c_int * 4)()
        self._check(self.lib.td1c_gpu_learned_dims(d))
        return dict(nu=d[0], nfe=d[1], npair=d[2], rec=d[3])

    def learned_pair_kind(self):
        n = self.learned_dims()["npair"]
        out = np.zeros(n, dtype=np.int32)
        self._check(self.lib.td1c_gpu_learned_pair_kind(_ip(out)))
        return out

    def set_learned(self, net=None, use_net=True, bound=1e-6):
        """Register a learned.DeviceMLP (widths 32 .. 8) for the predicted steps, or none (cubic weights)."""
        if net is None:
            self._check(self.lib.td1c_gpu_set_learned(0, None, None, None, None, 0, float(bound)))
            self._net = None
            return
        net.pack()
        net.torch.cuda.synchronize()  # the BF16 copy is written on torch's stream; the steps read it on the library's
        self._net = net
        self._check(self.lib.td1c_gpu_set_learned(net.depth, net._sizes, net._ptrs(net.W), net._ptrs(net.b),
                                                  ctypes.c_void_p(net._pack.data_ptr()), 1 if use_net else 0, float(bound)))

    def set_learned_policy(self, screen=True):
        """screen=True: predicted windows only after a history-filling window whose judge values
        pass the bound; False: after every such window (rolled back when rejected)."""
        self._check(self.lib.td1c_gpu_set_learned_policy(1 if screen else 0))

    def split2_learned_dev(self, d_wfn, d_cic, t0, dt, nstep, maxcyc=20, thresh=1e-10):
        """Learned split2 steps in place; returns the judge statistics."""
        wl = self.wl
        st = np.zeros(10)
        self._check(self.lib.td1c_gpu_split2_learned(ctypes.c_void_p(d_wfn), ctypes.c_void_p(d_cic), float(t0), float(dt),
                                                     int(nstep), float(wl["fint"]), float(wl["wlen"]), float(wl["numcyc"]),
                                                     float(wl.get("cep", 0.0)), int(maxcyc), float(thresh), _dp(st)))
        keys = ["accepted", "rejected", "exact_windows", "fills", "max_accepted_judge", "min_judge", "max_judge",
                "predicted_steps", "last_judge", "steps"]
        out = dict(zip(keys, st.tolist()))
        if out["min_judge"] > 1e299:
            out["min_judge"] = None
        return out

    def learned_record_dev(self, d_wfn, d_cic, t0, dt, nstep, d_record, fint=None, wlen=None, maxcyc=20, thresh=1e-10):
        """Exact split2 steps writing (nstep + 1) x units training records into the device buffer d_record."""
        wl = self.wl
        self._check(self.lib.td1c_gpu_learned_record(ctypes.c_void_p(d_wfn), ctypes.c_void_p(d_cic), float(t0), float(dt),
                                                     int(nstep), float(fint if fint is not None else wl["fint"]),
                                                     float(wlen if wlen is not None else wl["wlen"]), float(wl["numcyc"]),
                                                     float(wl.get("cep", 0.0)), int(maxcyc), float(thresh),
                                                     ctypes.c_void_p(d_record)))

    def wait_selftest(self):
        """Status bits of the bounded-wait self-test (ST_TIMEOUT = 32 when the wait bound works)."""
        return int(self.lib.td1c_gpu_wait_selftest())

    def last_status(self):
        return int(self.lib.td1c_gpu_last_status())

    def sync(self):
        self._check(self.lib.td1c_gpu_sync())
        self._status()

    def launch_count(self):
        return int(self.lib.td1c_gpu_launch_count())

    def set_tuning(self, mt=0, mf_cap=0, i2_split=0):
        """Launch shapes of this context: the FP64 Legendre GEMM's m-tiles (3 or 6; 0 by size), the
        persistent mean-field grid cap and the int2e split (0: built-in)."""
        self._check(self.lib.td1c_gpu_set_tuning(int(mt), int(mf_cap), int(i2_split)))

    def get_tuning(self):
        out = (ctypes.c_int * 4)()
        self._check(self.lib.td1c_gpu_get_tuning(out))
        return dict(mt=out[0], mf_cap=out[1], i2_split=out[2], i2_split_max=out[3])

    def final(self):
        self.lib.hprod_final_()
        self.lib._lib.td1c_gpu_ctx_select(0)
