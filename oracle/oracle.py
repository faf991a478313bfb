"""ctypes wrapper of the CPU oracle (liboracle built by oracle/Makefile).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline / reference leg of bench.py.  The product package never imports
this module.  See td1c_oracle.h for the restated reference routines and for
why parity against the reference binary is unpinned.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libtd1c_oracle.so")
_lib = None


def build():
    """Compile the oracle with its Makefile (system g++, OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def _load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        build()
    lib = ctypes.CDLL(_LIB_PATH)
    vp, dp, ip = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)
    lib.orc_create.restype = vp
    lib.orc_create.argtypes = [ctypes.POINTER(OrcConfig)]
    lib.orc_destroy.argtypes = [vp]
    lib.orc_dims.argtypes = [vp, ip]
    lib.orc_get.restype = ctypes.c_long
    lib.orc_get.argtypes = [vp, ctypes.c_char_p, dp]
    lib.orc_set_wfn0.argtypes = [vp, dp, dp]
    lib.orc_htot.argtypes = [vp, ctypes.c_double, dp, dp, dp, dp, dp]
    lib.orc_energies.argtypes = [vp, dp]
    lib.orc_field.argtypes = [ctypes.POINTER(OrcPulse), ctypes.c_double, dp]
    lib.orc_rk4.argtypes = [vp, ctypes.POINTER(OrcPulse), ctypes.c_double, ctypes.c_double, ctypes.c_int, dp, dp, dp]
    lib.orc_orth.argtypes = [vp, dp, dp]
    lib.orc_relax.argtypes = [vp, ctypes.c_double, ctypes.c_int, dp, dp, dp]
    lib.orc_set_split.argtypes = [vp, ctypes.c_int]
    lib.orc_h1itr_prop.restype = ctypes.c_int
    lib.orc_h1itr_prop.argtypes = [vp, dp, ctypes.c_double, ctypes.c_int, ctypes.c_double, dp]
    lib.orc_dpade_prod.restype = ctypes.c_int
    lib.orc_dpade_prod.argtypes = [vp, dp, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                   ctypes.c_double, dp]
    lib.orc_etd4_fun.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_int, dp]
    lib.orc_v2sph.restype = ctypes.c_int
    lib.orc_v2sph.argtypes = [vp, dp]
    lib.orc_dipole3.restype = ctypes.c_int
    lib.orc_dipole3.argtypes = [vp, dp, dp, dp, dp]
    for name in ("orc_split2", "orc_etdrk2", "orc_etdrk4"):
        getattr(lib, name).argtypes = [vp, ctypes.POINTER(OrcPulse), ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                       ctypes.c_int, ctypes.c_double, dp, dp, dp]
    lib.orc_relax_etdrk2.argtypes = [vp, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_double, dp, dp, dp]
    lib.orc_dipole.restype = ctypes.c_double
    lib.orc_dipole.argtypes = [vp, dp, dp]
    lib.orc_num_threads.restype = ctypes.c_int
    _lib = lib
    return lib


class OrcConfig(ctypes.Structure):
    _fields_ = [
        ("znuc", ctypes.c_double), ("rmin", ctypes.c_double), ("rmax", ctypes.c_double),
        ("ndvr", ctypes.c_int), ("nfe", ctypes.c_int),
        ("lmax1", ctypes.c_int), ("lmax2", ctypes.c_int), ("nlat", ctypes.c_int),
        ("nfun", ctypes.c_int),
        ("otype", ctypes.POINTER(ctypes.c_int)), ("mval", ctypes.POINTER(ctypes.c_int)),
        ("lval", ctypes.POINTER(ctypes.c_int)),
        ("nela", ctypes.c_int), ("nelb", ctypes.c_int), ("mtot", ctypes.c_int), ("smul", ctypes.c_int),
        ("igauge", ctypes.c_int), ("icomp", ctypes.c_int),
        ("rmask", ctypes.c_double), ("mask_cos_order", ctypes.c_double),
    ]


class OrcPulse(ctypes.Structure):
    _fields_ = [("fint", ctypes.c_double), ("wlen", ctypes.c_double), ("numcyc", ctypes.c_double),
                ("cep", ctypes.c_double), ("igauge", ctypes.c_int)]


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


DIM_NAMES = ["nrad", "nbas", "nbas2", "ngrid", "nlat", "lcic", "nfcore", "ndcore", "nact",
             "ncore", "nstr_a", "nstr_b", "ndvr", "lmax1", "lmax2", "nfun"]


class Oracle:
    """One oracle instance for a workload dict (see td1c_b200.workloads)."""

    def __init__(self, wl):
        self.lib = _load()
        self.wl = dict(wl)
        orbs = wl["orbitals"]
        self._ot = (ctypes.c_int * len(orbs))(*[o[3] for o in orbs])
        self._mv = (ctypes.c_int * len(orbs))(*[o[2] for o in orbs])
        self._lv = (ctypes.c_int * len(orbs))(*[o[1] for o in orbs])
        cfg = OrcConfig(
            znuc=wl["znuc"], rmin=wl["rmin"], rmax=wl["rmax"], ndvr=wl["ndvr"], nfe=wl["nfe"],
            lmax1=wl["lmax1"], lmax2=wl["lmax2"], nlat=wl.get("nlat", 0) or 0, nfun=len(orbs),
            otype=self._ot, mval=self._mv, lval=self._lv, nela=wl["nela"], nelb=wl["nelb"],
            mtot=wl.get("mtot", 0), smul=wl.get("smul", 1), igauge=wl["igauge"], icomp=wl.get("icomp", 1),
            rmask=wl["rmask"], mask_cos_order=wl["mask_cos_order"])
        self.h = self.lib.orc_create(ctypes.byref(cfg))
        d = (ctypes.c_int * 16)()
        self.lib.orc_dims(self.h, d)
        self.dims = dict(zip(DIM_NAMES, list(d)))

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.orc_destroy(self.h)
            self.h = None

    def get(self, name, complex_=None):
        n = self.lib.orc_get(self.h, name.encode(), None)
        if n < 0:
            raise KeyError(name)
        out = np.zeros(n, dtype=np.float64)
        self.lib.orc_get(self.h, name.encode(), _dp(out))
        if complex_:
            out = out.view(np.complex128)
        return out

    def set_wfn0(self, wfn, cic):
        wfn = np.ascontiguousarray(wfn, dtype=np.complex128)
        cic = np.ascontiguousarray(cic, dtype=np.complex128)
        self.lib.orc_set_wfn0(self.h, _dp(wfn.view(np.float64)), _dp(cic.view(np.float64)))

    def htot(self, dtime, lfield, wfn, cic):
        wfn = np.ascontiguousarray(wfn, dtype=np.complex128)
        cic = np.ascontiguousarray(cic, dtype=np.complex128)
        lf = np.ascontiguousarray(lfield, dtype=np.float64)
        hw = np.zeros_like(wfn)
        hc = np.zeros_like(cic)
        self.lib.orc_htot(self.h, float(dtime), _dp(lf), _dp(wfn.view(np.float64)), _dp(cic.view(np.float64)),
                          _dp(hw.view(np.float64)), _dp(hc.view(np.float64)))
        return hw, hc

    def v2sph(self):
        """Pair potentials v2sph of the last RHS for the 'dyn' pairs (j >= i, both dynamic):
        [npair][lmax2 + 1][nrad - 1] complex."""
        ndyn = len(self.wl["orbitals"]) - self.dims["nfcore"]
        shape = (ndyn * (ndyn + 1) // 2, self.wl["lmax2"] + 1, self.dims["nrad"] - 1)
        out = np.zeros(shape, dtype=np.complex128)
        n = self.lib.orc_v2sph(self.h, _dp(out.view(np.float64)))
        assert n == shape[0]
        return out

    def energies(self):
        e = np.zeros(5)
        self.lib.orc_energies(self.h, _dp(e))
        return dict(zip(["ene_fcore", "ene_dcore", "ene_core", "ene_act", "ene_tot"], e.tolist()))

    def pulse(self):
        wl = self.wl
        return OrcPulse(fint=wl["fint"], wlen=wl["wlen"], numcyc=wl["numcyc"], cep=wl.get("cep", 0.0),
                        igauge=wl["igauge"])

    def field(self, t):
        lf = np.zeros(9)
        p = self.pulse()
        self.lib.orc_field(ctypes.byref(p), float(t), _dp(lf))
        return lf

    def rk4(self, wfn, cic, t0, dt, nstep):
        wfn = np.array(wfn, dtype=np.complex128, copy=True)
        cic = np.array(cic, dtype=np.complex128, copy=True)
        dip = np.zeros(nstep)
        p = self.pulse()
        self.lib.orc_rk4(self.h, ctypes.byref(p), float(t0), float(dt), int(nstep), _dp(wfn.view(np.float64)),
                         _dp(cic.view(np.float64)), _dp(dip))
        return wfn, cic, dip

    def orth(self, wfn, cic):
        """Gram-Schmidt of the orbitals within each m and CI normalisation (returns copies)."""
        wfn = np.ascontiguousarray(wfn, dtype=np.complex128).copy()
        cic = np.ascontiguousarray(cic, dtype=np.complex128).copy()
        self.lib.orc_orth(self.h, _dp(wfn.view(np.float64)), _dp(cic.view(np.float64)))
        return wfn, cic

    def relax(self, wfn, cic, dt, ncyc):
        """Imaginary-time relaxation (icomp = 0); returns (wfn, cic, energy per cycle)."""
        wfn = np.ascontiguousarray(wfn, dtype=np.complex128).copy()
        cic = np.ascontiguousarray(cic, dtype=np.complex128).copy()
        ene = np.zeros(ncyc)
        self.lib.orc_relax(self.h, float(dt), int(ncyc), _dp(wfn.view(np.float64)), _dp(cic.view(np.float64)), _dp(ene))
        return wfn, cic, ene

    def set_split(self, isplit):
        """split_type: 0 full H in the RHS, 1 two-body part only, 2 h0 left out."""
        self.lib.orc_set_split(self.h, int(isplit))

    def h1itr_prop(self, lfield, dtime, wfn, maxcyc=20, thresh=1e-10):
        """One h1itr Crank-Nicolson step over dtime; returns (wfn, cycles)."""
        wfn = np.ascontiguousarray(wfn, dtype=np.complex128).copy()
        lf = np.ascontiguousarray(lfield, dtype=np.float64)
        n = self.lib.orc_h1itr_prop(self.h, _dp(lf), float(dtime), int(maxcyc), float(thresh), _dp(wfn.view(np.float64)))
        return wfn, n

    def dpade_prod(self, lfield, dtime, wfn, alpha=2.0, maxcyc=20, thresh=1e-10):
        """(1 + i dtime/alpha (T + V))^-1 on the non-frozen orbitals; returns (wfn, cycles)."""
        wfn = np.ascontiguousarray(wfn, dtype=np.complex128).copy()
        lf = np.ascontiguousarray(lfield, dtype=np.float64)
        a = complex(alpha)
        n = self.lib.orc_dpade_prod(self.h, _dp(lf), float(dtime), a.real, a.imag, int(maxcyc), float(thresh),
                                    _dp(wfn.view(np.float64)))
        return wfn, n

    def _prop(self, name, wfn, cic, t0, dt, nstep, maxcyc, thresh):
        wfn = np.array(wfn, dtype=np.complex128, copy=True)
        cic = np.array(cic, dtype=np.complex128, copy=True)
        dip = np.zeros(nstep)
        p = self.pulse()
        getattr(self.lib, name)(self.h, ctypes.byref(p), float(t0), float(dt), int(nstep), int(maxcyc), float(thresh),
                                _dp(wfn.view(np.float64)), _dp(cic.view(np.float64)), _dp(dip))
        return wfn, cic, dip

    def split2(self, wfn, cic, t0, dt, nstep, maxcyc=20, thresh=1e-10):
        """tdse_split2 (h1itr + RK4 + h1itr, mask); returns (wfn, cic, dipole per step)."""
        return self._prop("orc_split2", wfn, cic, t0, dt, nstep, maxcyc, thresh)

    def etdrk2(self, wfn, cic, t0, dt, nstep, maxcyc=20, thresh=1e-10):
        """ETD-RK2 with the Pade one-body inverse (mask per step); returns (wfn, cic, dipole per step)."""
        return self._prop("orc_etdrk2", wfn, cic, t0, dt, nstep, maxcyc, thresh)

    def etdrk4(self, wfn, cic, t0, dt, nstep, maxcyc=20, thresh=1e-10):
        """ETD-RK4 with the rational one-body functions of clh1rat (orders 2/2, mask per step);
        returns (wfn, cic, dipole per step)."""
        return self._prop("orc_etdrk4", wfn, cic, t0, dt, nstep, maxcyc, thresh)

    def dipole3(self, wfn, cic, lfield):
        """hprod_dipole: (dip[3], vel[3], acc[3]); with frozen-core orbitals vel[1], acc[1] are the
        generalized-Fock corrections and vel[2], acc[2] the totals."""
        wfn = np.ascontiguousarray(wfn, dtype=np.complex128)
        cic = np.ascontiguousarray(cic, dtype=np.complex128)
        out = np.zeros(9)
        rc = self.lib.orc_dipole3(self.h, _dp(wfn.view(np.float64)), _dp(cic.view(np.float64)),
                                  _dp(np.ascontiguousarray(lfield, dtype=np.float64)), _dp(out))
        return None if rc else (out[0:3], out[3:6], out[6:9])

    def etd4_fun(self, which, dt):
        """Coefficients of ETD-RK4 function `which` (0 exp1, 1 exp2, 2 gfun, 3 f0, 4 f1, 5 f2):
        dict n[3], d0[2], d1[2], rk (complex) and dt."""
        out = np.zeros(17)
        self.lib.orc_etd4_fun(int(which), float(dt), int(self.wl.get("icomp", 1)), _dp(out))
        z = out[:16].view(np.complex128)
        return {"n": z[0:3], "d0": z[3:5], "d1": z[5:7], "rk": z[7], "dt": out[16]}

    def relax_etdrk2(self, wfn, cic, dt, ncyc, maxcyc=20, thresh=1e-10):
        """Imaginary-time relaxation with ETD-RK2 steps (icomp = 0); returns (wfn, cic, energy per cycle)."""
        wfn = np.ascontiguousarray(wfn, dtype=np.complex128).copy()
        cic = np.ascontiguousarray(cic, dtype=np.complex128).copy()
        ene = np.zeros(ncyc)
        self.lib.orc_relax_etdrk2(self.h, float(dt), int(ncyc), int(maxcyc), float(thresh), _dp(wfn.view(np.float64)),
                                  _dp(cic.view(np.float64)), _dp(ene))
        return wfn, cic, ene

    def dipole(self, wfn, cic):
        wfn = np.ascontiguousarray(wfn, dtype=np.complex128)
        cic = np.ascontiguousarray(cic, dtype=np.complex128)
        return self.lib.orc_dipole(self.h, _dp(wfn.view(np.float64)), _dp(cic.view(np.float64)))

    def num_threads(self):
        return self.lib.orc_num_threads()
