"""Unsupported configurations are refused with a status, not approximated (no GPU needed).

The reference stops the program on configurations or inputs it cannot handle
(e.g. src/hprod/hprod_mkv2mf.F90:167-170).  The library instead records
ST_CONFIG (16) and refuses to initialise.  Two configurations the path does
not build are checked here: a frozen core of type -2 (nfcore2 of ormas_bind_,
the local-exchange frozen core of hprod_v2fc, src/hprod/hprod_set_wfn0.F90:
132-210) and ORMAS with more than one subspace (nsub > 1, the active-active
rotation solve of src/ormas/ormas_xact2.F90:46,82).  Both are host-side
checks: binding and hprod_init_ return before any device work.
"""
import ctypes

import numpy as np

from td1c_b200 import basis, workloads as W

ST_CONFIG = 16
DP = ctypes.POINTER(ctypes.c_double)
IP = ctypes.POINTER(ctypes.c_int)


def _bind_geometry(lib, wl):
    rad, ang = basis.build(wl)
    keep = []

    def d(a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        keep.append(a)
        return a.ctypes.data_as(DP)

    assert lib.td1c_gpu_bind_rad(rad["nfe"], rad["ndvr"], rad["nrad"], d(rad["xrad"]), d(rad["wrad"]), d(rad["radp"]),
                                 d(rad["radk"]), d(rad["radk0"]), float(rad["rmask"]), d(rad["mask"])) == 0
    assert lib.td1c_gpu_bind_sph(ang["lmax1"], ang["lmax2"], ang["mmax1"], ang["mmax2"], ang["nlat"], d(ang["wlat"]),
                                 d(ang["cost"]), d(ang["legf1"]), d(ang["legb1"]), d(ang["legf2"]), d(ang["legb2"])) == 0
    return keep


def _bind_bas(lib, wl, otype):
    orbs = wl["orbitals"]
    ot = np.array(otype, dtype=np.int32)
    mv = np.array([o[2] for o in orbs], dtype=np.int32)
    lv = np.array([o[1] for o in orbs], dtype=np.int32)
    rc = lib.td1c_gpu_bind_bas(float(wl["znuc"]), 1, 0, len(orbs), ot.ctypes.data_as(IP), mv.ctypes.data_as(IP),
                               lv.ctypes.data_as(IP), int(wl["nela"]), int(wl["nelb"]))
    return rc, (ot, mv, lv)


def test_frozen_core_type_minus2_refused():
    from td1c_b200 import _lib
    lib = _lib.load()
    lib.hprod_final_()  # a fresh context
    wl = W.NE_SMALL
    keep = _bind_geometry(lib, wl)
    otype = [o[3] for o in wl["orbitals"]]
    otype[0] = -2
    rc, arrs = _bind_bas(lib, wl, otype)
    assert rc == ST_CONFIG
    lib.hprod_init_()
    assert lib.td1c_gpu_last_status() & ST_CONFIG
    lib.hprod_final_()
    del keep, arrs


def test_ormas_subspaces_refused():
    from td1c_b200 import _lib
    lib = _lib.load()
    lib.hprod_final_()
    wl = W.NE_SMALL
    keep = _bind_geometry(lib, wl)
    rc, arrs = _bind_bas(lib, wl, [o[3] for o in wl["orbitals"]])
    assert rc == 0
    assert lib.td1c_gpu_bind_ormas(2) == ST_CONFIG
    lib.hprod_init_()
    assert lib.td1c_gpu_last_status() & ST_CONFIG
    lib.hprod_final_()
    assert lib.td1c_gpu_last_status() == 0  # the context is gone with its status
    del keep, arrs
