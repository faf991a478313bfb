"""The three forms of hprod_dipole on the device against the oracle.

Length, velocity and acceleration forms (hprod_dipole.F90:2-146) at several
points of a field-driven split2 trajectory on the device, within 1e-10 of the
oracle's restatement: states without frozen-core orbitals (He, one and two
orbitals) and with them (C with a frozen 1s, dynamic 2s and a 2s2p active
space, in both gauges), where the velocity and acceleration forms carry the
generalized-Fock corrections (hprod_gfock, hprod_projfc).  The drop-in
hprod_dipole_ (host buffers) gives the same numbers.
"""
import numpy as np
import pytest

from td1c_b200 import workloads as W

from .helpers import oracle_tables, oracle_state


@pytest.mark.gpu
@pytest.mark.parametrize("base", [W.HE_SMALL, W.HE_TDHF, W.MIXED_SMALL, W.LENGTH_SMALL], ids=lambda w: w["name"])
def test_dipole_forms_match_oracle(cuda_ok, base):
    import torch
    from oracle.oracle import Oracle
    from td1c_b200.hprod import HProd
    wl = dict(base, split_type=1)
    o = Oracle(wl)
    o.set_split(1)
    rad, ang = oracle_tables(o)
    h = HProd(wl, rad, ang)
    try:
        orb, cic = oracle_state(o)
        o.set_wfn0(orb, cic)
        h.set_wfn0(orb, cic)
        orb, cic = o.orth(orb, cic)
        freq = 1239.84190 / (wl["wlen"] * 27.2113845)
        t0, dt = 0.5 * wl["numcyc"] * 2 * np.pi / freq, 0.004
        d_orb = torch.from_numpy(orb.reshape(-1).copy()).cuda()
        d_cic = torch.from_numpy(cic.copy()).cuda()
        h.rk4_reset(None, None)
        for s in range(3):
            t = t0 + 2 * s * dt
            lf = o.field(t)
            g = h.dipole3_dev(d_orb.data_ptr(), d_cic.data_ptr(), lf)
            ref = o.dipole3(d_orb.cpu().numpy().reshape(orb.shape), d_cic.cpu().numpy(), lf)
            for gv, rv in zip(g, ref):
                scale = max(1e-3, np.abs(rv).max())
                assert np.abs(gv - rv).max() < 1e-10 * scale, (s, g, ref)
            assert g[1][2] != 0.0 and g[2][2] != 0.0
            assert (g[1][1] != 0.0 and g[2][1] != 0.0) == (o.dims["nfcore"] > 0)
            h.split2_dev(d_orb.data_ptr(), d_cic.data_ptr(), t, dt, 2)
            h.sync()
    finally:
        h.final()


def _host_dipole(h, orb, cic, lf):
    import ctypes
    dp = ctypes.POINTER(ctypes.c_double)
    o = np.ascontiguousarray(orb, dtype=np.complex128).reshape(-1)
    c = np.ascontiguousarray(cic, dtype=np.complex128)
    lf = np.ascontiguousarray(lf, dtype=np.float64)
    dip, vel, acc = np.zeros(3), np.zeros(3), np.zeros(3)
    h.lib.hprod_dipole_(*(a.ctypes.data_as(dp) for a in (lf, o.view(np.float64), c.view(np.float64), dip, vel, acc)))
    return dip, vel, acc


@pytest.mark.gpu
def test_hprod_dipole_dropin(cuda_ok):
    from oracle.oracle import Oracle
    from td1c_b200.hprod import HProd
    # without frozen core: all three forms, as td1c_gpu_dipole3 and the oracle
    wl = dict(W.HE_SMALL, split_type=1)
    o = Oracle(wl)
    rad, ang = oracle_tables(o)
    h = HProd(wl, rad, ang)
    try:
        orb, cic = oracle_state(o)
        o.set_wfn0(orb, cic)
        h.set_wfn0(orb, cic)
        lf = o.field(30.0)
        got = _host_dipole(h, orb, cic, lf)
        ref = o.dipole3(orb, cic, lf)
        for gv, rv in zip(got, ref):
            assert np.abs(gv - rv).max() < 1e-10 * max(1e-3, np.abs(rv).max()), (got, ref)
        assert h.lib.td1c_gpu_last_status() == 0
    finally:
        h.final()
    # with a frozen core: all three forms with their generalized-Fock corrections
    wl = dict(W.MIXED_SMALL, split_type=1)
    o = Oracle(wl)
    rad, ang = oracle_tables(o)
    h = HProd(wl, rad, ang)
    try:
        orb, cic = oracle_state(o)
        o.set_wfn0(orb, cic)
        h.set_wfn0(orb, cic)
        lf = o.field(30.0)
        got = _host_dipole(h, orb, cic, lf)
        ref = o.dipole3(orb, cic, lf)
        for gv, rv in zip(got, ref):
            assert np.abs(gv - rv).max() < 1e-10 * max(1e-3, np.abs(rv).max()), (got, ref)
        assert got[1][1] != 0.0 and h.lib.td1c_gpu_last_status() == 0
    finally:
        h.final()
