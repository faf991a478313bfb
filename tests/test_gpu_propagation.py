"""GPU RK4 propagation (clcrk + wfn_mask) against the oracle, and full-size
RHS checks.

The trajectory test runs on the small grids with a step inside RK4's
stability region (full-H RK4 at dt = 0.004 is outside it for the FEDVR
spectrum of these grids); tolerance 1e-10 relative on the state and on the
dipole trace.  The full-size tests compare one RHS of the Ne and He
workloads with the oracle (1e-10 relative) and check size-independent
properties of the RHS.
"""
import numpy as np
import pytest

from td1c_b200 import workloads as W

from .helpers import oracle_tables, oracle_state, rel_err

TOL = 1e-10


def _setup(wl):
    from oracle.oracle import Oracle
    from td1c_b200.hprod import HProd
    o = Oracle(wl)
    rad, ang = oracle_tables(o)
    h = HProd(wl, rad, ang)
    orb, cic = oracle_state(o)
    o.set_wfn0(orb, cic)
    h.set_wfn0(orb, cic)
    return o, h, orb, cic


@pytest.mark.gpu
@pytest.mark.parametrize("wl", [W.NE_SMALL, W.MIXED_SMALL, W.HE_SMALL], ids=lambda w: w["name"])
def test_rk4_trajectory(cuda_ok, wl):
    import torch
    o, h, orb, cic = _setup(wl)
    try:
        dt, nstep = 2e-4, 12
        freq = 1239.84190 / (wl["wlen"] * 27.2113845)
        t0 = 0.3 * wl["numcyc"] * 2 * np.pi / freq
        wo, co, dip = o.rk4(orb, cic, t0, dt, nstep)
        d_orb = torch.from_numpy(orb.reshape(-1).copy()).cuda()
        d_cic = torch.from_numpy(cic.copy()).cuda()
        h.rk4_reset(None, None)
        # one step per call, so the device dipole is recorded after every step
        dip_g = []
        for s in range(nstep):
            h.rk4_dev(d_orb.data_ptr(), d_cic.data_ptr(), t0 + s * dt, dt, 1, use_graph=True)
            dip_g.append(h.dipole_dev(d_orb.data_ptr(), d_cic.data_ptr()))
        h.sync()
        wg, cg = d_orb.cpu().numpy(), d_cic.cpu().numpy()
        assert rel_err(wg, wo) < TOL, rel_err(wg, wo)
        assert rel_err(cg, co) < TOL, rel_err(cg, co)
        # dipole(t): the device observable against the oracle's trace, step by step
        scale = max(1.0, np.abs(dip).max())
        assert np.abs(np.array(dip_g) - dip).max() < TOL * scale, (dip_g, dip)
        assert h.launch_count() > 0
    finally:
        h.final()


@pytest.mark.gpu
@pytest.mark.parametrize("wl", [W.NE_CAS, W.HE_TDHF], ids=lambda w: w["name"])
def test_full_size_rhs(cuda_ok, wl):
    o, h, orb, cic = _setup(wl)
    try:
        freq = 1239.84190 / (wl["wlen"] * 27.2113845)
        lf = o.field(0.4 * wl["numcyc"] * 2 * np.pi / freq)
        hw_o, hc_o = o.htot(1.0, lf, orb, cic)
        hw_g, hc_g = h.htot(1.0, lf, orb, cic)
        assert rel_err(hw_g, hw_o) < TOL, rel_err(hw_g, hw_o)
        if o.dims["nact"]:
            assert rel_err(hc_g, hc_o) < TOL, rel_err(hc_g, hc_o)
        eo, eg = o.energies(), h.energies()
        assert abs(eo["ene_tot"] - eg["ene_tot"]) < TOL * abs(eo["ene_tot"])
        # size-independent properties at zero field: orbital norms and CI norm conserved
        hw, hc = h.htot(1.0, np.zeros(9), orb, cic)
        nf = len(wl["orbitals"])
        nfc = o.dims["nfcore"]
        hw2, o2 = hw.reshape(nf, -1), orb.reshape(nf, -1)
        if nfc:
            assert np.abs(hw2[:nfc]).max() == 0.0
        for f in range(nfc, nf):
            assert abs(np.vdot(o2[f], hw2[f]).real) < 1e-11 * np.linalg.norm(hw2[f])
        if o.dims["nact"]:
            assert abs(np.vdot(cic, hc).real) < 1e-12 * max(1.0, np.linalg.norm(hc))
    finally:
        h.final()


@pytest.mark.gpu
@pytest.mark.parametrize("base", [W.NE_SMALL, W.MIXED_SMALL, W.HE_SMALL], ids=lambda w: w["name"])
def test_relaxation_trace(cuda_ok, base):
    """Imaginary-time relaxation (icomp = 0): the device orth matches the oracle's on a
    non-orthonormal state, and 20 relaxation cycles match its energy trace and final state."""
    import torch
    wl = dict(base, icomp=0)
    o, h, orb, cic = _setup(wl)
    try:
        d_orb = torch.from_numpy(orb.reshape(-1).copy()).cuda()
        d_cic = torch.from_numpy(cic.copy()).cuda()
        h.orth_dev(d_orb.data_ptr(), d_cic.data_ptr())
        h.sync()
        wo, co = o.orth(orb, cic)
        assert rel_err(d_orb.cpu().numpy(), wo) < TOL
        assert rel_err(d_cic.cpu().numpy(), co) < TOL
        ncyc = 20
        wr, cr, eo = o.relax(wo, co, 2e-4, ncyc)
        h.rk4_reset(None, None)
        eg = h.relax_dev(d_orb.data_ptr(), d_cic.data_ptr(), 2e-4, ncyc)
        assert np.all(np.diff(eg) < 0), eg
        assert np.abs(eg - eo).max() < TOL * np.abs(eo).max(), (eg, eo)
        assert rel_err(d_orb.cpu().numpy(), wr) < TOL
        assert rel_err(d_cic.cpu().numpy(), cr) < TOL
    finally:
        h.final()
