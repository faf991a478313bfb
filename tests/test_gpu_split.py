"""GPU one-body propagators of the split schemes against the oracle.

h1itr_prop (Crank-Nicolson of the one-body Hamiltonian with correction
cycles for the laser coupling) and dpade_prod (the Pade inverse of ETD-RK2)
on the device against the oracle's banded-LU restatement, through the device
entry points and the drop-in symbols; split2 (h1itr + RK4 on the two-body
RHS), ETD-RK2 and ETD-RK4 (the rational one-body functions of clh1rat)
trajectories with their dipole traces; imaginary-time
relaxation with ETD-RK2 steps; the full-size Ne grid for the one-body step
and a stability run at the workload's dt = 0.004.  Tolerance 1e-10 relative.
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
    o.set_split(wl.get("split_type", 0))
    rad, ang = oracle_tables(o)
    h = HProd(wl, rad, ang)
    orb, cic = oracle_state(o)
    o.set_wfn0(orb, cic)
    h.set_wfn0(orb, cic)
    return o, h, orb, cic


def _strong_field(wl):
    # a field near the pulse peak, large enough that several correction cycles run
    lf = np.zeros(9)
    lf[2] = 1.5 if wl["igauge"] == 1 else 0.3
    lf[5] = 0.1
    lf[8] = lf[2]
    return lf


@pytest.mark.gpu
@pytest.mark.parametrize("split", [1, 2])
@pytest.mark.parametrize("wl", [W.MIXED_SMALL, W.LENGTH_SMALL, W.NE_SMALL], ids=lambda w: w["name"])
def test_one_body_step_parity(cuda_ok, wl, split):
    import torch
    o, h, orb, cic = _setup(dict(wl, split_type=split))
    try:
        lf = _strong_field(wl)
        for dtime in (0.005, 0.05):
            wo, no = o.h1itr_prop(lf, dtime, orb, 20, 1e-10)
            d = torch.from_numpy(orb.reshape(-1).copy()).cuda()
            ng = h.h1itr_dev(d.data_ptr(), lf, dtime, 20, 1e-10)
            wg = d.cpu().numpy()
            assert rel_err(wg, wo) < TOL, ("h1itr", dtime, rel_err(wg, wo))
            assert ng == no, (ng, no)
            if split == 1:
                assert no >= 3  # the laser coupling needs several cycles at this field
            wh = h.h1itr_host(lf, dtime, orb, 20, 1e-10, split)
            assert rel_err(wh, wg) < 1e-15

            wo, no = o.dpade_prod(lf, dtime, orb, 2.0, 20, 1e-10)
            d = torch.from_numpy(orb.reshape(-1).copy()).cuda()
            ng = h.dpade_dev(d.data_ptr(), lf, dtime, 2.0, 20, 1e-10)
            wg = d.cpu().numpy()
            assert rel_err(wg, wo) < TOL, ("dpade", dtime, rel_err(wg, wo))
            assert ng == no, (ng, no)
            wh = h.dpade_host(lf, dtime, orb, 2.0, 20, 1e-10, split)
            assert rel_err(wh, wg) < 1e-15
        # frozen-core orbitals are left unchanged
        nfc, nbas = o.dims["nfcore"], o.dims["nbas"]
        if nfc:
            assert np.array_equal(wg[: nfc * nbas], orb.reshape(-1)[: nfc * nbas])
    finally:
        h.final()


@pytest.mark.gpu
def test_one_body_step_cycle_cap(cuda_ok):
    """maxcyc caps the correction cycles (the threshold is never reached at 0)."""
    import torch
    wl = dict(W.MIXED_SMALL, split_type=1)
    o, h, orb, cic = _setup(wl)
    try:
        lf = _strong_field(wl)
        wo, no = o.h1itr_prop(lf, 0.02, orb, 4, 0.0)
        d = torch.from_numpy(orb.reshape(-1).copy()).cuda()
        ng = h.h1itr_dev(d.data_ptr(), lf, 0.02, 4, 0.0)
        assert no == 4 and ng == 4
        assert rel_err(d.cpu().numpy(), wo) < TOL
    finally:
        h.final()


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["split2", "etdrk2", "etdrk4"])
@pytest.mark.parametrize("wl", [W.NE_SMALL, W.MIXED_SMALL, W.LENGTH_SMALL, W.HE_SMALL], ids=lambda w: w["name"])
def test_split_trajectory(cuda_ok, wl, kind):
    """dt = 0.01: outside full-H RK4's stability region on these grids.  etdrk4: cletdrk4 with
    the twelve rational one-body factors of clh1rat (orders 2/2)."""
    import torch
    o, h, orb, cic = _setup(dict(wl, split_type=1))
    try:
        dt, nstep = 0.01, 8
        freq = 1239.84190 / (wl["wlen"] * 27.2113845)
        t0 = 0.3 * wl["numcyc"] * 2 * np.pi / freq
        wo, co, dip = getattr(o, kind)(orb, cic, t0, dt, nstep)
        d_orb = torch.from_numpy(orb.reshape(-1).copy()).cuda()
        d_cic = torch.from_numpy(cic.copy()).cuda()
        h.rk4_reset(None, None)
        step = {"split2": h.split2_dev, "etdrk2": h.etdrk2_dev, "etdrk4": h.etdrk4_dev}[kind]
        dip_g = []
        for s in range(nstep):
            step(d_orb.data_ptr(), d_cic.data_ptr(), t0 + s * dt, dt, 1)
            dip_g.append(h.dipole_dev(d_orb.data_ptr(), d_cic.data_ptr()))
        h.sync()
        wg, cg = d_orb.cpu().numpy(), d_cic.cpu().numpy()
        bad = np.argwhere(~np.isfinite(wg.reshape(wo.shape)))
        assert rel_err(wg, wo) < TOL, (rel_err(wg, wo), len(bad), bad[:3], bad[-3:], dip_g)
        assert rel_err(cg, co) < TOL, rel_err(cg, co)
        scale = max(1.0, np.abs(dip).max())
        assert np.abs(np.array(dip_g) - dip).max() < TOL * scale, (dip_g, dip)
        # the same steps as one multi-step call (graph replays) give the same state
        d2 = torch.from_numpy(orb.reshape(-1).copy()).cuda()
        c2 = torch.from_numpy(cic.copy()).cuda()
        step(d2.data_ptr(), c2.data_ptr(), t0, dt, nstep)
        h.sync()
        assert rel_err(d2.cpu().numpy(), wo) < TOL
        assert h.launch_count() > 0
    finally:
        h.final()


@pytest.mark.gpu
@pytest.mark.parametrize("base", [W.HE_SMALL, W.MIXED_SMALL], ids=lambda w: w["name"])
def test_relax_etdrk2(cuda_ok, base):
    """init_prop12 with ETD-RK2 steps (imaginary time, Pade one-body inverse): energy trace
    and final state against the oracle at a step 250 times the full-H RK4 one."""
    import torch
    wl = dict(base, icomp=0, split_type=1)
    o, h, orb, cic = _setup(wl)
    try:
        wo, co = o.orth(orb, cic)
        d_orb = torch.from_numpy(wo.reshape(-1).copy()).cuda()
        d_cic = torch.from_numpy(co.copy()).cuda()
        ncyc, dt = 12, 0.05
        wr, cr, eo = o.relax_etdrk2(wo, co, dt, ncyc)
        eg = h.relax_etdrk2_dev(d_orb.data_ptr(), d_cic.data_ptr(), dt, ncyc)
        assert np.all(np.diff(eo) < 0), eo
        assert np.abs(eg - eo).max() < TOL * np.abs(eo).max(), (eg, eo)
        assert rel_err(d_orb.cpu().numpy(), wr) < TOL
        assert rel_err(d_cic.cpu().numpy(), cr) < TOL
    finally:
        h.final()


@pytest.mark.gpu
def test_full_size_one_body_step(cuda_ok):
    """Ne TD-CASSCF grid (60 elements, lmax 47): h1itr and dpade at the workload's
    dt = 0.004 near peak field against the oracle; the Crank-Nicolson step keeps
    every orbital's norm (unitary up to the cycle threshold)."""
    import torch
    wl = dict(W.NE_CAS, split_type=1)
    o, h, orb, cic = _setup(wl)
    try:
        lf = _strong_field(wl)
        dt2 = 0.002  # clh1itr's half step of dt = 0.004
        wo, no = o.h1itr_prop(lf, dt2, orb, 20, 1e-10)
        d = torch.from_numpy(orb.reshape(-1).copy()).cuda()
        ng = h.h1itr_dev(d.data_ptr(), lf, dt2, 20, 1e-10)
        wg = d.cpu().numpy()
        assert rel_err(wg, wo) < TOL, rel_err(wg, wo)
        assert ng == no
        nf = len(wl["orbitals"])
        n0 = np.linalg.norm(orb.reshape(nf, -1), axis=1)
        n1 = np.linalg.norm(wg.reshape(nf, -1), axis=1)
        assert np.abs(n1 - n0).max() < 1e-9, (n0, n1)
        wo, no = o.dpade_prod(lf, 0.004, orb, 2.0, 20, 1e-10)
        d = torch.from_numpy(orb.reshape(-1).copy()).cuda()
        ng = h.dpade_dev(d.data_ptr(), lf, 0.004, 2.0, 20, 1e-10)
        assert rel_err(d.cpu().numpy(), wo) < TOL
        assert ng == no
    finally:
        h.final()


@pytest.mark.gpu
def test_full_size_split2(cuda_ok):
    """Ne TD-CASSCF at dt = 0.004 (the workload's step) at the pulse peak: two split2
    steps against the oracle, then 200 more on the device stay finite with orbital and
    CI norms near 1 (full-H RK4 diverges at this step; the split scheme's own error on
    the seeded, unrelaxed orbitals moves the norms by well under 1e-2)."""
    import torch
    wl = dict(W.NE_CAS, split_type=1)
    o, h, orb, cic = _setup(wl)
    try:
        nf = len(wl["orbitals"])
        wo, co = o.orth(orb, cic)
        freq = 1239.84190 / (wl["wlen"] * 27.2113845)
        t0 = 0.5 * wl["numcyc"] * 2 * np.pi / freq - 0.2  # around the envelope maximum
        wr, cr, dip = o.split2(wo, co, t0, 0.004, 2)
        d_orb = torch.from_numpy(wo.reshape(-1).copy()).cuda()
        d_cic = torch.from_numpy(co.copy()).cuda()
        h.rk4_reset(None, None)
        h.split2_dev(d_orb.data_ptr(), d_cic.data_ptr(), t0, 0.004, 2)
        h.sync()
        assert rel_err(d_orb.cpu().numpy(), wr) < TOL, rel_err(d_orb.cpu().numpy(), wr)
        assert rel_err(d_cic.cpu().numpy(), cr) < TOL
        h.split2_dev(d_orb.data_ptr(), d_cic.data_ptr(), t0 + 0.008, 0.004, 200)
        h.sync()
        wg = d_orb.cpu().numpy().reshape(nf, -1)
        cg = d_cic.cpu().numpy()
        assert np.all(np.isfinite(wg)) and np.all(np.isfinite(cg))
        norms = np.linalg.norm(wg, axis=1)
        assert np.abs(norms - 1.0).max() < 1e-2, norms
        assert abs(np.linalg.norm(cg) - 1.0) < 1e-2
    finally:
        h.final()


@pytest.mark.gpu
def test_full_size_split2_peak_relaxed(cuda_ok):
    """Ne TD-CASSCF from the committed relaxed state, 12 split2 steps at dt = 0.004 starting at the
    |A(t)| maximum of the pulse (the most one-body correction cycles): state and the dipole after
    every step against the oracle, 1e-10 relative."""
    import torch
    from td1c_b200.data.make_relaxed_state import load
    from oracle.oracle import Oracle
    from td1c_b200.hprod import HProd
    wl = dict(W.NE_CAS, split_type=1)
    o = Oracle(wl)
    o.set_split(1)
    rad, ang = oracle_tables(o)
    h = HProd(wl, rad, ang)
    try:
        orb, cic, info = load()
        assert info["workload"] == wl["name"]
        # set_wfn0 once (the oracle, like hprod_addfc_tmat, adds the frozen-core potential to tmat)
        o.set_wfn0(orb, cic)
        h.set_wfn0(orb, cic)
        freq = 1239.84190 / (wl["wlen"] * 27.2113845)
        period = wl["numcyc"] * 2 * np.pi / freq
        ts = np.linspace(0.3 * period, 0.7 * period, 4001)
        amp = [abs(h.pulse_lfield(t)[2]) for t in ts]
        t0 = float(ts[int(np.argmax(amp))])
        dt, nstep = 0.004, 12
        wo, co, dip = o.split2(orb, cic, t0, dt, nstep)
        d_orb = torch.from_numpy(orb.reshape(-1).copy()).cuda()
        d_cic = torch.from_numpy(cic.copy()).cuda()
        h.rk4_reset(None, None)
        dip_g = []
        for s in range(nstep):
            h.split2_dev(d_orb.data_ptr(), d_cic.data_ptr(), t0 + s * dt, dt, 1)
            dip_g.append(h.dipole_dev(d_orb.data_ptr(), d_cic.data_ptr()))
        h.sync()
        assert h.last_status() == 0
        assert rel_err(d_orb.cpu().numpy(), wo.reshape(-1)) < TOL, rel_err(d_orb.cpu().numpy(), wo.reshape(-1))
        assert rel_err(d_cic.cpu().numpy(), co) < TOL, rel_err(d_cic.cpu().numpy(), co)
        scale = max(1.0, np.abs(dip).max())
        assert np.abs(np.array(dip_g) - dip).max() < TOL * scale, (dip_g, dip)
    finally:
        h.final()
