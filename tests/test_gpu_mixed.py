"""The mixed-precision form of the RHS against the plain FP64 path on the device.

The mean field's pair-density multipoles and pair potentials on the grid run in
split TF32 on the tensor cores (FP32 accumulation); everything else stays
FP64.  One RHS: the two transformed fields deviate from FP64 by FP32-class
amounts, and so does hwfn.  A field-driven split2 trajectory: the
length-form dipole stays within 1e-5 a.u. and the CI and orbital norms (the
absorbing mask acts on the orbitals) within 1e-8 of the
FP64 trajectory (the FP64 device path itself matches the oracle to 1e-10 in
the other GPU tests).
"""
import numpy as np
import pytest

from td1c_b200 import workloads as W

from .helpers import oracle_tables, oracle_state


def _setup(base):
    from oracle.oracle import Oracle
    from td1c_b200.hprod import HProd
    wl = dict(base, split_type=1)
    o = Oracle(wl)
    o.set_split(1)
    rad, ang = oracle_tables(o)
    h = HProd(wl, rad, ang)
    orb, cic = oracle_state(o)
    o.set_wfn0(orb, cic)
    h.set_wfn0(orb, cic)
    orb, cic = o.orth(orb, cic)
    return o, h, wl, orb, cic


@pytest.mark.gpu
@pytest.mark.parametrize("base", [W.NE_SMALL, W.MIXED_SMALL], ids=lambda w: w["name"])
def test_mixed_rhs_deviation(cuda_ok, base):
    import torch
    o, h, wl, orb, cic = _setup(base)
    try:
        d_orb = torch.from_numpy(orb.reshape(-1).copy()).cuda()
        d_cic = torch.from_numpy(cic.copy()).cuda()
        dev = h.mixed_selftest(d_orb.data_ptr(), d_cic.data_ptr(), o.field(30.0))
        assert np.all(dev > 0.0), dev            # the tensor-core path ran and rounds differently
        assert dev[0] < 2e-6 and dev[1] < 2e-6, dev
        assert dev[2] < 1e-5, dev
        assert h.lib.td1c_gpu_last_status() == 0
    finally:
        h.final()


@pytest.mark.gpu
def test_mixed_trajectory_dipole_and_norm(cuda_ok):
    import torch
    o, h, wl, orb, cic = _setup(W.MIXED_SMALL)
    try:
        freq = 1239.84190 / (wl["wlen"] * 27.2113845)
        t0, dt, nseg, per = 0.4 * wl["numcyc"] * 2 * np.pi / freq, 0.004, 10, 5
        res = {}
        for mixed in (False, True):
            h.set_mixed(mixed)
            h.rk4_reset(None, None)
            d_orb = torch.from_numpy(orb.reshape(-1).copy()).cuda()
            d_cic = torch.from_numpy(cic.copy()).cuda()
            dip, norm = [], []
            for s in range(nseg):
                h.split2_dev(d_orb.data_ptr(), d_cic.data_ptr(), t0 + s * per * dt, dt, per)
                h.sync()
                dip.append(h.dipole_dev(d_orb.data_ptr(), d_cic.data_ptr()))
                norm.append([float(torch.linalg.vector_norm(d_cic).item()), float(torch.linalg.vector_norm(d_orb).item())])
            res[mixed] = (np.array(dip), np.array(norm))
        h.set_mixed(False)
        ddip = np.abs(res[True][0] - res[False][0]).max()
        dnorm = np.abs(res[True][1] - res[False][1]).max()
        assert 0.0 < ddip <= 1e-5, ddip
        assert dnorm <= 1e-8, dnorm
        assert h.lib.td1c_gpu_last_status() == 0
    finally:
        h.final()


@pytest.mark.gpu
@pytest.mark.parametrize("base", [W.NE_SMALL, W.MIXED_SMALL, W.NE_CAS], ids=lambda w: w["name"])
def test_persistent_and_per_tile_kernels_agree(cuda_ok, base):
    """The persistent split-TF32 kernel (mode 1) and the per-tile one (mode 2) give the same
    pair-density multipoles and pair potentials to FP32 rounding, both within 2e-6 of FP64; on the
    full-size Ne configuration as well (the persistent kernel's tables resident per CTA)."""
    import torch
    from td1c_b200 import basis
    from td1c_b200.hprod import HProd
    from td1c_b200.wfn import seeded_orbitals, seeded_cic
    from .helpers import rel_err
    if base is W.NE_CAS:
        wl = dict(base, split_type=1)
        rad, ang = basis.build(wl)
        h = HProd(wl, rad, ang)
        tb = h.ci_tables()
        orb = seeded_orbitals(wl, rad["xrad"], rad["wrad"], rad["mask"])
        cic = seeded_cic(wl, h.dims["lcic"], tb["stra"], tb["strb"], tb["detoff"], tb["afirst"], tb["acount"])
        h.set_wfn0(orb, cic)
        lf = h.pulse_lfield(100.0)
    else:
        o, h, wl, orb, cic = _setup(base)
        lf = o.field(30.0)
    try:
        d_orb = torch.from_numpy(orb.reshape(-1).copy()).cuda()
        d_cic = torch.from_numpy(cic.copy()).cuda()
        d_hw, d_hc = torch.empty_like(d_orb), torch.empty_like(d_cic)
        out = {}
        for mode in (0, 1, 2):
            h.set_mixed(mode)
            h.htot_dev(1.0, lf, d_orb.data_ptr(), d_cic.data_ptr(), d_hw.data_ptr(), d_hc.data_ptr())
            h.sync()
            out[mode] = (h.debug("rho2"), h.debug("W"), d_hw.cpu().numpy())
        h.set_mixed(False)
        for mode in (1, 2):
            assert rel_err(out[mode][0], out[0][0]) < 2e-6, (mode, rel_err(out[mode][0], out[0][0]))
            assert rel_err(out[mode][1], out[0][1]) < 2e-6, (mode, rel_err(out[mode][1], out[0][1]))
            assert rel_err(out[mode][2], out[0][2]) < 1e-5
        assert rel_err(out[1][0], out[2][0]) < 1e-6 and rel_err(out[1][1], out[2][1]) < 1e-6
        assert h.lib.td1c_gpu_last_status() == 0
    finally:
        h.final()


@pytest.mark.gpu
@pytest.mark.parametrize("base", [W.NE_SMALL, W.MIXED_SMALL, W.NE_CAS], ids=lambda w: w["name"])
def test_mixed_int2e_tensor_cores(cuda_ok, base):
    """Mixed mode 3's int2e in split TF32 on tcgen05: on the same pair densities and potentials it
    matches the FP64 DMMA kernel to FP32 accumulation (5e-6 of the largest integral; 1.8e-6 measured
    on the full-size Ne configuration), and the mode-3 RHS's int2e stays within 5e-6 of the FP64
    RHS's."""
    import torch
    from td1c_b200 import basis
    from td1c_b200.hprod import HProd
    from td1c_b200.wfn import seeded_orbitals, seeded_cic
    if base is W.NE_CAS:
        wl = dict(base, split_type=1)
        rad, ang = basis.build(wl)
        h = HProd(wl, rad, ang)
        tb = h.ci_tables()
        orb = seeded_orbitals(wl, rad["xrad"], rad["wrad"], rad["mask"])
        cic = seeded_cic(wl, h.dims["lcic"], tb["stra"], tb["strb"], tb["detoff"], tb["afirst"], tb["acount"])
        h.set_wfn0(orb, cic)
        lf = h.pulse_lfield(100.0)
    else:
        o, h, wl, orb, cic = _setup(base)
        lf = o.field(30.0)
    try:
        d_orb = torch.from_numpy(orb.reshape(-1).copy()).cuda()
        d_cic = torch.from_numpy(cic.copy()).cuda()
        dev = h.mixed_int2e_selftest(d_orb.data_ptr(), d_cic.data_ptr(), lf)
        assert dev is not None
        assert 0.0 < dev[0] < 5e-6, dev
        assert dev[1] < 5e-6, dev
        assert h.last_status() == 0
    finally:
        h.final()


@pytest.mark.gpu
@pytest.mark.parametrize("base", [W.NE_SMALL, W.NE_CAS], ids=lambda w: w["name"])
def test_mode3_poisson_interior_in_tf32(cuda_ok, base):
    """Mixed mode 3 also runs the condensed Poisson solve's interior products (pair density times
    the element's Poisson inverse) in split TF32: the multipole potentials v2sph of one RHS deviate
    from FP64 by FP32-class amounts (the transforms' pair densities feed them too), and hwfn stays
    within 1e-5 of FP64."""
    import torch
    from td1c_b200 import basis
    from td1c_b200.hprod import HProd
    from td1c_b200.wfn import seeded_orbitals, seeded_cic
    from .helpers import rel_err
    if base is W.NE_CAS:
        wl = dict(base, split_type=1)
        rad, ang = basis.build(wl)
        h = HProd(wl, rad, ang)
        tb = h.ci_tables()
        orb = seeded_orbitals(wl, rad["xrad"], rad["wrad"], rad["mask"])
        cic = seeded_cic(wl, h.dims["lcic"], tb["stra"], tb["strb"], tb["detoff"], tb["afirst"], tb["acount"])
        h.set_wfn0(orb, cic)
        lf = h.pulse_lfield(100.0)
    else:
        o, h, wl, orb, cic = _setup(base)
        lf = o.field(30.0)
    try:
        d_orb = torch.from_numpy(orb.reshape(-1).copy()).cuda()
        d_cic = torch.from_numpy(cic.copy()).cuda()
        d_hw, d_hc = torch.empty_like(d_orb), torch.empty_like(d_cic)
        out = {}
        for mode in (0, 1, 3):
            h.set_mixed(mode)
            h.htot_dev(1.0, lf, d_orb.data_ptr(), d_cic.data_ptr(), d_hw.data_ptr(), d_hc.data_ptr())
            h.sync()
            out[mode] = (h.debug("v2sph"), d_hw.cpu().numpy())
        h.set_mixed(False)
        d1, d3 = rel_err(out[1][0], out[0][0]), rel_err(out[3][0], out[0][0])
        assert 0.0 < d1 < 2e-6 and 0.0 < d3 < 5e-6, (d1, d3)
        assert rel_err(out[3][0], out[1][0]) > 0.0  # the TF32 interior products ran
        assert rel_err(out[3][1], out[0][1]) < 1e-5
        assert h.last_status() == 0
    finally:
        h.final()


@pytest.mark.gpu
@pytest.mark.parametrize("base", [W.NE_SMALL, W.MIXED_SMALL], ids=lambda w: w["name"])
def test_mixed_against_the_oracle(cuda_ok, base):
    """The mixed form against the oracle directly (not only against the device's FP64 path): one
    RHS (hwfn and hcic within 1e-5 relative) and 8 split2 steps at dt = 0.004 (state within 1e-5,
    the dipole after every step within 1e-5 a.u.)."""
    import torch
    from .helpers import rel_err
    o, h, wl, orb, cic = _setup(base)
    try:
        lf = o.field(30.0)
        hw_o, hc_o = o.htot(1.0, lf, orb, cic)
        d_orb = torch.from_numpy(orb.reshape(-1).copy()).cuda()
        d_cic = torch.from_numpy(cic.copy()).cuda()
        d_hw, d_hc = torch.empty_like(d_orb), torch.empty_like(d_cic)
        h.set_mixed(1)
        h.htot_dev(1.0, lf, d_orb.data_ptr(), d_cic.data_ptr(), d_hw.data_ptr(), d_hc.data_ptr())
        h.sync()
        assert rel_err(d_hw.cpu().numpy(), np.asarray(hw_o).reshape(-1)) < 1e-5
        assert rel_err(d_hc.cpu().numpy(), np.asarray(hc_o).reshape(-1)) < 1e-5
        freq = 1239.84190 / (wl["wlen"] * 27.2113845)
        t0, dt, nstep = 0.4 * wl["numcyc"] * 2 * np.pi / freq, 0.004, 8
        wo, co, dip = o.split2(orb, cic, t0, dt, nstep)
        h.rk4_reset(None, None)
        dip_g = []
        for s in range(nstep):
            h.split2_dev(d_orb.data_ptr(), d_cic.data_ptr(), t0 + s * dt, dt, 1)
            dip_g.append(h.dipole_dev(d_orb.data_ptr(), d_cic.data_ptr()))
        h.sync()
        h.set_mixed(0)
        assert rel_err(d_orb.cpu().numpy(), np.asarray(wo).reshape(-1)) < 1e-5
        assert np.abs(np.array(dip_g) - np.asarray(dip)).max() < 1e-5, (dip_g, dip)
        assert h.last_status() == 0
    finally:
        h.final()
