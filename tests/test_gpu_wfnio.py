"""A device-propagated state through the reference's .orb / .cic files and back.

Two split2 steps on the device, the state written as td1c's .orb/.cic text,
read back, uploaded and propagated two more steps: the result agrees with
four uninterrupted steps within 1e-10 relative (the files carry 16
significant digits, so the restart differs from the uninterrupted run by
rounding only).
"""
import numpy as np
import pytest

from td1c_b200 import workloads as W
from td1c_b200 import wfnio

from .helpers import oracle_tables, oracle_state, rel_err

TOL = 1e-10


@pytest.mark.gpu
def test_restart_through_orb_cic_files(cuda_ok, tmp_path):
    import torch
    from oracle.oracle import Oracle
    from td1c_b200.hprod import HProd
    wl = dict(W.MIXED_SMALL, split_type=1)
    o = Oracle(wl)
    o.set_split(1)
    rad, ang = oracle_tables(o)
    h = HProd(wl, rad, ang)
    try:
        orb, cic = oracle_state(o)
        h.set_wfn0(orb, cic)
        orb, cic = o.orth(orb, cic)
        nrad, lmax1, nfun = o.dims["nrad"], o.dims["lmax1"], len(wl["orbitals"])
        mmax1 = max(abs(x[2]) for x in wl["orbitals"])
        dt, t0 = 0.01, 0.0
        h.rk4_reset(None, None)
        # four uninterrupted steps
        d_orb = torch.from_numpy(orb.reshape(-1).copy()).cuda()
        d_cic = torch.from_numpy(cic.copy()).cuda()
        h.split2_dev(d_orb.data_ptr(), d_cic.data_ptr(), t0, dt, 4)
        h.sync()
        ref_orb, ref_cic = d_orb.cpu().numpy(), d_cic.cpu().numpy()
        # two steps, files, two more
        d_orb = torch.from_numpy(orb.reshape(-1).copy()).cuda()
        d_cic = torch.from_numpy(cic.copy()).cuda()
        h.split2_dev(d_orb.data_ptr(), d_cic.data_ptr(), t0, dt, 2)
        h.sync()
        po, pc = tmp_path / "mid.orb", tmp_path / "mid.cic"
        wfnio.write_wfn(po, pc, d_orb.cpu().numpy(), d_cic.cpu().numpy(), nrad, lmax1, mmax1)
        r_orb, r_cic = wfnio.read_wfn(po, pc, nrad, lmax1, nfun, cic.size)
        assert r_cic is not None
        d_orb = torch.from_numpy(r_orb.reshape(-1).copy()).cuda()
        d_cic = torch.from_numpy(r_cic.copy()).cuda()
        h.split2_dev(d_orb.data_ptr(), d_cic.data_ptr(), t0 + 2 * dt, dt, 2)
        h.sync()
        assert rel_err(d_orb.cpu().numpy(), ref_orb) < TOL, rel_err(d_orb.cpu().numpy(), ref_orb)
        assert rel_err(d_cic.cpu().numpy(), ref_cic) < TOL
    finally:
        h.final()
