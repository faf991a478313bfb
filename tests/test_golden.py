"""Oracle and GPU path against the committed fixtures (tests/golden)."""
import os

import numpy as np
import pytest

from td1c_b200 import workloads as W

from .helpers import oracle_tables, rel_err

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = [W.NE_SMALL, W.MIXED_SMALL, W.LENGTH_SMALL, W.OPEN_SMALL, W.HE_SMALL]


def load(wl):
    return dict(np.load(os.path.join(HERE, wl["name"] + ".npz")))


@pytest.mark.parametrize("wl", CASES, ids=lambda w: w["name"])
def test_oracle_reproduces_fixture(wl):
    from oracle.oracle import Oracle
    g = load(wl)
    o = Oracle(wl)
    o.set_wfn0(g["orb"], g["cic"])
    for k in range(2):
        hw, hc = o.htot(1.0, g["lfield%d" % k], g["orb"], g["cic"])
        assert rel_err(hw, g["hwfn%d" % k]) < 1e-12
        assert rel_err(hc, g["hcic%d" % k]) < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("wl", CASES, ids=lambda w: w["name"])
def test_gpu_matches_fixture(cuda_ok, wl):
    from oracle.oracle import Oracle
    from td1c_b200.hprod import HProd
    g = load(wl)
    rad, ang = oracle_tables(Oracle(wl))
    h = HProd(wl, rad, ang)
    try:
        h.set_wfn0(g["orb"], g["cic"])
        for k in range(2):
            hw, hc = h.htot(1.0, g["lfield%d" % k], g["orb"], g["cic"])
            assert rel_err(hw, g["hwfn%d" % k]) < 1e-10
            assert rel_err(hc, g["hcic%d" % k]) < 1e-10
            e = h.energies()
            ref = g["ene%d" % k]
            got = np.array([e["ene_fcore"], e["ene_dcore"], e["ene_core"], e["ene_act"], e["ene_tot"]])
            assert np.abs(got - ref).max() < 1e-10 * max(1.0, np.abs(ref).max())
    finally:
        h.final()
