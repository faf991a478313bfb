"""GPU parity of the RHS (hprod_htot) against the CPU oracle, through the C-ABI.

Tolerance: the plain FP64 path must match the oracle to <= 1e-10 relative
(max-norm of the difference over max-norm of the oracle value) in hwfn,
hcic and every intermediate checked, on seeded inputs.
"""
import numpy as np
import pytest

from td1c_b200 import workloads as W

from .helpers import oracle_tables, oracle_state, rel_err

TOL = 1e-10
SMALL = [W.HE_SMALL, W.NE_SMALL, W.MIXED_SMALL, W.LENGTH_SMALL, W.OPEN_SMALL]


def _pair(wl):
    from oracle.oracle import Oracle
    from td1c_b200.hprod import HProd
    o = Oracle(wl)
    rad, ang = oracle_tables(o)
    h = HProd(wl, rad, ang)
    assert h.dims["lcic"] == o.dims["lcic"]
    if o.dims["nact"]:
        t = h.ci_tables()
        assert np.array_equal(t["stra"].astype(np.int64), o.get("stra").astype(np.int64))
        assert np.array_equal(t["strb"].astype(np.int64), o.get("strb").astype(np.int64))
        assert np.array_equal(t["detoff"].astype(np.int64), o.get("detoff").astype(np.int64))
    orb, cic = oracle_state(o)
    o.set_wfn0(orb, cic)
    h.set_wfn0(orb, cic)
    return o, h, orb, cic


@pytest.mark.gpu
@pytest.mark.parametrize("wl", SMALL, ids=[w["name"] for w in SMALL])
def test_htot_parity_small(cuda_ok, wl):
    o, h, orb, cic = _pair(wl)
    try:
        for t in (0.0, 37.0, 61.5):
            lf = o.field(t)
            hw_o, hc_o = o.htot(1.0, lf, orb, cic)
            hw_g, hc_g = h.htot(1.0, lf, orb, cic)
            assert rel_err(hw_g, hw_o) < TOL, (t, rel_err(hw_g, hw_o))
            if o.dims["nact"]:
                assert rel_err(hc_g, hc_o) < TOL, (t, rel_err(hc_g, hc_o))
            eo, eg = o.energies(), h.energies()
            for k in eo:
                assert abs(eo[k] - eg[k]) <= TOL * max(1.0, abs(eo[k])), (k, eo[k], eg[k])
    finally:
        h.final()


@pytest.mark.gpu
def test_intermediates_ne_small(cuda_ok):
    o, h, orb, cic = _pair(W.NE_SMALL)
    try:
        lf = o.field(40.0)
        o.htot(1.0, lf, orb, cic)
        h.htot(1.0, lf, orb, cic)
        for name in ["orbg", "h0orb", "h1orb", "gorb", "v2orb", "den1", "den2", "int1e", "int2e", "xmat"]:
            a, b = h.debug(name), o.get(name, True)
            if name == "orbg":
                b = b[: a.size]
            assert rel_err(a, b) < TOL, (name, rel_err(a, b))
    finally:
        h.final()
