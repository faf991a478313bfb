"""Failure detection on the device, without a GPU fault.

- A NaN in the orbitals a host passes to hprod_htot_ comes back as
  ST_NONFINITE (4) in td1c_gpu_last_status(); the reference would carry the
  NaN on or stop in a solver (src/hprod/hprod_mkv2mf.F90:167-170).
- The bounded wait that the staged kernels use on their mbarriers runs out on
  a barrier that nothing arrives on and reports ST_TIMEOUT (32); no copy or
  tensor-core operation is in flight, and the context stays usable: the next
  RHS still matches the oracle to 1e-10.
"""
import numpy as np
import pytest

from td1c_b200 import workloads as W

from .helpers import oracle_tables, oracle_state, rel_err

ST_NONFINITE, ST_TIMEOUT = 4, 32


@pytest.mark.gpu
def test_nan_input_reports_nonfinite(cuda_ok):
    from oracle.oracle import Oracle
    from td1c_b200.hprod import HProd
    o = Oracle(W.NE_SMALL)
    rad, ang = oracle_tables(o)
    h = HProd(W.NE_SMALL, rad, ang)
    try:
        orb, cic = oracle_state(o)
        h.set_wfn0(orb, cic)
        lf = o.field(20.0)
        h.htot(1.0, lf, orb, cic)  # clean input: no status
        assert h.last_status() == 0
        bad = orb.copy()
        bad.reshape(-1)[bad.size // 2] = np.nan
        h.lib.hprod_htot_  # the drop-in symbol itself
        import ctypes
        dp = ctypes.POINTER(ctypes.c_double)
        hw = np.zeros_like(bad)
        hc = np.zeros_like(cic)
        dt = ctypes.c_double(1.0)
        h.lib.hprod_htot_(ctypes.byref(dt), lf.ctypes.data_as(dp), bad.view(np.float64).ctypes.data_as(dp),
                          cic.view(np.float64).ctypes.data_as(dp), hw.view(np.float64).ctypes.data_as(dp),
                          hc.view(np.float64).ctypes.data_as(dp))
        assert h.last_status() & ST_NONFINITE
    finally:
        h.final()


@pytest.mark.gpu
def test_bounded_wait_times_out_and_context_survives(cuda_ok):
    from oracle.oracle import Oracle
    from td1c_b200.hprod import HProd
    o = Oracle(W.NE_SMALL)
    rad, ang = oracle_tables(o)
    h = HProd(W.NE_SMALL, rad, ang)
    try:
        orb, cic = oracle_state(o)
        o.set_wfn0(orb, cic)
        h.set_wfn0(orb, cic)
        assert h.wait_selftest() == ST_TIMEOUT
        lf = o.field(40.0)
        hw_o, hc_o = o.htot(1.0, lf, orb, cic)
        hw_g, hc_g = h.htot(1.0, lf, orb, cic)
        assert rel_err(hw_g, hw_o) < 1e-10 and rel_err(hc_g, hc_o) < 1e-10
        assert h.last_status() == 0
    finally:
        h.final()
