"""td1c_gpu_int2e_static: MO two-electron integrals without any GPU allocation.

Some callers cannot let a library call cudaMalloc: a host whose GPU memory
belongs to its own pool allocator, a real-time loop that must not stall on
(or fail in) an allocation, a framework that lends only its own buffers.
td1c_gpu_int2e_static serves them with its scratch in a fixed 8 MiB device
array built into the library.

The test gives it the active-pair densities and potentials that hprod_htot_
formed, and checks its output against the int2e that hprod_htot_ computed
with its own allocated scratch (read back with td1c_gpu_debug_get). It does
this on two calls in a row, so the second call meets the array as the first
left it. The tolerance is 1e-10 relative, the parity tolerance of the other
GPU tests. The output buffer is filled with NaN before each call, to show
that the call writes every entry, and checks that the second call leaves the
device's free memory unchanged. The file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest

from td1c_b200 import workloads as W

from .helpers import oracle_tables, oracle_state, rel_err

TOL = 1e-10
ST_CONFIG = 16


def _ctx_pair_index(a, b, nfcore, nfun):
    """Index of the stored pair (a, b), a >= b, both dynamic, in the RHS's own pair list."""
    return sum(nfun - x for x in range(nfcore, b)) + (a - b)


def _run(lib, nact, mval, K, d_rho, d_v2, d_out, stream):
    m = (ctypes.c_int * len(mval))(*mval)
    return lib.td1c_gpu_int2e_static(nact, m, K, ctypes.c_void_p(d_rho), ctypes.c_void_p(d_v2),
                                     ctypes.c_void_p(d_out), ctypes.c_void_p(stream))


@pytest.mark.gpu
@pytest.mark.parametrize("wl", [W.NE_SMALL, W.MIXED_SMALL], ids=lambda w: w["name"])
def test_int2e_static_matches_htot(cuda_ok, wl):
    import torch
    from oracle.oracle import Oracle
    from td1c_b200 import _lib
    from td1c_b200.hprod import HProd

    o = Oracle(wl)
    rad, ang = oracle_tables(o)
    h = HProd(wl, rad, ang)
    try:
        orb, cic = oracle_state(o)
        h.set_wfn0(orb, cic)
        h.htot(1.0, o.field(37.0), orb, cic)
        d = h.dims
        nfun = len(wl["orbitals"])
        nfcore, ncore, nact, K = d["nfcore"], d["ncore"], d["nact"], d["nbas2"]
        mval = [x[2] for x in wl["orbitals"][ncore:]]
        rho2 = h.debug("rho2").reshape(-1, K)
        v2sph = h.debug("v2sph").reshape(-1, K)
        ref = h.debug("int2e")
        # active pairs (a >= b) in the packed order the entry point takes
        idx = [_ctx_pair_index(ncore + a, ncore + b, nfcore, nfun) for b in range(nact) for a in range(b, nact)]
        dev = torch.device("cuda:0")
        t_rho = torch.from_numpy(np.ascontiguousarray(rho2[idx]).view(np.float64)).to(dev)
        t_v2 = torch.from_numpy(np.ascontiguousarray(v2sph[idx]).view(np.float64)).to(dev)
        t_out = torch.empty(2 * nact ** 4, dtype=torch.float64, device=dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        lib = _lib.load()
        results = []
        for call in range(2):
            t_out.fill_(float("nan"))
            torch.cuda.synchronize()
            free0 = torch.cuda.mem_get_info(dev)[0]
            rc = _run(lib, nact, mval, K, t_rho.data_ptr(), t_v2.data_ptr(), t_out.data_ptr(), stream)
            assert rc == 0, (call, rc)
            torch.cuda.synchronize()
            if call == 1:
                # the first call may have had CUDA load the module (and with it the array); the
                # second reserves nothing: the device's free memory is unchanged
                assert torch.cuda.mem_get_info(dev)[0] == free0
            got = t_out.cpu().numpy().view(np.complex128)
            assert np.isfinite(got).all(), call
            assert rel_err(got, ref) < TOL, (call, rel_err(got, ref))
            results.append(got)
        assert np.array_equal(results[0], results[1])
    finally:
        h.final()


@pytest.mark.gpu
def test_int2e_static_rejects_oversize(cuda_ok):
    import torch
    from td1c_b200 import _lib

    lib = _lib.load()
    t = torch.zeros(2, dtype=torch.float64, device="cuda:0")
    p = t.data_ptr()
    # more active orbitals than the fixed scratch is sized for
    assert _run(lib, 17, [0] * 17, 1, p, p, p, 0) == ST_CONFIG
    # empty basis and null buffers
    assert _run(lib, 1, [0], 0, p, p, p, 0) == ST_CONFIG
    assert _run(lib, 1, [0], 1, p, p, 0, 0) == ST_CONFIG
