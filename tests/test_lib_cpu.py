"""CPU checks of the product side: the host table builder against the oracle,
the C-ABI library loads and exports every symbol the header declares (no
compute calls without a GPU), and the CI string layout."""
import ctypes
import os
import re

import numpy as np
import pytest

from td1c_b200 import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    src = open(os.path.join(ROOT, "include", "td1c_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(td1c_gpu_\w+|td1c_mlp_\w+|td1c_lp_\w+|hprod_\w+_|h1itr_\w+_|dpade_\w+_)\s*\(", src)))


def test_header_symbols_exported():
    from td1c_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        _lib.build()
    lib = ctypes.CDLL(_lib.LIB_PATH)
    syms = header_symbols()
    assert len(syms) >= 15
    for s in syms:
        assert hasattr(lib, s), s
    assert set(syms) == set(_lib.EXPORTED)


@pytest.mark.parametrize("wl", [W.NE_SMALL, W.HE_TDHF], ids=lambda w: w["name"])
def test_host_tables_match_oracle(wl):
    from oracle.oracle import Oracle
    from td1c_b200 import basis
    rad, ang = basis.build(wl)
    o = Oracle(wl)
    for k in ["xrad", "wrad", "mask"]:
        assert np.abs(rad[k] - o.get(k)).max() < 1e-13 * max(1.0, np.abs(o.get(k)).max())
    for k in ["radk", "radk0", "radp"]:
        ref = o.get(k)
        assert np.abs(rad[k].ravel() - ref).max() < 1e-13 * np.abs(ref).max()
    for k in ["cost", "wlat", "legf1", "legb1", "legf2", "legb2"]:
        ref = o.get(k)
        assert np.abs(np.asarray(ang[k]).ravel() - ref).max() < 1e-12 * max(1.0, np.abs(ref).max())


def test_seeded_cic_singlet_symmetric():
    from oracle.oracle import Oracle
    from .helpers import oracle_state, ci_blocks
    o = Oracle(W.NE_SMALL)
    orb, cic = oracle_state(o)
    stra, strb, detoff = o.get("stra").astype(int), o.get("strb").astype(int), o.get("detoff").astype(int)
    afirst, acount = ci_blocks(o.wl, stra, strb)
    idx = {}
    for ib in range(len(strb)):
        for p in range(acount[ib]):
            idx[(stra[afirst[ib] + p], strb[ib])] = detoff[ib] + p
    for (a, b), k in idx.items():
        assert abs(cic[k] - cic[idx[(b, a)]]) < 1e-15
    assert abs(np.linalg.norm(cic) - 1) < 1e-14
