"""The CI determinant order and excitation signs at the boundary equal the reference's.

A CI vector crosses the drop-in boundary (hprod_htot_'s cic/hcic, the .cic
files) as a flat array, so its layout must be the reference's.  This file
restates how td1c numbers determinants and signs its excitations, and checks
the oracle's (CPU) and the library's (GPU) tables and 1-RDMs against it:

- strings of one spin are numbered by the arc weights of the string graph
  (ormas_arcwgt_spin, src/ormas/ormas_arcwgt.F90:52-105) and decoded by
  ormas_occvec (src/ormas/ormas_occvec.F90:2-30);
- ormas_madapt_str re-orders them by M, keeping the graph order within one M
  (src/ormas/ormas_madapt.F90:245-300; one distribution for CAS);
- determinants run over the M-ordered beta strings, each followed by the
  alpha strings whose M completes mtot (ormas_madapt.F90:554-569);
- the excitation a+_p a_h of a string has the sign (-1)^(occupied orbitals
  strictly between p and h) (ormas_sgn1x, src/ormas/ormas_sgn1x.F90:2-20);
- den1(p, h) = sum conj(c_I) sgn c_K over I, K = sgn a+_p a_h I, both spins
  (ormas_mkden1_ras_bb/_aa, src/ormas/ormas_mkden1_ras.F90:42-180).
The library's own layout is documented as strings sorted by (M, bit mask);
these tests show that this is the graph order within M.
"""
from itertools import combinations

import numpy as np
import pytest

from td1c_b200 import workloads as W

from .helpers import oracle_state, oracle_tables, rel_err

CASES = [W.NE_SMALL, W.MIXED_SMALL, W.LENGTH_SMALL, W.OPEN_SMALL]  # NE_SMALL carries the Ne CAS(8e,9o) orbitals


def arcwgt(nel, nact):
    """ormas_arcwgt_spin: arc weights arc[m, k] (m = 1..nact, k = 1..nel; 1-based)."""
    vtx = np.zeros((nact + 1, nel + 1), dtype=np.int64)
    vtx[0, 0] = 1
    for k in range(nel + 1):
        vtx[k, k] = 1
    for m in range(nact - nel + 1):
        vtx[m, 0] = 1
    for k in range(1, nel + 1):
        for m in range(k + 1, k + nact - nel + 1):
            vtx[m, k] = vtx[m - 1, k] + vtx[m - 1, k - 1]
    arc = np.zeros((nact + 1, nel + 1), dtype=np.int64)
    for k in range(1, nel + 1):
        for m in range(k, k + nact - nel + 1):
            arc[m, k] = vtx[m, k] - vtx[m - 1, k - 1]
    return arc


def occvec(nel, nact, istr, arc):
    """ormas_occvec: occupation (1-based orbitals) of the graph-numbered string istr (1-based)."""
    occ = [0] * (nact + 1)
    iel, rest = nel, istr - 1
    for iorb in range(nact, 0, -1):
        if iel <= 0:
            break
        if rest >= arc[iorb, iel]:
            occ[iorb] = 1
            rest -= arc[iorb, iel]
            iel -= 1
    return occ[1:]


def reference_strings(nel, mact):
    """Bit masks of one spin's strings in the reference's order: graph order, then M-ordered."""
    nact = len(mact)
    if nel == 0:
        return [0]
    arc = arcwgt(nel, nact)
    nstr = len(list(combinations(range(nact), nel)))
    masks = []
    for istr in range(1, nstr + 1):
        occ = occvec(nel, nact, istr, arc)
        assert sum(occ) == nel
        masks.append(sum(1 << a for a in range(nact) if occ[a]))
    assert len(set(masks)) == nstr  # the graph numbering is a bijection
    mval = [sum(mact[a] for a in range(nact) if (s >> a) & 1) for s in masks]
    order = [i for M in range(min(mval), max(mval) + 1) for i in range(nstr) if mval[i] == M]
    return [masks[i] for i in order]


def reference_dets(wl):
    ncore = sum(1 for o in wl["orbitals"] if o[3] <= 0)
    mact = [o[2] for o in wl["orbitals"][ncore:]]
    na, nb = wl["nela"] - ncore, wl["nelb"] - ncore
    sa, sb = reference_strings(na, mact), reference_strings(nb, mact)
    Mof = lambda s: sum(mact[a] for a in range(len(mact)) if (s >> a) & 1)  # noqa: E731
    dets = []  # (alpha mask, beta mask) in cic order
    for b in sb:
        for a in sa:
            if Mof(a) + Mof(b) == wl.get("mtot", 0):
                dets.append((a, b))
    return sa, sb, dets, mact


def sgn1x(p, h, mask):
    lo, hi = min(p, h), max(p, h)
    return -1 if bin(mask & (((1 << hi) - 1) & ~((1 << (lo + 1)) - 1))).count("1") % 2 else 1


def reference_den1(wl, cic):
    """den1(p, h) = <a+_h a_p> by the reference's excitation loops (M-conserving excitations)."""
    sa, sb, dets, mact = reference_dets(wl)
    nact = len(mact)
    index = {d: i for i, d in enumerate(dets)}
    den1 = np.zeros((nact, nact), dtype=np.complex128)  # den1[p, h] as Fortran den1(p, h)
    for i, (a, b) in enumerate(dets):
        for spin in (0, 1):
            s = a if spin == 0 else b
            for h in range(nact):
                if not (s >> h) & 1:
                    continue
                for p in range(nact):
                    if mact[p] != mact[h] or (p != h and (s >> p) & 1):
                        continue
                    t = (s & ~(1 << h)) | (1 << p)
                    k = index[(t, b) if spin == 0 else (a, t)]
                    den1[p, h] += np.conj(cic[i]) * sgn1x(p, h, s) * cic[k]
    return den1


def oracle_dets(o):
    stra = o.get("stra").astype(np.int64)
    strb = o.get("strb").astype(np.int64)
    detoff = o.get("detoff").astype(np.int64)
    from .helpers import ci_blocks
    afirst, acount = ci_blocks(o.wl, stra, strb)
    dets = []
    for ib, b in enumerate(strb):
        assert acount[ib] == 0 or detoff[ib] == len(dets)  # a beta string without alpha partners holds no determinant
        for p in range(acount[ib]):
            dets.append((int(stra[afirst[ib] + p]), int(b)))
    return [int(x) for x in stra], [int(x) for x in strb], dets


@pytest.mark.parametrize("wl", CASES, ids=lambda w: w["name"])
def test_oracle_ci_order_is_the_reference_order(wl):
    from oracle.oracle import Oracle
    o = Oracle(wl)
    sa, sb, dets, _ = reference_dets(wl)
    osa, osb, odets = oracle_dets(o)
    assert osa == sa and osb == sb
    assert odets == dets
    assert o.dims["lcic"] == len(dets)


@pytest.mark.parametrize("wl", CASES, ids=lambda w: w["name"])
def test_oracle_den1_follows_reference_signs(wl):
    from oracle.oracle import Oracle
    o = Oracle(wl)
    orb, cic = oracle_state(o)
    o.set_wfn0(orb, cic)
    o.htot(1.0, np.zeros(9), orb, cic)
    nact = o.dims["nact"]
    got = o.get("den1", complex_=True).reshape(nact, nact)  # oracle layout den1[j][i] = Fortran den1(i, j)
    ref = reference_den1(wl, cic)
    assert rel_err(got.T, ref) < 1e-13


def test_graph_order_is_mask_order_within_m():
    """For one subspace the arc-weight numbering is the colexicographic rank, i.e. ascending mask."""
    for nact in range(1, 10):
        for nel in range(0, nact + 1):
            if nel == 0:
                continue
            arc = arcwgt(nel, nact)
            n = len(list(combinations(range(nact), nel)))
            masks = []
            for istr in range(1, n + 1):
                occ = occvec(nel, nact, istr, arc)
                masks.append(sum(1 << a for a in range(nact) if occ[a]))
            assert masks == sorted(masks)


@pytest.mark.gpu
@pytest.mark.parametrize("wl", CASES, ids=lambda w: w["name"])
def test_library_ci_tables_and_den1(cuda_ok, wl):
    from oracle.oracle import Oracle
    from td1c_b200.hprod import HProd
    o = Oracle(wl)
    rad, ang = oracle_tables(o)
    h = HProd(wl, rad, ang)
    try:
        sa, sb, dets, _ = reference_dets(wl)
        tb = h.ci_tables()
        assert [int(x) for x in tb["stra"]] == sa and [int(x) for x in tb["strb"]] == sb
        ldets = []
        for ib, b in enumerate(tb["strb"]):
            assert tb["acount"][ib] == 0 or tb["detoff"][ib] == len(ldets)
            for p in range(tb["acount"][ib]):
                ldets.append((int(tb["stra"][tb["afirst"][ib] + p]), int(b)))
        assert ldets == dets
        orb, cic = oracle_state(o)
        h.set_wfn0(orb, cic)
        h.htot(1.0, np.zeros(9), orb, cic)
        nact = h.dims["nact"]
        got = h.debug("den1").reshape(nact, nact)
        assert rel_err(got.T, reference_den1(wl, cic)) < 1e-12
    finally:
        h.final()
