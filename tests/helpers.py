"""Shared helpers of the test suite: oracle-driven set-up of both paths.

The parity tests bind the oracle's base tables (grid, weights, kinetic bands,
Legendre tables) into the CUDA library, so a difference in the RHS isolates
the device kernels; the host-side table builder of the package is checked
against the oracle separately.
"""
import numpy as np

from oracle.oracle import Oracle
from td1c_b200.wfn import seeded_orbitals, seeded_cic


def oracle_tables(o):
    d = o.dims
    nd, nrad = d["ndvr"], d["nrad"]
    rad = dict(nrad=nrad, ndvr=nd, nfe=nrad // nd, xrad=o.get("xrad"), wrad=o.get("wrad"), mask=o.get("mask"),
               radk=o.get("radk"), radk0=o.get("radk0"), radp=o.get("radp"), rmask=o.wl["rmask"])
    mmax1 = max(abs(x[2]) for x in o.wl["orbitals"])
    ang = dict(lmax1=d["lmax1"], lmax2=d["lmax2"], mmax1=mmax1, mmax2=2 * mmax1, nlat=d["nlat"],
               cost=o.get("cost"), wlat=o.get("wlat"), legf1=o.get("legf1"), legb1=o.get("legb1"),
               legf2=o.get("legf2"), legb2=o.get("legb2"))
    return rad, ang


def oracle_state(o, seed=None):
    d = o.dims
    orb = seeded_orbitals(o.wl, o.get("xrad"), o.get("wrad"), o.get("mask"), seed=seed)
    if d["nact"] > 0:
        stra, strb, detoff = o.get("stra").astype(np.int64), o.get("strb").astype(np.int64), o.get("detoff").astype(np.int64)
        # afirst / acount from the oracle's layout (alpha strings of matching M, contiguous)
        afirst, acount = ci_blocks(o.wl, stra, strb)
        cic = seeded_cic(o.wl, d["lcic"], stra, strb, detoff, afirst, acount, seed=seed)
    else:
        cic = np.ones(1, dtype=np.complex128)
    return orb, cic


def ci_blocks(wl, stra, strb):
    ncore = sum(1 for x in wl["orbitals"] if x[3] <= 0)
    mact = [x[2] for x in wl["orbitals"][ncore:]]

    def M(s):
        return sum(mact[a] for a in range(len(mact)) if (int(s) >> a) & 1)

    Ma = [M(s) for s in stra]
    afirst, acount = [], []
    for sb in strb:
        need = wl.get("mtot", 0) - M(sb)
        idx = [i for i, m in enumerate(Ma) if m == need]
        afirst.append(idx[0] if idx else 0)
        acount.append(len(idx))
    return np.array(afirst), np.array(acount)


def rel_err(a, b):
    a = np.asarray(a).ravel()
    b = np.asarray(b).ravel()
    if b.size == 0:
        return 0.0
    den = np.abs(b).max()
    if den == 0:
        return float(np.abs(a).max())
    return float(np.abs(a - b).max() / den)
