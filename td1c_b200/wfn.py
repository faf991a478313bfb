"""Seeded initial states (host set-up, numpy).

td1c reads its initial orbitals from a card/file guess (guess.cpp:6-60) and
has no random guess; the workloads here start from a seeded one instead:
a Philox stream gives complex Gaussian coefficients of a few smooth radial
functions r^(l+1) exp(-zeta r) per orbital, the result is masked and
Gram-Schmidt orthonormalised within each m (wfn_orth.F90:31-100 restated),
and the CI vector gets seeded complex Gaussian entries, made singlet-symmetric
(c(Ia,Ib) = c(Ib,Ia)) when nela = nelb and smul = 1, and normalised.
"""
import numpy as np


def orbital_layout(wl):
    orbs = wl["orbitals"]
    nrad = wl["ndvr"] * wl["nfe"]
    return nrad - 1, wl["lmax1"] + 1, len(orbs)


def seeded_orbitals(wl, xrad, wrad, mask, seed=None):
    """orb(1:nrad-1, 0:lmax1, 1:nfun) as a complex128 array of shape
    (nfun, lmax1+1, nrad-1) (C order == Fortran column-major orb)."""
    seed = wl.get("seed", 0) if seed is None else seed
    rng = np.random.Generator(np.random.Philox(seed))
    Nr, L1, nfun = orbital_layout(wl)
    r = np.asarray(xrad[1:Nr + 1])
    sw = np.sqrt(np.asarray(wrad[1:Nr + 1]))
    mk = np.asarray(mask[1:Nr + 1])
    orb = np.zeros((nfun, L1, Nr), dtype=np.complex128)
    z = wl["znuc"]
    for f, (n, l, m, _t) in enumerate(wl["orbitals"]):
        g = rng.standard_normal(4) + 1j * rng.standard_normal(4)
        zetas = z / n * np.array([1.0, 0.75, 0.5, 0.35])
        rad = np.zeros(Nr, dtype=np.complex128)
        for k in range(4):
            rad += g[k] * r ** (l + 1) * np.exp(-zetas[k] * r)
        # a weak admixture of l+1 keeps every l-channel of the path busy
        orb[f, l, :] = rad * sw
        if l + 1 < L1:
            g2 = rng.standard_normal() + 1j * rng.standard_normal()
            orb[f, l + 1, :] = 0.05 * g2 * r ** (l + 2) * np.exp(-zetas[0] * r) * sw
        orb[f] *= mk[None, :]
    # Gram-Schmidt within each m, in orbital order
    mval = [o[2] for o in wl["orbitals"]]
    for f in range(nfun):
        v = orb[f].reshape(-1)
        for g_ in range(f):
            if mval[g_] != mval[f]:
                continue
            u = orb[g_].reshape(-1)
            v = v - u * np.vdot(u, v)
        v = v / np.sqrt(np.vdot(v, v).real)
        orb[f] = v.reshape(L1, Nr)
    return orb


def seeded_cic(wl, lcic, stra=None, strb=None, detoff=None, afirst=None, acount=None, seed=None):
    """Seeded normalised CI vector; singlet-symmetric when the string tables
    are given and nela == nelb, smul == 1."""
    seed = (wl.get("seed", 0) if seed is None else seed) + 1000
    rng = np.random.Generator(np.random.Philox(seed))
    c = rng.standard_normal(lcic) + 1j * rng.standard_normal(lcic)
    if lcic == 1:
        return np.ones(1, dtype=np.complex128)
    if stra is not None and wl["nela"] == wl["nelb"] and wl.get("smul", 1) == 1:
        # symmetrise c(Ia, Ib) <- (c(Ia, Ib) + c(Ib, Ia)) / 2
        idx = {}
        for ib in range(len(strb)):
            if detoff[ib] < 0:
                continue
            for p in range(acount[ib]):
                idx[(int(stra[afirst[ib] + p]), int(strb[ib]))] = detoff[ib] + p
        s = c.copy()
        for (a, b), k in idx.items():
            s[k] = 0.5 * (c[k] + c[idx[(b, a)]])
        c = s
    return c / np.linalg.norm(c)


def velocity_gauge_phase(wl, orb, rad, ang, A):
    """The non-frozen orbitals times exp(-i A r cos(theta)): a length-gauge state
    expressed in the velocity gauge at vector potential A (the phase the RHS
    gives the frozen core, hprod_orbin.F90:68-105).  orb has shape
    (nfun, lmax1+1, nrad-1); returns a new array.  The product is formed on the
    Gauss-Legendre theta grid and projected back onto l <= lmax1."""
    orbs = wl["orbitals"]
    nfun = len(orbs)
    L1, nlat, mmax1 = ang["lmax1"] + 1, ang["nlat"], ang["mmax1"]
    Nr = orb.shape[-1]
    lf1 = np.asarray(ang["legf1"]).reshape(2 * mmax1 + 1, nlat, L1)
    lb1 = np.asarray(ang["legb1"]).reshape(2 * mmax1 + 1, L1, nlat)
    r = np.asarray(rad["xrad"])[1:Nr + 1]
    ph = np.exp(-1j * A * np.outer(np.asarray(ang["cost"]), r))
    out = np.array(orb, dtype=np.complex128, copy=True).reshape(nfun, L1, Nr)
    for f, (_n, _l, m, typ) in enumerate(orbs):
        if typ == -1:
            continue
        g = lf1[m + mmax1] @ out[f]
        out[f] = lb1[m + mmax1] @ (g * ph)
    return out
