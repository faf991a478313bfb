"""Host-side grid and table set-up (numpy), mirroring td1c's C++ host layer.

This is what td1c's clbas::gen does before any hprod call (clbas.cpp:52-171):
the FEDVR radial grid of clfedvr/cldvr and the Gauss-Legendre theta grid with
the normalised associated Legendre tables of clsph/sph_gen.  The results are
handed to the device library through its td1c_gpu_bind_* entry points, the
way td1c binds them to its Fortran side with bas_rad_bind_/bas_sph_bind_.

Array conventions follow the reference exactly (indices 0..nrad for the radial
arrays, band arrays (2*ndvr+1) x (nrad+1) with the band index fastest, Legendre
tables legf1(0:lmax1, 1:nlat, -mmax1:mmax1) etc. flattened in Fortran order).
"""
import numpy as np


def lobatto(n):
    """Gauss-Lobatto nodes and weights on [-1, 1] (cldvr.cpp:82-158): the
    interior nodes are the eigenvalues of the symmetric tridiagonal matrix
    with off-diagonal sqrt(a_m b_m), a_m = (m+1)/(2m+1), b_m = (m-1)/(2m-1)."""
    x = np.zeros(n + 1)
    x[0], x[n] = -1.0, 1.0
    nled = n - 1
    if n > 1:
        A = np.zeros((nled, nled))
        for m in range(2, nled + 1):
            a = (m + 1.0) / (2.0 * m + 1.0)
            b = (m - 1.0) / (2.0 * m - 1.0)
            A[m - 2, m - 1] = A[m - 1, m - 2] = np.sqrt(a * b)
        x[1:n] = np.linalg.eigvalsh(A)
    scale = 2.0 / (n * (n + 1.0))
    w = np.full(n + 1, scale)
    for k in range(1, n):
        xa = np.longdouble(abs(x[k]))
        p0, p1 = np.longdouble(1), xa
        for kk in range(2, n + 1):
            p0, p1 = p1, ((2 * kk - 1) * xa * p1 - (kk - 1) * p0) / kk
        w[k] = float(scale / (p1 * p1))
    return x, w


def fedvr(rmin, rmax, ndvr, nfe, rmask, mask_cos_order):
    """One uniform FEDVR segment "grid: rmin rmax ndvr nfe" (clfedvr.cpp:253-338,
    361-398, 676-793).  Returns dict of xrad, wrad, mask (0..nrad) and the band
    matrices radk, radk0, radp of shape (nrad+1, 2 ndvr + 1)."""
    nd = ndvr
    nrad = nd * nfe
    x01, w01 = lobatto(nd)
    dfe = (rmax - rmin) / nfe
    bw = 2 * nd + 1
    xrad = np.zeros(nrad + 1)
    wrad = np.zeros(nrad + 1)
    xe = np.zeros((nfe, nd + 1))
    we = np.zeros((nfe, nd + 1))
    for i in range(nfe):
        x0 = rmin + dfe * i
        x1 = x0 + dfe
        xe[i] = x01 * (0.5 * (x1 - x0)) + 0.5 * (x1 + x0)
        we[i] = w01 * (0.5 * (x1 - x0))
    for iB in range(nrad + 1):
        i = min(iB // nd, nfe - 1)
        m = iB - nd * i
        xrad[iB], wrad[iB] = xe[i, m], we[i, m]
    for i in range(1, nfe):
        wrad[nd * i] += we[i - 1, nd]
    # derivative of the Lagrange shape functions: dsh[m, k] = f_m'(x_k) (cldvr.cpp:186-215)
    radk = np.zeros((nrad + 1, bw))
    radk0 = np.zeros((nrad + 1, bw))
    radp = np.zeros((nrad + 1, bw))
    for i in range(nfe):
        xp = xe[i]
        dsh = np.zeros((nd + 1, nd + 1))
        idx = np.arange(nd + 1)
        for m in range(nd + 1):
            for k in range(nd + 1):
                if m == k:
                    continue
                sel = (idx != m) & (idx != k)
                dsh[m, k] = np.prod((xp[k] - xp[sel]) / (xp[m] - xp[sel])) / (xp[m] - xp[k])
        dsh[0, 0] = -0.5 / we[i, 0]
        dsh[nd, nd] = 0.5 / we[i, nd]
        iB0 = nd * i
        wl = we[i]
        lmask0 = np.ones(nd + 1)
        if i == 0:
            lmask0[0] = 0.0
        tk = (dsh * wl[None, :]) @ dsh.T
        tk0 = (dsh * (wl * lmask0)[None, :]) @ dsh.T
        for m in range(nd + 1):
            for k in range(nd + 1):
                if (i == 0 and (m == 0 or k == 0)) or (i == nfe - 1 and (m == nd or k == nd)):
                    continue
                mB, kB = iB0 + m, iB0 + k
                nrm = np.sqrt(wrad[mB] * wrad[kB])
                jb = nd + kB - mB
                radk[mB, jb] += 0.5 * tk[m, k] / nrm
                radk0[mB, jb] += 0.5 * tk0[m, k] / nrm
                radp[mB, jb] += we[i, m] * dsh[k, m] / nrm
    mask = np.zeros(nrad + 1)
    order = 1.0 / mask_cos_order if mask_cos_order > 0 else abs(mask_cos_order)
    for iB in range(1, nrad):
        ax = abs(xrad[iB])
        if ax <= rmask:
            mask[iB] = 1.0
        else:
            mask[iB] = np.cos(0.5 * np.pi * (ax - rmask) / (rmax - rmask)) ** order
    return dict(nrad=nrad, ndvr=nd, nfe=nfe, xrad=xrad, wrad=wrad, mask=mask,
                radk=radk, radk0=radk0, radp=radp, rmask=rmask)


def assoc_legendre_table(lmax, mmax, x):
    """Th[m, l, i] = normalised P_l^m(x_i) with the Condon-Shortley phase,
    int_{-1}^{1} Th^2 dx = 1 (SHTOOLS orthonormalised, complex norm, times
    sqrt(2 pi); sph_gen.F90:37,62-86)."""
    x = np.asarray(x, dtype=np.longdouble)
    s = np.sqrt(np.maximum(0, 1 - x * x))
    th = np.zeros((mmax + 1, lmax + 1, x.size), dtype=np.longdouble)
    pmm = np.full(x.size, np.sqrt(np.longdouble(0.5)))
    for m in range(mmax + 1):
        if m > 0:
            pmm = -np.sqrt(np.longdouble(2 * m + 1) / (2 * m)) * s * pmm
        if m > lmax:
            break
        th[m, m] = pmm
        if m + 1 <= lmax:
            th[m, m + 1] = np.sqrt(np.longdouble(2 * m + 3)) * x * pmm
        for l in range(m + 2, lmax + 1):
            a = np.sqrt((4 * np.longdouble(l) ** 2 - 1) / (np.longdouble(l) ** 2 - m * m))
            b = np.sqrt((np.longdouble(l - 1) ** 2 - m * m) / (4 * np.longdouble(l - 1) ** 2 - 1))
            th[m, l] = a * (x * th[m, l - 1] - b * th[m, l - 2])
    return th


def gauss_legendre(n):
    """Gauss-Legendre nodes (ascending) and weights on [-1, 1] (SHGLQ's quadrature)."""
    x, w = np.polynomial.legendre.leggauss(n)
    return x, w


def sph(lmax1, lmax2, mmax1, mmax2, nlat=0):
    """clsph::gen (clsph.cpp:97-134): theta grid and the four Legendre tables,
    flattened in the reference's Fortran order."""
    nlat = nlat or lmax2 + 1
    cost, wlat = gauss_legendre(nlat)
    th = assoc_legendre_table(lmax2, mmax2, cost)
    L1, L2 = lmax1 + 1, lmax2 + 1
    legf1 = np.zeros((2 * mmax1 + 1, nlat, L1))
    legb1 = np.zeros((2 * mmax1 + 1, L1, nlat))
    legf2 = np.zeros((2 * mmax2 + 1, nlat, L2))
    legb2 = np.zeros((2 * mmax2 + 1, L2, nlat))
    wl = np.asarray(wlat, dtype=np.longdouble)
    for m in range(-mmax2, mmax2 + 1):
        am = abs(m)
        t = th[am]  # (L2, nlat)
        legf2[m + mmax2, :, am:] = t[am:].T.astype(np.float64)
        legb2[m + mmax2, am:, :] = (t[am:] * wl[None, :]).astype(np.float64)
        if am <= mmax1:
            legf1[m + mmax1, :, am:L1] = t[am:L1].T.astype(np.float64)
            legb1[m + mmax1, am:L1, :] = (t[am:L1] * wl[None, :]).astype(np.float64)
    return dict(lmax1=lmax1, lmax2=lmax2, mmax1=mmax1, mmax2=mmax2, nlat=nlat, cost=cost, wlat=wlat,
                legf1=legf1.ravel(), legb1=legb1.ravel(), legf2=legf2.ravel(), legb2=legb2.ravel())


def build(wl):
    """Radial + angular set-up of a workload dict (td1c_b200.workloads)."""
    rad = fedvr(wl["rmin"], wl["rmax"], wl["ndvr"], wl["nfe"], wl["rmask"], wl["mask_cos_order"])
    mmax1 = max(abs(o[2]) for o in wl["orbitals"])
    ang = sph(wl["lmax1"], wl["lmax2"], mmax1, 2 * mmax1, wl.get("nlat", 0) or 0)
    return rad, ang
