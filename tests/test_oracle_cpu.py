"""Known-answer checks that pin the CPU oracle (no GPU needed).

The reference ships no tests or golden outputs and cannot be built here, so
the oracle is pinned by analytic properties of the restated algorithm:
hydrogenic spectra of the FEDVR one-body table, Legendre-table
orthonormality, the Poisson solve of a closed-form density, Hermiticity and
conservation properties of the RHS, RDM traces, and LAPACK cross-checks.
"""
import numpy as np
import pytest
import scipy.linalg as sl

from oracle.oracle import Oracle
from td1c_b200 import workloads as W

from .helpers import oracle_state, rel_err


def band_to_dense(band, Nr, nd):
    A = np.zeros((Nr, Nr))
    for i in range(Nr):
        for jb in range(2 * nd + 1):
            j = i + jb - nd
            if 0 <= j < Nr:
                A[i, j] = band[i, jb]
    return A


@pytest.fixture(scope="module")
def he():
    return Oracle(W.HE_TDHF)


def test_hydrogenic_spectrum(he):
    """tmat (bas_gen_tmat.F90) at l = 0, 1 reproduces -Z^2 / 2 n^2 for Z = 2."""
    d = he.dims
    Nr, nd, L1 = d["nrad"] - 1, d["ndvr"], d["lmax1"] + 1
    tm = he.get("tmat").reshape(L1, Nr, 2 * nd + 1)
    for l in (0, 1):
        A = band_to_dense(tm[l], Nr, nd)
        assert np.abs(A - A.T).max() < 1e-10
        ev = np.linalg.eigvalsh(A)
        for k, n in enumerate(range(l + 1, l + 4)):
            assert abs(ev[k] + 2.0 / n ** 2) < 2e-6, (l, n, ev[k])


def test_legendre_orthonormal(he):
    """sum_theta legb(theta, l, m) legf(l', theta, m) = delta_ll' (sph_gen.F90)."""
    d = he.dims
    nlat, L1, L2 = d["nlat"], d["lmax1"] + 1, d["lmax2"] + 1
    lf2 = he.get("legf2").reshape(-1, nlat, L2)
    lb2 = he.get("legb2").reshape(-1, L2, nlat)
    for mi in range(lf2.shape[0]):
        G = lb2[mi] @ lf2[mi]
        nz = np.abs(np.diag(G)) > 0
        assert np.abs(G[np.ix_(nz, nz)] - np.eye(nz.sum())).max() < 1e-12


def test_legendre_tables_against_scipy():
    """The theta tables against an independent associated-Legendre evaluation (scipy's lpmv, with
    the Condon-Shortley phase): legf(theta, l, m) = sqrt((2l+1)/2 (l-|m|)!/(l+|m|)!) P_l^|m|(cos theta),
    zero below |m|; legb = w_theta legf^T; the theta nodes and weights are the Gauss-Legendre rule."""
    from scipy.special import gammaln, lpmv
    o = Oracle(dict(W.MIXED_SMALL))
    d = o.dims
    nlat = d["nlat"]
    cost, wlat = o.get("cost"), o.get("wlat")
    x, w = np.polynomial.legendre.leggauss(nlat)
    assert np.abs(np.sort(cost) - x).max() < 1e-14 and np.abs(wlat[np.argsort(cost)] - w).max() < 1e-14
    for nf, nb, L in (("legf1", "legb1", d["lmax1"] + 1), ("legf2", "legb2", d["lmax2"] + 1)):
        lf = o.get(nf).reshape(-1, nlat, L)
        lb = o.get(nb).reshape(-1, L, nlat)
        mm = (lf.shape[0] - 1) // 2
        assert mm >= 1
        for m in range(-mm, mm + 1):
            am = abs(m)
            ref = np.zeros((nlat, L))
            for l in range(am, L):
                ref[:, l] = np.sqrt((2 * l + 1) / 2.0 * np.exp(gammaln(l - am + 1) - gammaln(l + am + 1))) * lpmv(am, l, cost)
            assert np.abs(lf[m + mm] - ref).max() < 1e-13 * max(1.0, np.abs(ref).max()), (nf, m)
            assert np.abs(lb[m + mm] - (lf[m + mm] * wlat[:, None]).T).max() < 1e-15, (nb, m)


def test_gauss_lobatto_against_dsyev():
    """Lobatto interior nodes = eigenvalues of the cldvr.cpp:82-139 Jacobi matrix."""
    from td1c_b200.basis import lobatto
    o = Oracle(W.HE_SMALL)
    x = o.get("xrad")
    # first element of the oracle grid on [0, 2] mapped back to [-1, 1]
    nd = o.dims["ndvr"]
    xe = x[: nd + 1] - 1.0
    xl, _ = lobatto(nd)
    assert np.abs(xe - xl).max() < 1e-14


def test_poisson_against_lapack_and_slater():
    """d2ll (bas_gen_d2ll.F90) equals scipy's dpbtrf factor, and the frozen-core
    Hartree potential of a doubly occupied hydrogen 1s core (density 4 r^2
    e^{-2r} per electron) is the closed form 2 [1/r - (1 + 1/r) e^{-2r}]
    (hprod_mkv2jfc in hprod_set_wfn0.F90)."""
    wl = dict(W.NE_SMALL, rmax=30.0, nfe=15, ndvr=10, orbitals=[(1, 0, 0, -1), (2, 0, 0, 1)], nela=2, nelb=2,
              znuc=1.0, rmask=25.0)
    o = Oracle(wl)
    d = o.dims
    Nr, nd = d["nrad"] - 1, d["ndvr"]
    xr, wr = o.get("xrad"), o.get("wrad")
    radk = o.get("radk").reshape(-1, 2 * nd + 1)
    d2ll = o.get("d2ll").reshape(d["lmax2"] + 1, Nr, nd + 1)
    for l in (0, 3):
        A = np.zeros((nd + 1, Nr))
        A[0] = l * (l + 1) / xr[1:Nr + 1] ** 2
        for ir in range(1, Nr + 1):
            for jr in range(ir, min(Nr, ir + nd) + 1):
                A[jr - ir, ir - 1] += 2.0 * radk[ir, jr - ir + nd]
        ref, info = sl.lapack.dpbtrf(A, lower=1)
        assert info == 0
        assert np.abs(ref - d2ll[l].T).max() < 1e-10 * np.abs(ref).max()
    # hydrogen 1s frozen core: rho(r) = 4 r^2 e^{-2r} (unit norm), V = 1/r - (1 + 1/r) e^{-2r}
    r = xr[1:Nr + 1]
    orb = np.zeros((2, d["lmax1"] + 1, Nr), dtype=np.complex128)
    orb[0, 0] = 2.0 * r * np.exp(-r) * np.sqrt(wr[1:Nr + 1])
    orb[1, 0] = orb[0, 0]
    o.set_wfn0(orb, np.ones(1, dtype=np.complex128))
    v = o.get("v2jfc", True).real
    exact = 2.0 * (1.0 / r - (1.0 + 1.0 / r) * np.exp(-2 * r))
    inner = r < 20
    assert np.abs(v[inner] - exact[inner]).max() < 1e-7  # FEDVR discretisation error of the 1s density


@pytest.mark.parametrize("wl", [W.NE_SMALL, W.MIXED_SMALL, W.OPEN_SMALL], ids=lambda w: w["name"])
def test_rhs_structure(wl):
    """Properties of hprod_htot that hold exactly: zero field preserves orbital
    norms (Re <phi|dphi/dt> = 0 with the Q projector), the CI derivative is
    orthogonal to c for the Hermitian sigma, den1 is Hermitian with trace
    N_active, frozen-core rows of hwfn vanish, int1e / int2e symmetries."""
    o = Oracle(wl)
    d = o.dims
    orb, cic = oracle_state(o)
    o.set_wfn0(orb, cic)
    hw, hc = o.htot(1.0, np.zeros(9), orb, cic)
    nf = len(wl["orbitals"])
    hw2, orb2 = hw.reshape(nf, -1), orb.reshape(nf, -1)
    nfc = d["nfcore"]
    assert np.abs(hw2[:nfc]).max() == 0.0
    for f in range(nfc, nf):
        assert abs(np.vdot(orb2[f], hw2[f]).real) < 1e-12
    assert abs(np.vdot(cic, hc).real) < 1e-12
    n = d["nact"]
    D = o.get("den1", True).reshape(n, n).T
    assert np.abs(D - D.conj().T).max() < 1e-13
    nel_act = wl["nela"] + wl["nelb"] - 2 * d["ncore"]
    assert abs(np.trace(D).real - nel_act) < 1e-12
    I1 = o.get("int1e", True).reshape(n, n).T
    assert np.abs(I1 - I1.conj().T).max() < 1e-12
    I2 = o.get("int2e", True).reshape(n, n, n, n, order="F")
    assert np.abs(I2 - np.conj(I2.transpose(1, 0, 3, 2))).max() < 1e-11
    e = o.energies()
    assert abs(e["ene_tot"] - (e["ene_core"] + e["ene_act"])) < 1e-12


def test_hermitian_regularised_inverse():
    """invden: U diag(d/(d^2 + 1e-15)) U^H equals scipy's eigh-based value."""
    wl = W.NE_SMALL
    o = Oracle(wl)
    orb, cic = oracle_state(o)
    o.set_wfn0(orb, cic)
    o.htot(1.0, np.zeros(9), orb, cic)
    n = o.dims["nact"]
    D = o.get("den1", True).reshape(n, n).T
    R = o.get("rden", True).reshape(n, n).T
    w, U = np.linalg.eigh(D)
    ref = (U * (w / (w * w + 1e-15))) @ U.conj().T
    assert np.abs(R - ref).max() < 1e-12 * np.abs(ref).max()


def test_field_sin2_velocity():
    """clfield1 velocity1: A = env F0/w sin(w t + cep), E = -dA/dt (6-point rule)."""
    wl = W.NE_CAS
    o = Oracle(wl)
    famp = np.sqrt(wl["fint"] / 3.50944506e16)
    w = 1239.84190 / (wl["wlen"] * 27.2113845)
    T = wl["numcyc"] * 2 * np.pi / w
    for t in (0.1 * T, 0.37 * T, 0.5 * T):
        env = np.sin(np.pi * t / T) ** 2
        A = env * famp / w * np.sin(w * t)
        dA = famp / w * (2 * np.sin(np.pi * t / T) * np.cos(np.pi * t / T) * np.pi / T * np.sin(w * t)
                         + env * w * np.cos(w * t))
        lf = o.field(t)
        assert abs(lf[2] - A) < 1e-14 and abs(lf[8] - A) < 1e-14
        assert abs(lf[5] + dA) < 1e-8 * famp


@pytest.mark.parametrize("base", [W.HE_SMALL, W.MIXED_SMALL], ids=lambda w: w["name"])
def test_imaginary_time_relaxation(base):
    """init_prop12 form: the energy falls monotonically, and orth leaves an orthonormal set and a unit CI vector."""
    wl = dict(base, icomp=0)
    o = Oracle(wl)
    orb, cic = oracle_state(o)
    orb, cic = o.orth(orb, cic)
    nf = len(wl["orbitals"])
    mval = [x[2] for x in wl["orbitals"]]
    w2 = orb.reshape(nf, -1)
    for i in range(nf):
        for j in range(nf):
            if mval[i] == mval[j] and i >= o.dims["nfcore"]:
                assert abs(np.vdot(w2[j], w2[i]) - (1.0 if i == j else 0.0)) < 1e-12
    assert abs(np.linalg.norm(cic) - 1.0) < 1e-14
    w, c, e = o.relax(orb, cic, 2e-4, 25)
    assert np.all(np.diff(e) < 0), e
    assert abs(np.linalg.norm(c) - 1.0) < 1e-14


def _dense_T(o, l):
    d = o.dims
    Nr, nd, L1 = d["nrad"] - 1, d["ndvr"], d["lmax1"] + 1
    tm = o.get("tmat").reshape(L1, Nr, 2 * nd + 1)
    return band_to_dense(tm[l], Nr, nd)


@pytest.mark.parametrize("wl", [W.MIXED_SMALL, W.NE_SMALL], ids=lambda w: w["name"])
def test_one_body_inverse_against_lapack(wl):
    """dpade_prod with split_type 2 (no laser cycles) is (1 + i dt/2 T_l)^-1 per channel:
    the oracle's ZGBTF2/ZGBTRS restatement against LAPACK ?gbsv through scipy."""
    o = Oracle(dict(wl, split_type=2))
    o.set_split(2)
    orb, cic = oracle_state(o)
    o.set_wfn0(orb, cic)
    d = o.dims
    Nr, nd, L1, nfc = d["nrad"] - 1, d["ndvr"], d["lmax1"] + 1, d["nfcore"]
    mval = [x[2] for x in wl["orbitals"]]
    nf = len(mval)
    dt = 0.05
    w2, ncorr = o.dpade_prod(np.zeros(9), dt, orb, alpha=2.0)
    assert ncorr == 0
    W0, W2 = orb.reshape(nf, L1, Nr), w2.reshape(nf, L1, Nr)
    assert np.array_equal(W2[:nfc], W0[:nfc])
    for l in range(L1):
        M = np.eye(Nr) + 1j * dt / 2 * _dense_T(o, l).T
        ab = np.zeros((2 * nd + 1, Nr), complex)
        for i in range(Nr):
            for j in range(max(0, i - nd), min(Nr, i + nd + 1)):
                ab[nd + i - j, j] = M[i, j]
        for f in range(nfc, nf):
            if l < abs(mval[f]):
                assert np.array_equal(W2[f, l], W0[f, l])
                continue
            x = sl.solve_banded((nd, nd), ab, W0[f, l])
            assert np.abs(x - W2[f, l]).max() <= 1e-13 * np.abs(x).max()


@pytest.mark.parametrize("wl", [W.MIXED_SMALL, W.LENGTH_SMALL], ids=lambda w: w["name"])
def test_crank_nicolson_one_body_step(wl):
    """h1itr_prop: without the laser the step is the Cayley form of exp(-i dt T), exactly
    unitary; with the laser the correction cycles converge to the Cayley form of T + V
    (unitary to the threshold) and stop once the correction norm is below it."""
    o = Oracle(dict(wl, split_type=2))
    o.set_split(2)
    orb, cic = oracle_state(o)
    o.set_wfn0(orb, cic)
    nf = len(wl["orbitals"])
    n0 = np.linalg.norm(orb.reshape(nf, -1), axis=1)
    w, ncorr = o.h1itr_prop(np.zeros(9), 0.05, orb)
    assert ncorr == 0
    assert np.abs(np.linalg.norm(w.reshape(nf, -1), axis=1) - n0).max() < 1e-13
    # backward step returns the state: (1 + i dt/2 T)(1 - i dt/2 T)^-1 inverts the Cayley map
    wb, _ = o.h1itr_prop(np.zeros(9), -0.05, w)
    assert rel_err(wb, orb) < 1e-13
    o.set_split(1)
    lf = np.zeros(9)
    lf[2] = lf[8] = 1.5 if wl["igauge"] == 1 else 0.3
    w1, n1 = o.h1itr_prop(lf, 0.05, orb, 30, 1e-12)
    assert 3 <= n1 < 30
    assert np.abs(np.linalg.norm(w1.reshape(nf, -1), axis=1) - n0).max() < 1e-10
    wb, _ = o.h1itr_prop(lf, -0.05, w1, 30, 1e-12)
    assert rel_err(wb, orb) < 1e-10


def test_split_propagators_beyond_rk4_limit():
    """split2 and ETD-RK2 stay bounded at dt = 0.05 on a grid where full-H RK4 needs dt < 1e-3."""
    wl = dict(W.MIXED_SMALL, split_type=1)
    o = Oracle(wl)
    o.set_split(1)
    orb, cic = oracle_state(o)
    o.set_wfn0(orb, cic)
    nf = len(wl["orbitals"])
    for prop in (o.split2, o.etdrk2):
        w, c, dip = prop(orb, cic, 10.0, 0.05, 20)
        assert np.all(np.isfinite(w)) and np.all(np.isfinite(dip))
        assert np.abs(np.linalg.norm(w.reshape(nf, -1), axis=1) - 1).max() < 0.3
    o.set_split(0)
    w, c, dip = o.rk4(orb, cic, 10.0, 0.05, 3)
    assert not np.all(np.abs(w) < 10)  # full-H RK4 blows up at this step


def test_etdrk4_functions_and_order():
    """cletdrk4's rational one-body functions (orders 2/2, as restated in the oracle) against the
    exact exp / phi functions they approximate, and fourth-order convergence of the ETD-RK4
    trajectory (mask moved outside the grid) against a fine split2 reference."""
    from oracle.oracle import Oracle
    from .helpers import oracle_state
    wl = dict(W.HE_SMALL, split_type=1, rmask=1e9)
    o = Oracle(wl)
    o.set_split(1)
    dt = 0.01
    g = lambda x: (np.exp(x) - 1) / x
    f0 = lambda x: (-4 - x + np.exp(x) * (4 - 3 * x + x * x)) / x**3
    f1 = lambda x: 2 * (2 + x + np.exp(x) * (x - 2)) / x**3
    f2 = lambda x: (-4 - 3 * x - x * x + np.exp(x) * (4 - x)) / x**3
    exact = [lambda l: np.exp(-1j * l * dt), lambda l: np.exp(-1j * l * dt / 2), lambda l: dt / 2 * g(-1j * l * dt / 2),
             lambda l: dt * f0(-1j * l * dt), lambda l: dt * f1(-1j * l * dt), lambda l: dt * f2(-1j * l * dt)]
    for w in range(6):
        F = o.etd4_fun(w, dt)
        for lam in (3.0, 30.0):
            num = sum(F["n"][k] * (F["dt"] * lam) ** k for k in range(3))
            den = np.prod([F["d0"][k] + F["d1"][k] * lam for k in range(2)])
            assert abs(num / den - exact[w](lam)) < 1e-5 * abs(exact[w](lam)), (w, lam)
    orb, cic = oracle_state(o)
    o.set_wfn0(orb, cic)
    orb, cic = o.orth(orb, cic)
    freq = 1239.84190 / (wl["wlen"] * 27.2113845)
    t0, T = 0.3 * wl["numcyc"] * 2 * np.pi / freq, 0.04
    ref = o.split2(orb, cic, t0, T / 400, 400)[0]
    err = [np.linalg.norm(o.etdrk4(orb, cic, t0, T / n, n)[0] - ref) / np.linalg.norm(ref) for n in (4, 8)]
    assert err[1] < 1e-6 and err[0] / err[1] > 10, err


def test_dipole_forms_ehrenfest():
    """hprod_dipole without a frozen core (He, velocity gauge, mask outside the grid): along a short
    split2 trajectory, d<z>/dt equals the velocity form and d<v>/dt the acceleration form (central
    differences), which fixes the operators, their signs and the field terms."""
    from oracle.oracle import Oracle
    from .helpers import oracle_state
    wl = dict(W.HE_SMALL, split_type=1, rmask=1e9)
    o = Oracle(wl)
    o.set_split(1)
    orb, cic = oracle_state(o)
    o.set_wfn0(orb, cic)
    orb, cic = o.orth(orb, cic)
    freq = 1239.84190 / (wl["wlen"] * 27.2113845)
    t0, dt = 0.5 * wl["numcyc"] * 2 * np.pi / freq, 2e-3
    vals, w, c = [], orb, cic
    for s in range(5):
        vals.append(o.dipole3(w, c, o.field(t0 + s * dt)))
        w, c, _ = o.split2(w, c, t0 + s * dt, dt, 1)
    d = np.array([v[0][2] for v in vals])
    v = np.array([v[1][2] for v in vals])
    a = np.array([v[2][2] for v in vals])
    for s in (1, 2, 3):
        assert abs((d[s + 1] - d[s - 1]) / (2 * dt) - v[s]) < 1e-4 * abs(v[s]), (s, d, v)
        assert abs((v[s + 1] - v[s - 1]) / (2 * dt) - a[s]) < 1e-2 * abs(a[s]), (s, v, a)


def _ehrenfest_trace(wl, nstep=3, dt=2e-3):
    """dipole3 at nstep points of a split2 trajectory from the middle of the pulse."""
    from oracle.oracle import Oracle
    from .helpers import oracle_state
    o = Oracle(wl)
    o.set_split(1)
    orb, cic = oracle_state(o)
    o.set_wfn0(orb, cic)
    orb, cic = o.orth(orb, cic)
    freq = 1239.84190 / (wl["wlen"] * 27.2113845)
    t0 = 0.5 * wl["numcyc"] * 2 * np.pi / freq
    vals, w, c = [], orb, cic
    for s in range(nstep):
        vals.append(o.dipole3(w, c, o.field(t0 + s * dt)))
        w, c, _ = o.split2(w, c, t0 + s * dt, dt, 1)
    return [np.array([v[k] for v in vals]) for k in range(3)]  # dip, vel, acc: [step][3]


@pytest.mark.parametrize("gauge", ["length", "velocity"])
def test_dipole_forms_frozen_core(gauge):
    """hprod_dipole with a frozen core (hprod_gfock, hprod_projfc; C with a frozen 1s, a dynamic
    2s and a 2s2p active space; elements of 0.875 bohr, mask outside the grid).  Along a split2
    trajectory the corrected velocity form vel(3) is d<z>/dt while the plain trace vel(1) is far
    from it; the corrected acceleration form acc(3) is d/dt of the plain momentum trace vel(1)
    (the same identity with p_z in place of z) while acc(1) alone is not.  The acceleration
    identity is checked in the length gauge: the seeded state's grid-frequency components make
    the velocity-gauge momentum vary faster than a 2e-3 difference resolves."""
    base = W.LENGTH_SMALL if gauge == "length" else W.MIXED_SMALL
    dt = 2e-3
    dip, vel, acc = _ehrenfest_trace(dict(base, split_type=1, rmask=1e9, nfe=16), dt=dt)
    dd = (dip[2, 2] - dip[0, 2]) / (2 * dt)
    assert abs(dd - vel[1, 2]) < 2e-4 * abs(vel[1, 2]), (dd, vel[1])
    assert abs(dd - vel[1, 0]) > 0.2 * abs(vel[1, 2])  # the corrections are needed
    assert dip[1, 1] == 0.0 and vel[1, 2] == vel[1, 0] + vel[1, 1] and acc[1, 2] == acc[1, 0] + acc[1, 1]
    if gauge == "length":
        dv1 = (vel[2, 0] - vel[0, 0]) / (2 * dt)
        assert abs(dv1 - acc[1, 2]) < 3e-2 * abs(acc[1, 2]), (dv1, acc[1])
        assert abs(dv1 - acc[1, 0]) > 0.1 * abs(acc[1, 2])
