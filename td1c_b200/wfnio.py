"""The reference's on-disk formats for states and the energy trace.

Text files, as td1c writes and reads them (src/wfn/clwfn.cpp:156-305,
src/main/tdse.cpp:352-366):

``.orb``  four header lines ``%10d``: nrad, lmax1, mmax1, nfun; then one
          line ``%25.15le%25.15le`` (real, imaginary) per orbital value, in
          the order orbital, l = 0 .. lmax1, radial point 1 .. nrad - 1
          (radial index fastest: the layout of the library's orbital arrays,
          [nfun][lmax1 + 1][nrad - 1]).
``.cic``  one header line ``%10d``: lcic; then one ``%25.15le%25.15le``
          line per CI coefficient.
``.ene``  one line per printed step: ``%10d`` step, then time, time in
          optical cycles, E_z(t), A_z(t) and the total energy as ``%20.10e``,
          separated by single spaces.
``.op1``  the same five leading columns, then the total dipole in the length,
          velocity and acceleration forms (dip(3), vel(3), acc(3) of
          hprod_dipole; tdse.cpp:365-366).

Reading follows ``clwfn::read_orb`` / ``clwfn::read_cic``: an orbital file
written on another basis is projected onto the current one (values of
orbitals, l or radial points outside the current basis are dropped, the
missing ones stay zero), and a CI file whose length differs from the current
lcic is not read (the reference then falls back to its default CI vector,
``ormas_cic0``; here the reader returns None and the caller chooses the
state).  The optional ``symlm`` symmetrisation that the reference applies
after reading orbitals is not part of the format and is not done here.
"""
import numpy as np


def _pair(z):
    return "%25.15e%25.15e\n" % (z.real, z.imag)


def write_orb(path, orb, nrad, lmax1, mmax1):
    """Write orbitals [nfun][lmax1 + 1][nrad - 1] (any array reshapeable to that) as ``.orb``
    (clwfn::write, clwfn.cpp:270-288)."""
    L1, Nr = lmax1 + 1, nrad - 1
    a = np.asarray(orb, dtype=np.complex128).reshape(-1, L1, Nr)
    with open(path, "w") as f:
        f.write("%10d\n%10d\n%10d\n%10d\n" % (nrad, lmax1, mmax1, a.shape[0]))
        f.writelines(_pair(z) for z in a.reshape(-1))


def read_orb(path, nrad, lmax1, nfun):
    """Read a ``.orb`` file onto the current basis (nrad, lmax1, nfun): returns
    (orbitals [nfun][lmax1 + 1][nrad - 1], header dict).  Entries of the file outside the
    basis are dropped; orbitals, l or radial points the file lacks are zero
    (clwfn::read_orb, clwfn.cpp:208-242)."""
    with open(path) as f:
        tok = f.read().split()
    if len(tok) < 4:
        raise ValueError("%s: truncated .orb header" % path)
    nrad0, lmax0, mmax0, nfun0 = (int(t) for t in tok[:4])
    n0 = nfun0 * (lmax0 + 1) * (nrad0 - 1)
    if len(tok) < 4 + 2 * n0:
        raise ValueError("%s: %d values expected, %d found" % (path, n0, (len(tok) - 4) // 2))
    v = np.array(tok[4:4 + 2 * n0], dtype=np.float64)
    src = (v[0::2] + 1j * v[1::2]).reshape(nfun0, lmax0 + 1, nrad0 - 1)
    out = np.zeros((nfun, lmax1 + 1, nrad - 1), dtype=np.complex128)
    nf, nl, nr = min(nfun, nfun0), min(lmax1, lmax0) + 1, min(nrad, nrad0) - 1
    out[:nf, :nl, :nr] = src[:nf, :nl, :nr]
    return out, {"nrad": nrad0, "lmax1": lmax0, "mmax1": mmax0, "nfun": nfun0}


def write_cic(path, cic):
    """Write CI coefficients as ``.cic`` (clwfn::write, clwfn.cpp:290-304)."""
    c = np.asarray(cic, dtype=np.complex128).reshape(-1)
    with open(path, "w") as f:
        f.write("%10d\n" % c.size)
        f.writelines(_pair(z) for z in c)


def read_cic(path, lcic):
    """Read a ``.cic`` file of the current length lcic: the coefficients, or None when the
    file holds another length (the reference then keeps its default CI vector;
    clwfn::read_cic, clwfn.cpp:244-262)."""
    with open(path) as f:
        tok = f.read().split()
    if not tok:
        raise ValueError("%s: empty .cic file" % path)
    lcic0 = int(tok[0])
    if lcic0 != lcic:
        return None
    if len(tok) < 1 + 2 * lcic:
        raise ValueError("%s: %d coefficients expected, %d found" % (path, lcic, (len(tok) - 1) // 2))
    v = np.array(tok[1:1 + 2 * lcic], dtype=np.float64)
    return v[0::2] + 1j * v[1::2]


def write_wfn(orb_path, cic_path, orb, cic, nrad, lmax1, mmax1):
    """clwfn::write: the orbital and CI files of one state."""
    write_orb(orb_path, orb, nrad, lmax1, mmax1)
    write_cic(cic_path, cic)


def read_wfn(orb_path, cic_path, nrad, lmax1, nfun, lcic):
    """clwfn::read: (orbitals, CI coefficients or None when the CI length differs)."""
    orb, _ = read_orb(orb_path, nrad, lmax1, nfun)
    return orb, read_cic(cic_path, lcic)


def ene_line(step, time, ncyc, efield, afield, ene):
    """One line of the ``.ene`` trace (tdse.cpp:353-354): step, time (au), time in optical
    cycles, E_z(t) = lfield(3, 2), A_z(t) = lfield(3, 3), total energy."""
    return "%10d %20.10e %20.10e %20.10e %20.10e %20.10e\n" % (step, time, ncyc, efield, afield, ene)


def op1_line(step, time, ncyc, efield, afield, dip, vel, acc):
    """One line of the ``.op1`` trace (tdse.cpp:365-366): the ``.ene`` leading columns, then
    the length, velocity and acceleration forms of the total dipole."""
    return "%10d %20.10e %20.10e %20.10e %20.10e %20.10e %20.10e %20.10e\n" % (step, time, ncyc, efield, afield, dip,
                                                                              vel, acc)


def read_ene(path):
    """Parse a ``.ene`` trace into columns (step, time, ncyc, E_z, A_z, energy)."""
    rows = [ln.split() for ln in open(path) if ln.strip() and not ln.lstrip().startswith("#")]
    a = np.array(rows, dtype=np.float64).reshape(-1, 6)
    return {"step": a[:, 0].astype(np.int64), "time": a[:, 1], "ncyc": a[:, 2], "efield": a[:, 3],
            "afield": a[:, 4], "ene": a[:, 5]}
