"""The reference's .orb / .cic / .ene text formats (clwfn.cpp:156-305, tdse.cpp:352-354).

No state file ships with the reference, so the checks are the exact line
layout of the C format strings (field widths, 15-digit mantissas, exponent
form), bit-exact round trips, and the projection rules of clwfn::read_orb
and clwfn::read_cic on a basis that differs from the file's.
"""
import numpy as np
import pytest

from td1c_b200 import wfnio


def _state(nfun, L1, Nr, seed=0):
    rng = np.random.default_rng(seed)
    orb = rng.standard_normal((nfun, L1, Nr)) + 1j * rng.standard_normal((nfun, L1, Nr))
    orb[0, 0, 0] = complex(-0.0, 1e-300)  # signed zero and a 3-digit exponent
    orb[0, 0, 1] = 123456.789 - 1e-5j
    return orb


def test_orb_layout_and_round_trip(tmp_path):
    nrad, lmax1, mmax1, nfun = 9, 3, 1, 2
    orb = _state(nfun, lmax1 + 1, nrad - 1)
    p = tmp_path / "x.orb"
    wfnio.write_orb(p, orb, nrad, lmax1, mmax1)
    lines = p.read_text().splitlines()
    assert lines[:4] == ["%10d" % v for v in (nrad, lmax1, mmax1, nfun)]
    assert len(lines) == 4 + orb.size
    # every data line is two 25-wide %le fields, orbital-major, radial index fastest
    for ln in lines[4:]:
        assert len(ln) == 50 and "e" in ln[:25] and "e" in ln[25:]
    assert lines[4] == "%25.15e%25.15e" % (-0.0, 1e-300)
    assert lines[5] == "    1.234567890000000e+05   -1.000000000000000e-05"
    k = 4 + 1 * (lmax1 + 1) * (nrad - 1) + 2 * (nrad - 1) + 3  # orbital 1, l = 2, radial point 4
    assert lines[k] == "%25.15e%25.15e" % (orb[1, 2, 3].real, orb[1, 2, 3].imag)
    back, hdr = wfnio.read_orb(p, nrad, lmax1, nfun)
    assert hdr == {"nrad": nrad, "lmax1": lmax1, "mmax1": mmax1, "nfun": nfun}
    # 15 digits after the point: 16 significant digits, within one rounding of a double
    assert np.allclose(back, orb, rtol=2e-16 * 8, atol=0)


def test_orb_projection_onto_another_basis(tmp_path):
    nrad, lmax1, nfun = 9, 3, 3
    orb = _state(nfun, lmax1 + 1, nrad - 1, seed=1)
    p = tmp_path / "big.orb"
    wfnio.write_orb(p, orb, nrad, lmax1, 0)
    # smaller basis: the extra orbitals, l and radial points are dropped
    small, _ = wfnio.read_orb(p, 6, 1, 2)
    assert small.shape == (2, 2, 5)
    assert np.allclose(small, orb[:2, :2, :5], rtol=1e-15, atol=0)
    # larger basis: the file's values in place, the rest zero
    big, _ = wfnio.read_orb(p, 12, 5, 4)
    assert big.shape == (4, 6, 11)
    assert np.allclose(big[:3, :4, :8], orb, rtol=1e-15, atol=0)
    big[:3, :4, :8] = 0
    assert not big.any()


def test_cic_round_trip_and_length_mismatch(tmp_path):
    rng = np.random.default_rng(2)
    cic = rng.standard_normal(7) + 1j * rng.standard_normal(7)
    p = tmp_path / "x.cic"
    wfnio.write_cic(p, cic)
    lines = p.read_text().splitlines()
    assert lines[0] == "%10d" % 7 and len(lines) == 8
    assert all(len(ln) == 50 for ln in lines[1:])
    assert np.allclose(wfnio.read_cic(p, 7), cic, rtol=2e-15, atol=0)
    assert wfnio.read_cic(p, 8) is None  # another CI space: not read


def test_wfn_pair_and_truncation_errors(tmp_path):
    orb = _state(2, 2, 4, seed=3)
    cic = np.array([1.0 + 0j, -0.5j])
    po, pc = tmp_path / "s.orb", tmp_path / "s.cic"
    wfnio.write_wfn(po, pc, orb, cic, 5, 1, 0)
    o, c = wfnio.read_wfn(po, pc, 5, 1, 2, 2)
    assert np.allclose(o, orb, rtol=2e-15, atol=0) and np.allclose(c, cic, rtol=2e-15, atol=0)
    po.write_text("\n".join(po.read_text().splitlines()[:-1]) + "\n")  # drop the last value
    with pytest.raises(ValueError):
        wfnio.read_orb(po, 5, 1, 2)


def test_ene_line(tmp_path):
    ln = wfnio.ene_line(1200, 4.8, 0.087, -0.0119, 0.2, -128.54712)
    assert ln == "      1200 %20.10e %20.10e %20.10e %20.10e %20.10e\n" % (4.8, 0.087, -0.0119, 0.2, -128.54712)
    assert len(ln) == 10 + 5 * 21 + 1
    p = tmp_path / "x.ene"
    p.write_text(ln + wfnio.ene_line(1201, 4.804, 0.0871, -0.012, 0.2001, -128.5471))
    t = wfnio.read_ene(p)
    assert list(t["step"]) == [1200, 1201] and np.allclose(t["ene"], [-128.54712, -128.5471])


def test_op1_line():
    ln = wfnio.op1_line(7, 0.028, 0.0005, 1e-3, -2e-2, 0.125, -0.5, 3.25)
    assert ln == "         7 %20.10e %20.10e %20.10e %20.10e %20.10e %20.10e %20.10e\n" % (
        0.028, 0.0005, 1e-3, -2e-2, 0.125, -0.5, 3.25)
    assert len(ln) == 10 + 7 * 21 + 1
