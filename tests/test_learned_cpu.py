"""CPU reference of the learned mean-field predictor (oracle/mlp.py).

The network's hand-written backward pass agrees with central differences,
bfloat16 rounding is round-to-nearest-even, Adam fits a small map, the cubic
extrapolation weights reproduce cubics exactly at the RK stage times, and the
oracle's pair potentials come out with the shape and symmetry the predictor's
data path assumes.
"""
import numpy as np

from oracle.mlp import MLP, bf16_round
from td1c_b200 import workloads as W


def test_backward_matches_central_differences():
    m = MLP([12, 32, 32, 32, 5], seed=3)
    rng = np.random.default_rng(0)
    x, y = rng.standard_normal((16, 12)), rng.standard_normal((16, 5))
    assert m.grad_check(x, y) < 1e-5


def test_bf16_rounding_ties_to_even():
    a = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -8, 3.14159265, -2.5e-3, np.inf], dtype=np.float32)
    r = bf16_round(a)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2.0 ** -6  # halfway cases go to the even mantissa
    assert r[3] == 3.140625 and np.isinf(r[5])
    assert np.all(r.view(np.uint32) & 0xFFFF == 0)
    m = MLP([4, 8, 3], seed=1, dtype=np.float32)
    x = np.random.default_rng(2).standard_normal((5, 4)).astype(np.float32)
    assert np.abs(m.forward(x, bf16=True) - m.forward(x)).max() < 5e-2


def test_adam_fits_a_small_map():
    rng = np.random.default_rng(4)
    x = rng.standard_normal((128, 6))
    y = np.stack([np.sin(x[:, 0]) + 0.5 * x[:, 1], x[:, 2] * x[:, 3]], axis=1)
    m = MLP([6, 64, 64, 2], seed=5)
    l0 = m.loss_grad(x, y)[0]
    for _ in range(600):
        _, dW, db = m.loss_grad(x, y)
        m.adam_step(dW, db, lr=3e-3)
    assert m.loss_grad(x, y)[0] < 0.05 * l0


def test_cubic_extrapolation_weights():
    from oracle.mlp import CUBIC
    p = np.poly1d([0.3, -1.2, 0.7, 2.0])
    hist = np.array([p(-k) for k in range(4)])
    for c, w in CUBIC.items():
        assert abs(w.sum() - 1.0) < 1e-15
        assert abs(w @ hist - p(c)) < 1e-12


def test_pair_potentials_accessor():
    from oracle.oracle import Oracle
    from .helpers import oracle_state
    wl = dict(W.MIXED_SMALL, split_type=1)
    o = Oracle(wl)
    orb, cic = oracle_state(o)
    o.set_wfn0(orb, cic)
    orb, cic = o.orth(orb, cic)
    o.htot(1.0, np.zeros(9), orb, cic)
    v = o.v2sph()
    ndyn = len(wl["orbitals"]) - o.dims["nfcore"]
    assert v.shape == (ndyn * (ndyn + 1) // 2, wl["lmax2"] + 1, o.dims["nrad"] - 1)
    assert np.all(np.isfinite(v)) and np.abs(v).max() > 0
    # the first pair is a diagonal one (j = i): its l = 0 potential is that of a real density
    assert np.abs(v[0, 0].imag).max() <= 1e-12 * np.abs(v[0, 0]).max()
