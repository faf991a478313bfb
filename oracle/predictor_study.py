"""CPU study of the learned mean-field predictor's data (test infrastructure; run as a script).

The predictor would replace the exact pair potentials v2sph(r, l, pair) at the
RK stages of a split2 step (times t_n + c dt, c = 1/2 and 1) by a prediction
from the last four full steps.  This script measures, with the oracle on the
frozen-core C workload (1 frozen, 1 dynamic core, 4 active orbitals; mask
outside the grid; dt = 0.004), how far the stage values lie from:
  hold   v(t_n),
  cubic  the cubic extrapolation through v(t_n), ..., v(t_{n-3}),
  c+mlp  cubic plus the correction of the reference network (oracle/mlp.py:
         width 256, 4 linear layers, tanh; inputs the four normalised history
         vectors and c; trained with Adam on one pulse's cubic residuals),
on a second pulse the network never saw.  Errors are per (pair, l) vector,
relative to that vector's largest history value.  `--relax` starts both
pulses from a state relaxed in imaginary time (300 ETD-RK2 cycles, dt 0.01).

    python oracle/predictor_study.py [--relax] [--epochs N]
"""
import argparse
import os
import sys

import numpy as np

sys.path[0] = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))  # the repository, not this folder

from oracle.mlp import MLP  # noqa: E402
from oracle.oracle import Oracle  # noqa: E402
from td1c_b200 import workloads as W  # noqa: E402

# Lagrange weights of the cubic through tau = 0, -1, -2, -3 evaluated at tau = c
CUBIC = {1.0: np.array([4.0, -6.0, 4.0, -1.0]), 0.5: np.array([2.1875, -2.1875, 1.3125, -0.3125])}


def seeded_state(o):
    from tests.helpers import oracle_state
    return oracle_state(o)


def series(fint, wlen, nfine, dt=0.004, relax=False):
    """v2sph at t0 + s dt / 2, s < nfine, along a split2 trajectory of half steps: [time][vector][Nr]."""
    wl = dict(W.MIXED_SMALL, split_type=1, rmask=1e9, fint=fint, wlen=wlen)
    if relax:
        o0 = Oracle(dict(wl, icomp=0))
        o0.set_split(1)
        orb, cic = seeded_state(o0)
        o0.set_wfn0(orb, cic)
        orb, cic = o0.orth(orb, cic)
        orb, cic, _ = o0.relax_etdrk2(orb, cic, 0.01, 300)
        o = Oracle(wl)
        o.set_split(1)
        o.set_wfn0(orb, cic)
    else:
        o = Oracle(wl)
        o.set_split(1)
        orb, cic = seeded_state(o)
        o.set_wfn0(orb, cic)
        orb, cic = o.orth(orb, cic)
    freq = 1239.84190 / (wl["wlen"] * 27.2113845)
    t0 = 0.4 * wl["numcyc"] * 2 * np.pi / freq
    vs, w, c = [], orb, cic
    for s in range(nfine):
        t = t0 + s * dt / 2
        o.htot(1.0, o.field(t), w, c)
        vs.append(o.v2sph().reshape(-1, o.dims["nrad"] - 1))
        w, c, _ = o.split2(w, c, t, dt / 2, 1)
    return np.array(vs)


def samples(V):
    """Network inputs, cubic-residual targets, and (cubic, hold, true) stage values, all scaled."""
    X, Y, cub_l, hold_l, true_l = [], [], [], [], []
    for n in range(3, (V.shape[0] - 2) // 2):
        hist = np.stack([V[2 * (n - k)] for k in range(4)])
        s = np.abs(hist).max(axis=(0, 2))[:, None] + 1e-300
        h = hist / s
        for c, fi in ((0.5, 2 * n + 1), (1.0, 2 * n + 2)):
            cub = np.tensordot(CUBIC[c], h, axes=1)
            nv = h.shape[1]
            X.append(np.concatenate([h.real.transpose(1, 0, 2).reshape(nv, -1), h.imag.transpose(1, 0, 2).reshape(nv, -1),
                                     np.full((nv, 1), c)], axis=1))
            r = V[fi] / s - cub
            Y.append(np.concatenate([r.real, r.imag], axis=1))
            cub_l.append(cub)
            hold_l.append(h[0])
            true_l.append(V[fi] / s)
    return (np.concatenate(X), np.concatenate(Y), np.concatenate(cub_l), np.concatenate(hold_l), np.concatenate(true_l))


def run(relax=False, epochs=300, nfine=40, seed=0):
    XA, YA, _, _, _ = samples(series(1e14, 800.0, nfine, relax=relax))
    XB, _, cubB, holdB, trueB = samples(series(2e14, 700.0, nfine, relax=relax))
    ys = np.abs(YA).max()
    net = MLP([XA.shape[1], 256, 256, 256, YA.shape[1]], seed=seed, dtype=np.float32)
    rng = np.random.default_rng(seed)
    for _ in range(epochs):
        idx = rng.permutation(len(XA))
        for b0 in range(0, len(XA), 256):
            j = idx[b0:b0 + 256]
            _, dW, db = net.loss_grad(XA[j].astype(np.float32), (YA[j] / ys).astype(np.float32))
            net.adam_step(dW, db, lr=3e-4)
    p = net.forward(XB.astype(np.float32)) * ys
    nr = trueB.shape[1]
    mlp = cubB + p[:, :nr] + 1j * p[:, nr:]
    out = {}
    for name, v in (("hold", holdB), ("cubic", cubB), ("c+mlp", mlp)):
        e = np.abs(v - trueB).max(axis=1)
        out[name] = (float(np.median(e)), float(e.max()))
    return out


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--relax", action="store_true")
    ap.add_argument("--epochs", type=int, default=300)
    a = ap.parse_args()
    for k, (med, mx) in run(a.relax, a.epochs).items():
        print("%-6s median %.3e  max %.3e" % (k, med, mx))
