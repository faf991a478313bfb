"""The learned predictor's network kernels on the device against the CPU reference network.

oracle/mlp.py states the network (linear layers, tanh), its hand-written
backward pass (checked there against central differences) and Adam.  Here the
device kernels (mlp.cu) start from the same weights and must agree with it:
- the FP32 forward pass, to FP32 rounding (1e-5 relative);
- the gradients of the mean squared error, to 1e-4 relative (the device sums
  in FP32, the reference in FP64);
- one Adam step, to 1e-5 relative on the updated weights;
- the BF16 tensor-core inference (tcgen05 kind::f16, FP32 accumulation)
  against the reference's own BF16 forward (operands rounded to bfloat16 at
  every layer), to 2e-3 relative: the two differ only in the order of the FP32
  accumulation and the rounding of intermediate activations it feeds.
The shapes are the predictor's (width 256, 4 layers) with a row count that
leaves a partial 128-row tile.
"""
import numpy as np
import pytest

from td1c_b200 import workloads as W

SIZES = [24, 256, 256, 256, 8]


def _rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-30))


@pytest.mark.gpu
def test_device_network_matches_reference(cuda_ok):
    import torch
    from oracle.mlp import MLP
    from td1c_b200.learned import DeviceMLP
    rng = np.random.default_rng(11)
    ref = MLP(SIZES, seed=3, dtype=np.float64)
    # weights representable in FP32, so both sides start from identical values
    ref.W = [w.astype(np.float32).astype(np.float64) for w in ref.W]
    ref.b = [rng.standard_normal(b.shape).astype(np.float32).astype(np.float64) * 0.1 for b in ref.b]
    dev = DeviceMLP(SIZES, weights=(ref.W, ref.b))
    rows = 300
    x = rng.standard_normal((rows, SIZES[0])).astype(np.float32)
    y = rng.standard_normal((rows, SIZES[-1])).astype(np.float32)
    xt = torch.tensor(x, device="cuda")
    # forward
    out, acts = dev.forward(xt)
    ref_out = ref.forward(x.astype(np.float64))
    assert _rel(out.cpu().numpy(), ref_out) < 1e-5
    # backward of 0.5 mean sum (f - y)^2
    dy = (out - torch.tensor(y, device="cuda")) / rows
    dev.backward(xt, acts, dy)
    _, dW, db = ref.loss_grad(x.astype(np.float64), y.astype(np.float64))
    for k in range(len(SIZES) - 1):
        assert _rel(dev.dW[k].cpu().numpy(), dW[k]) < 1e-4, k
        assert _rel(dev.db[k].cpu().numpy(), db[k]) < 1e-4, k
    # one Adam step from the same gradients
    dev.dW = [torch.tensor(g.astype(np.float32), device="cuda") for g in dW]
    dev.db = [torch.tensor(g.astype(np.float32), device="cuda") for g in db]
    ref.adam_step(dW, db, lr=1e-3)
    dev.adam_step(lr=1e-3)
    Wd, bd = dev.numpy_weights()
    for k in range(len(SIZES) - 1):
        assert _rel(Wd[k], ref.W[k]) < 1e-5 and _rel(bd[k], ref.b[k]) < 1e-5, k
    # BF16 inference on the tensor cores against the reference's BF16 forward (updated weights)
    ref32 = MLP(SIZES, seed=0, dtype=np.float32)
    ref32.W = [w.astype(np.float32) for w in Wd]
    ref32.b = [x_.astype(np.float32) for x_ in bd]
    yi = dev.infer_bf16(xt)
    torch.cuda.synchronize()
    assert dev.status() == 0
    assert _rel(yi.cpu().numpy(), ref32.forward(x, bf16=True)) < 2e-3
    # and it is not just the FP32 result: BF16 rounding shows at the 1e-3 level
    assert _rel(yi.cpu().numpy(), ref32.forward(x)) > 1e-5


def _learned_setup(base):
    import torch
    from oracle.oracle import Oracle
    from td1c_b200.hprod import HProd
    from .helpers import oracle_tables, oracle_state
    wl = dict(base, split_type=1)
    o = Oracle(wl)
    o.set_split(1)
    rad, ang = oracle_tables(o)
    h = HProd(wl, rad, ang)
    orb, cic = oracle_state(o)
    h.set_wfn0(orb, cic)
    orb, cic = o.orth(orb, cic)
    freq = 1239.84190 / (wl["wlen"] * 27.2113845)
    t0 = 0.4 * wl["numcyc"] * 2 * np.pi / freq
    A0 = h.pulse_lfield(t0)[2]
    if A0 != 0.0:
        from td1c_b200.wfn import velocity_gauge_phase
        orb = velocity_gauge_phase(wl, orb.reshape(len(wl["orbitals"]), wl["lmax1"] + 1, -1), rad, ang, A0)
    d_orb = torch.from_numpy(np.ascontiguousarray(orb).reshape(-1).copy()).cuda()
    d_cic = torch.from_numpy(cic.copy()).cuda()
    return h, wl, d_orb, d_cic, t0


@pytest.mark.gpu
def test_learned_fallback_reproduces_split2(cuda_ok):
    """Bound 0 rejects every predicted window: the driver returns to each window's start and
    recomputes it with exact steps, so the result is the plain FP64 split2 trajectory."""
    h, wl, d_orb, d_cic, t0 = _learned_setup(W.MIXED_SMALL)
    try:
        dt, n = 0.002, 48
        ref_o, ref_c = d_orb.clone(), d_cic.clone()
        start_o, start_c = d_orb.clone(), d_cic.clone()
        h.split2_dev(ref_o.data_ptr(), ref_c.data_ptr(), t0, dt, n)
        h.set_learned(None, bound=0.0)
        # without screening every predicted window is tried, judged (values > 0) and rolled back
        h.set_learned_policy(screen=False)
        st = h.split2_learned_dev(d_orb.data_ptr(), d_cic.data_ptr(), t0, dt, n)
        h.sync()
        assert st["steps"] == n and st["rejected"] >= 1 and st["accepted"] == 0, st
        assert st["min_judge"] > 0.0
        e = float((d_orb - ref_o).abs().max() / ref_o.abs().max())
        ec = float((d_cic - ref_c).abs().max() / ref_c.abs().max())
        assert e <= 1e-12 and ec <= 1e-12, (e, ec)
        # with screening (the default) the fill windows' judges keep predicted windows from being tried
        h.set_learned_policy(screen=True)
        o2, c2 = start_o.clone(), start_c.clone()
        st2 = h.split2_learned_dev(o2.data_ptr(), c2.data_ptr(), t0, dt, n)
        h.sync()
        assert st2["rejected"] == 0 and st2["accepted"] == 0 and st2["fills"] >= 1, st2
        assert float((o2 - ref_o).abs().max() / ref_o.abs().max()) <= 1e-12
        assert h.last_status() == 0
    finally:
        h.final()


@pytest.mark.gpu
def test_learned_records_match_host_gram(cuda_ok):
    """The judge's per-unit quantities (Gram matrix of the four previous step-start pair potentials,
    their products with the new one, its norm) against a host computation from the exact W(y_n)."""
    import torch
    h, wl, d_orb, d_cic, t0 = _learned_setup(W.NE_SMALL)
    try:
        dt, n = 0.002, 8
        d = h.learned_dims()
        nu, nfe, nrec = d["nu"], d["nfe"], d["rec"]
        rec = torch.zeros((n + 1) * nu * nrec, dtype=torch.float64, device="cuda")
        y0o, y0c = d_orb.clone(), d_cic.clone()
        h.learned_record_dev(d_orb.data_ptr(), d_cic.data_ptr(), t0, dt, n, rec.data_ptr())
        h.sync()
        rec = rec.view(n + 1, nu, nrec).cpu().numpy()
        # host: W(y_s) of the exact trajectory (the RHS at y_s forms it), one split2 step at a time
        Ws = []
        yo, yc = y0o.clone(), y0c.clone()
        hw, hc = torch.empty_like(yo), torch.empty_like(yc)
        for s in range(n + 1):
            h.htot_dev(1.0, h.pulse_lfield(t0 + s * dt), yo.data_ptr(), yc.data_ptr(), hw.data_ptr(), hc.data_ptr())
            h.sync()
            Ws.append(h.debug("W").copy())
            if s < n:
                h.split2_dev(yo.data_ptr(), yc.data_ptr(), t0 + s * dt, dt, 1, use_graph=False)
        npair = d["npair"]
        nd, Nr, nlat = h.dims["ndvr"], h.dims["nrad"] - 1, h.dims["nlat"]
        Wv = [w.reshape(npair, nlat, Nr) for w in Ws]
        worst = 0.0
        for s in range(4, n + 1):
            for u in range(0, nu, max(1, nu // 17)):
                p, e = u // nfe, u % nfe
                sl = slice(e * nd, min((e + 1) * nd, Nr))
                x = [Wv[s - 1 - h_][p][:, sl].ravel() for h_ in range(4)]
                new = Wv[s][p][:, sl].ravel()
                G = np.array([[np.vdot(x[i], x[j]) for j in range(4)] for i in range(4)])
                g = np.array([np.vdot(x[i], new) for i in range(4)])
                t = np.vdot(new, new).real
                r = rec[s, u]
                Gd = (r[0:32:2] + 1j * r[1:32:2]).reshape(4, 4)
                gd = r[32:40:2] + 1j * r[33:40:2]
                scale = max(np.abs(G).max(), 1e-300)
                worst = max(worst, np.abs(Gd - G).max() / scale, np.abs(gd - g).max() / scale, abs(r[40] - t) / scale)
        assert worst < 1e-12, worst
    finally:
        h.final()


@pytest.mark.gpu
def test_learned_training_and_prediction(cuda_ok):
    """Records from exact trajectories train the network on the GPU (the loss falls); with the bound
    open the driver keeps predicted windows and the trajectory stays finite, and the network's
    one-step error on held-out records is reported next to the cubic's."""
    import torch
    from td1c_b200 import learned as L
    h, wl, d_orb, d_cic, t0 = _learned_setup(W.MIXED_SMALL)
    try:
        dt, n = 0.002, 24
        R = L.Records(h, n)
        start_o, start_c = d_orb.clone(), d_cic.clone()
        for k, (fint, wlen) in enumerate([(1e14, 800.0), (2e14, 700.0), (5e13, 900.0)]):
            buf = R.new_buffer()
            yo, yc = start_o.clone(), start_c.clone()
            h.learned_record_dev(yo.data_ptr(), yc.data_ptr(), t0 + 3 * k * dt, dt, n, buf.data_ptr(), fint=fint, wlen=wlen)
            h.sync()
            R.add(buf)
        rec = R.all()
        ntrain = (rec.shape[0] // R.nu * 2 // 3) * R.nu
        net = L.new_predictor_net(seed=1)
        curve = L.train(net, rec[:ntrain], R.nu, R.nfe, R.pair_kind, steps=150, batch=2048, lr=1e-5)
        # the objective starts at the cubic's (zero output layer); the kept weights are the best seen
        assert np.all(np.isfinite(curve)) and len(curve) >= 2, curve
        assert min(curve) <= curve[0], curve
        ev = L.evaluate(net, rec[ntrain:].contiguous(), R.nu, R.nfe, R.pair_kind)
        assert np.isfinite(ev["net_rms"]) and np.isfinite(ev["cubic_rms"]), ev
        print("held-out one-step relative error:", ev)
        h.set_learned(net, use_net=True, bound=1e9)
        st = h.split2_learned_dev(d_orb.data_ptr(), d_cic.data_ptr(), t0, dt, 40)
        h.sync()
        assert st["accepted"] >= 1 and st["predicted_steps"] >= 8, st
        assert bool(torch.isfinite(d_orb).all()) and h.last_status() == 0
    finally:
        h.final()
