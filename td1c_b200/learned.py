"""Host side of the learned mean-field predictor: the device network and its training loop.

The network's arithmetic runs in libtd1c_b200.so (mlp.cu): FP32 forward and
hand-written backward passes, Adam, and BF16 inference on the tensor cores.
This module holds the parameters in device memory (torch tensors serve only as
allocations) and sequences the kernel calls.  The predictor it serves, the
judge and the fallback live in the library's learned split2 steps (hprod.cu);
the reference (td1c) has no learned component.
"""
import ctypes

import numpy as np

from . import _lib as _libmod


def _vp(t):
    return ctypes.c_void_p(t.data_ptr())


class DeviceMLP:
    """A stack of linear layers with tanh between them (widths sizes[0] .. sizes[-1]) whose FP32
    master weights, gradients and Adam moments live on the GPU."""

    def __init__(self, sizes, seed=0, device="cuda", weights=None):
        import torch
        self.lib = _libmod.load()
        self.torch = torch
        self.sizes = [int(s) for s in sizes]
        self.depth = len(self.sizes) - 1
        self.device = torch.device(device)
        rng = np.random.default_rng(seed)
        W, b = [], []
        for k, (i, o) in enumerate(zip(self.sizes[:-1], self.sizes[1:])):
            if weights is not None:
                w0, b0 = weights[0][k], weights[1][k]
            else:
                w0, b0 = rng.standard_normal((o, i)) / np.sqrt(i), np.zeros(o)
            W.append(torch.tensor(np.asarray(w0, dtype=np.float32), device=self.device))
            b.append(torch.tensor(np.asarray(b0, dtype=np.float32), device=self.device))
        self.W, self.b = W, b
        self.dW = [torch.zeros_like(w) for w in W]
        self.db = [torch.zeros_like(x) for x in b]
        self.mW = [torch.zeros_like(w) for w in W]
        self.vW = [torch.zeros_like(w) for w in W]
        self.mb = [torch.zeros_like(x) for x in b]
        self.vb = [torch.zeros_like(x) for x in b]
        self.step_count = 0
        self._sizes = (ctypes.c_int * len(self.sizes))(*self.sizes)
        self._pack = torch.empty(int(self.lib.td1c_mlp_pack_size(self.depth, self._sizes)), dtype=torch.uint8,
                                 device=self.device)
        self._packed = False
        self._status = torch.zeros(1, dtype=torch.int32, device=self.device)

    def _ptrs(self, ts):
        return (ctypes.c_void_p * len(ts))(*[t.data_ptr() for t in ts])

    def _stream(self):
        return ctypes.c_void_p(self.torch.cuda.current_stream(self.device).cuda_stream)

    def forward(self, x):
        """FP32 forward of x [rows x sizes[0]] (device float32); returns (output, activations)."""
        torch = self.torch
        rows = int(x.shape[0])
        acts = torch.empty(sum(rows * n for n in self.sizes[1:]), dtype=torch.float32, device=self.device)
        rc = self.lib.td1c_mlp_forward(self.depth, self._sizes, self._ptrs(self.W), self._ptrs(self.b), _vp(x), rows,
                                       _vp(acts), self._stream())
        if rc:
            raise RuntimeError("td1c_mlp_forward failed (%d)" % rc)
        out = acts[-rows * self.sizes[-1]:].view(rows, self.sizes[-1])
        return out, acts

    def backward(self, x, acts, dy):
        """Gradients of the parameters for the output gradient dy [rows x sizes[-1]] into dW, db."""
        torch = self.torch
        rows = int(x.shape[0])
        work = torch.empty(2 * rows * max(self.sizes), dtype=torch.float32, device=self.device)
        rc = self.lib.td1c_mlp_backward(self.depth, self._sizes, self._ptrs(self.W), _vp(x), rows, _vp(acts),
                                        _vp(dy.contiguous()), self._ptrs(self.dW), self._ptrs(self.db), _vp(work),
                                        self._stream())
        if rc:
            raise RuntimeError("td1c_mlp_backward failed (%d)" % rc)

    def adam_step(self, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8):
        self.step_count += 1
        for p, g, m, v in list(zip(self.W, self.dW, self.mW, self.vW)) + list(zip(self.b, self.db, self.mb, self.vb)):
            rc = self.lib.td1c_mlp_adam(p.numel(), _vp(p), _vp(g), _vp(m), _vp(v), lr, beta1, beta2, eps, self.step_count,
                                        self._stream())
            if rc:
                raise RuntimeError("td1c_mlp_adam failed (%d)" % rc)
        self._packed = False

    def infer_bf16(self, x, y=None):
        """BF16 tensor-core inference of x [rows x sizes[0]] into y [rows x sizes[-1]] (FP32)."""
        torch = self.torch
        rows = int(x.shape[0])
        if y is None:
            y = torch.empty(rows, self.sizes[-1], dtype=torch.float32, device=self.device)
        rc = self.lib.td1c_mlp_infer_bf16(self.depth, self._sizes, self._ptrs(self.W), self._ptrs(self.b), _vp(self._pack),
                                          0 if self._packed else 1, _vp(x), rows, _vp(y), _vp(self._status), self._stream())
        if rc:
            raise RuntimeError("td1c_mlp_infer_bf16 failed (%d)" % rc)
        self._packed = True
        return y

    def pack(self):
        """Refresh the BF16 copy of the weights that the predicted steps read (one inference call)."""
        torch = self.torch
        if not self._packed:
            x = torch.zeros(1, self.sizes[0], dtype=torch.float32, device=self.device)
            self.infer_bf16(x)
        return self._pack

    def status(self):
        return int(self._status.item())

    def numpy_weights(self):
        return [w.cpu().numpy() for w in self.W], [x.cpu().numpy() for x in self.b]


# ---------------------------------------------------------------------------
# training on recorded trajectories
# ---------------------------------------------------------------------------
SIZES = [32, 256, 256, 256, 8]  # the predictor's network: Gram features -> weight corrections, width 256, 4 layers


def new_predictor_net(seed=0, device="cuda"):
    """The predictor's network with a zero output layer, so that it starts as the cubic extrapolation."""
    net = DeviceMLP(SIZES, seed=seed, device=device)
    net.W[-1].zero_()
    net.b[-1].zero_()
    return net


class Records:
    """Training records on the device (per step and unit: Gram matrix, targets, norm) with the
    unit layout of the context that wrote them."""

    def __init__(self, h, steps_per_traj):
        import torch
        self.torch = torch
        d = h.learned_dims()
        self.nu, self.nfe, self.rec = d["nu"], d["nfe"], d["rec"]
        self.pair_kind = torch.tensor(h.learned_pair_kind(), device="cuda")
        self.steps = steps_per_traj
        self.chunks = []

    def new_buffer(self):
        return self.torch.zeros((self.steps + 1) * self.nu * self.rec, dtype=self.torch.float64, device="cuda")

    def add(self, buf, skip=4):
        """Keep the records of one trajectory after the first `skip` steps (history not yet full)."""
        self.chunks.append(buf.view(self.steps + 1, self.nu, self.rec)[skip:].reshape(-1, self.rec))

    def all(self):
        return self.torch.cat(self.chunks).contiguous()


def features(lib, rec, idx, nu, nfe, pair_kind, stream=None):
    import torch
    n = int(idx.numel()) if idx is not None else int(rec.shape[0])
    x = torch.empty(n, 32, dtype=torch.float32, device="cuda")
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream if stream is None else stream)
    rc = lib.td1c_lp_features(n, _vp(rec), _vp(idx) if idx is not None else None, nu, nfe, _vp(pair_kind), _vp(x), st)
    if rc:
        raise RuntimeError("td1c_lp_features failed (%d)" % rc)
    return x


def loss(lib, rec, idx, out, want_grad=True, use_net=True):
    """Per-sample relative squared error (FP64) and the gradient of its mean w.r.t. the network output."""
    import torch
    n = int(idx.numel()) if idx is not None else int(rec.shape[0])
    per = torch.empty(n, dtype=torch.float64, device="cuda")
    dy = torch.empty(n, 8, dtype=torch.float32, device="cuda") if want_grad else None
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = lib.td1c_lp_loss(n, _vp(rec), _vp(idx) if idx is not None else None, _vp(out) if out is not None else None,
                          _vp(dy) if dy is not None else None, _vp(per), 1 if use_net else 0, st)
    if rc:
        raise RuntimeError("td1c_lp_loss failed (%d)" % rc)
    return per, dy


def evaluate(net, rec, nu, nfe, pair_kind, batch=65536):
    """Median and root-mean-square relative error of the one-step prediction over the records: with the
    network (BF16 inference, as the steps run it) and with the cubic alone."""
    import torch
    lib = net.lib
    errs_net, errs_cub = [], []
    for b0 in range(0, rec.shape[0], batch):
        idx = torch.arange(b0, min(b0 + batch, rec.shape[0]), dtype=torch.int32, device="cuda")
        x = features(lib, rec, idx, nu, nfe, pair_kind)
        out = net.infer_bf16(x)
        e, _ = loss(lib, rec, idx, out, want_grad=False)
        c, _ = loss(lib, rec, idx, None, want_grad=False, use_net=False)
        errs_net.append(e)
        errs_cub.append(c)
    en, ec = torch.cat(errs_net), torch.cat(errs_cub)
    return {"net_median": float(en.median().sqrt()), "net_rms": float(en.mean().sqrt()),
            "cubic_median": float(ec.median().sqrt()), "cubic_rms": float(ec.mean().sqrt())}


def train(net, rec, nu, nfe, pair_kind, steps=400, batch=4096, lr=3e-4, seed=0, robust=True):
    """Adam on the one-step prediction error; returns the objective on a fixed evaluation batch of
    the training records, before training and at about twenty points on the way.

    The per-record loss L is the relative squared error of a unit's prediction. Its mean is ruled by
    a heavy tail (units where the mean field is small), so by default the objective is
    mean(log(1 + L / eps)) with eps the median L of the evaluation batch before training (the
    cubic's typical error): the gradient of the mean (from the loss kernel) is scaled per record by
    1 / (eps + L), which weighs the typical unit as much as the tail. robust=False minimises mean(L).
    With the robust objective a useful learning rate is about the typical relative error over the
    output scale of the correction (1e-3) and the width: 1e-5 for the Ne records. The weights with
    the lowest evaluation objective are kept (the zero-output start, the cubic, included), so the
    returned network is never worse than the cubic on that batch."""
    import torch
    lib = net.lib
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    n_eval = min(int(rec.shape[0]), 16384)
    idx_eval = torch.randperm(int(rec.shape[0]), generator=g, device="cuda")[:n_eval].to(torch.int32)
    x_eval = features(lib, rec, idx_eval, nu, nfe, pair_kind)
    per0, _ = loss(lib, rec, idx_eval, net.forward(x_eval)[0], want_grad=False)
    eps = max(float(per0.median()), 1e-300)

    def objective(per):
        return torch.log1p(per / eps).mean() if robust else per.mean()

    def evaluate_now():
        out, _ = net.forward(x_eval)
        per, _ = loss(lib, rec, idx_eval, out, want_grad=False)
        return float(objective(per))

    best = evaluate_now()
    curve = [best]
    keep = ([w.clone() for w in net.W], [b.clone() for b in net.b])
    warm = max(1, steps // 10)
    for it in range(steps):
        idx = torch.randint(0, rec.shape[0], (batch,), generator=g, device="cuda", dtype=torch.int64).to(torch.int32)
        x = features(lib, rec, idx, nu, nfe, pair_kind)
        out, acts = net.forward(x)
        per, dy = loss(lib, rec, idx, out)
        if robust:
            dy = dy * (1.0 / (eps + per)).to(torch.float32)[:, None]
        net.backward(x, acts, dy)
        # a linear warm-up over the first tenth of the steps, from lr / 10
        net.adam_step(lr=lr * min(1.0, 0.1 + 0.9 * it / warm))
        if (it + 1) % max(1, steps // 20) == 0 or it == steps - 1:
            cur = evaluate_now()
            curve.append(cur)
            if cur < best:
                best = cur
                keep = ([w.clone() for w in net.W], [b.clone() for b in net.b])
    for w, k in zip(net.W, keep[0]):
        w.copy_(k)
    for b, k in zip(net.b, keep[1]):
        b.copy_(k)
    net._packed = False  # the BF16 copy follows the kept weights at the next inference
    return curve
