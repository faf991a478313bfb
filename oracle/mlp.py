"""CPU reference of the learned mean-field predictor's network (test infrastructure).

A fully connected network of `depth` linear layers with tanh between them:
    h_0 = x,  h_k = tanh(W_k h_{k-1} + b_k) (k < depth),  y = W_depth h_{depth-1} + b_depth,
trained on the mean squared error with Adam (Kingma and Ba, 2015: first and
second moment estimates with bias correction).  The backward pass is written out
by hand (chain rule through tanh: d tanh(u) = 1 - tanh(u)^2), so the device
training kernels can be checked against it value by value; `grad_check`
compares it with central differences.

Arithmetic is in the dtype of the parameters (float64 for the checks, float32 as
the device keeps its weights); `bf16` rounds the inputs and weights of a forward
pass to bfloat16 (round to nearest even), the device's inference precision.
Nothing in the product imports this module.
"""
import numpy as np

# Lagrange weights of the cubic through the step offsets tau = 0, -1, -2, -3 (latest history value
# first), evaluated at tau = c: the extrapolation the predictor's weights start from
CUBIC = {1.0: np.array([4.0, -6.0, 4.0, -1.0]), 0.5: np.array([2.1875, -2.1875, 1.3125, -0.3125])}


def bf16_round(a):
    """Round float32 values to the nearest bfloat16 (ties to even), returned as float32."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32)
    return np.where(np.isfinite(a), out, a)


class MLP:
    def __init__(self, sizes, seed=0, dtype=np.float64):
        """sizes = [n_in, width, ..., n_out] (depth = len(sizes) - 1 linear layers); weights
        scaled by 1/sqrt(fan_in) from a seeded normal draw, biases zero."""
        rng = np.random.default_rng(seed)
        self.dtype = dtype
        self.W = [(rng.standard_normal((o, i)) / np.sqrt(i)).astype(dtype) for i, o in zip(sizes[:-1], sizes[1:])]
        self.b = [np.zeros(o, dtype=dtype) for o in sizes[1:]]
        self.m = [np.zeros_like(p) for p in self.W + self.b]
        self.v = [np.zeros_like(p) for p in self.W + self.b]
        self.t = 0

    def forward(self, x, bf16=False, keep=False):
        """x [batch, n_in] -> y [batch, n_out]; keep=True also returns the activations."""
        h = np.asarray(x, dtype=self.dtype)
        acts = [h]
        for k, (W, b) in enumerate(zip(self.W, self.b)):
            if bf16:
                u = bf16_round(h) @ bf16_round(W).T + b.astype(np.float32)
            else:
                u = h @ W.T + b
            h = np.tanh(u) if k < len(self.W) - 1 else u
            acts.append(h)
        return (h, acts) if keep else h

    def loss_grad(self, x, y):
        """Mean squared error 0.5 mean_batch sum_out (f(x) - y)^2 and its gradients
        (dW_k, db_k) by the hand-written backward pass."""
        out, acts = self.forward(x, keep=True)
        n = x.shape[0]
        g = (out - y) / n
        loss = 0.5 * float(np.sum((out - y) ** 2)) / n
        dW, db = [None] * len(self.W), [None] * len(self.W)
        for k in range(len(self.W) - 1, -1, -1):
            dW[k] = g.T @ acts[k]
            db[k] = g.sum(axis=0)
            if k > 0:
                g = (g @ self.W[k]) * (1.0 - acts[k] ** 2)
        return loss, dW, db

    def adam_step(self, dW, db, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8):
        self.t += 1
        params, grads = self.W + self.b, dW + db
        c1, c2 = 1.0 - beta1 ** self.t, 1.0 - beta2 ** self.t
        for p, g, m, v in zip(params, grads, self.m, self.v):
            m *= beta1
            m += (1.0 - beta1) * g
            v *= beta2
            v += (1.0 - beta2) * g * g
            p -= lr * (m / c1) / (np.sqrt(v / c2) + eps)

    def grad_check(self, x, y, h=1e-6, samples=20, seed=1):
        """Largest relative difference between the backward pass and central differences over
        `samples` random parameter entries of every layer."""
        rng = np.random.default_rng(seed)
        _, dW, db = self.loss_grad(x, y)
        worst = 0.0
        for P, G in list(zip(self.W, dW)) + list(zip(self.b, db)):
            flat, gflat = P.reshape(-1), G.reshape(-1)
            for idx in rng.integers(0, flat.size, size=samples):
                keep = flat[idx]
                flat[idx] = keep + h
                lp = self.loss_grad(x, y)[0]
                flat[idx] = keep - h
                lm = self.loss_grad(x, y)[0]
                flat[idx] = keep
                fd = (lp - lm) / (2 * h)
                worst = max(worst, abs(fd - gflat[idx]) / max(abs(fd), abs(gflat[idx]), 1e-12))
        return worst
