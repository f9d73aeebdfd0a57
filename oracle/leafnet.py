"""CPU restatement of the turn-leaf value network (test infrastructure only:
the checker the GPU tests compare the tcgen05 kernels with, never a product
path).

The reference has no learned leaf; this is the network its depth-limited
configuration describes -- inputs (board one-hot, pot/stack, both ranges),
hidden GELU layers, linear counterfactual-value outputs -- with the device
path's arithmetic: inputs, weights and hidden activations rounded to bf16
(round to nearest even), products accumulated in f32 (here f64, then f32),
bias adds, GELU(z) = z * Phi(z) and GELU'(z) = Phi(z) + z * phi(z), the loss
mean(mask * (y - t)^2) over rows x outputs, and its gradient rounded to bf16
where the device feeds it to a matrix product.
"""
import math

import numpy as np

_erf = np.vectorize(math.erf, otypes=[np.float64])


def bf16_round(x):
    """f32 values rounded to the nearest bf16 (ties to even), as f32."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32)


def bf16_bits(x):
    """bf16 bit patterns (uint16) of f32 values, ties to even."""
    return (bf16_round(x).view(np.uint32) >> 16).astype(np.uint16)


def from_bf16_bits(b):
    return (np.asarray(b, np.uint16).astype(np.uint32) << 16).view(np.float32)


def _mm(a, b_t):
    """a @ b_t.T accumulated in f64, rounded to f32."""
    return (a.astype(np.float64) @ b_t.astype(np.float64).T).astype(np.float32)


def gelu(z):
    z64 = z.astype(np.float64)
    return (0.5 * z64 * (1.0 + _erf(z64 / math.sqrt(2.0)))).astype(np.float32)


def gelu_grad(z):
    z64 = z.astype(np.float64)
    cdf = 0.5 * (1.0 + _erf(z64 / math.sqrt(2.0)))
    pdf = np.exp(-0.5 * z64 * z64) / math.sqrt(2.0 * math.pi)
    return (cdf + z64 * pdf).astype(np.float32)


def forward(params, x, keep=False):
    """params: [(W [out x in], b [out])] per layer, the last one linear."""
    h = bf16_round(np.asarray(x, np.float32))
    acts = [h]
    zs = []
    for l, (w, b) in enumerate(params):
        z = _mm(h, bf16_round(w)) + np.asarray(b, np.float32)
        if l == len(params) - 1:
            return (z, acts, zs) if keep else z
        zs.append(z)
        h = bf16_round(gelu(z))
        acts.append(h)


def gradients(params, x, t, mask):
    """(loss, [(dW, db)] per layer) of mean(mask * (y - t)^2)."""
    y, acts, zs = forward(params, x, keep=True)
    rows, dout = y.shape
    inv = np.float32(1.0 / (rows * dout))
    d = (y - t) * mask
    loss = float(np.sum(d.astype(np.float64) ** 2) * inv)
    g = (np.float32(2.0) * d * inv).astype(np.float32)
    grads = [None] * len(params)
    for l in range(len(params) - 1, -1, -1):
        gb16 = bf16_round(g)
        dw = _mm(gb16.T, acts[l].T)
        db = g.sum(axis=0, dtype=np.float64).astype(np.float32)
        grads[l] = (dw, db)
        if l > 0:
            dh = _mm(gb16, bf16_round(params[l][0]).T)
            g = (dh * gelu_grad(zs[l - 1])).astype(np.float32)
    return loss, grads


def gradients_f64(params, x, t, mask):
    """The same loss and gradients in plain f64 with no bf16 rounding: the
    reference for a finite-difference check of the formulas."""
    p64 = [(np.asarray(w, np.float64), np.asarray(b, np.float64)) for w, b in params]
    h = np.asarray(x, np.float64)
    acts, zs = [h], []
    for l, (w, b) in enumerate(p64):
        z = h @ w.T + b
        if l == len(p64) - 1:
            y = z
            break
        zs.append(z)
        h = 0.5 * z * (1.0 + _erf(z / math.sqrt(2.0)))
        acts.append(h)
    rows, dout = y.shape
    d = (y - t) * mask
    loss = float(np.sum(d * d) / (rows * dout))
    g = 2.0 * d / (rows * dout)
    grads = [None] * len(p64)
    for l in range(len(p64) - 1, -1, -1):
        grads[l] = (g.T @ acts[l], g.sum(axis=0))
        if l > 0:
            z = zs[l - 1]
            gp = 0.5 * (1.0 + _erf(z / math.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / math.sqrt(2.0 * math.pi)
            g = (g @ p64[l][0]) * gp
    return loss, grads
