"""CPU FP64 oracle of the nucleation-rate surrogate network.

TEST INFRASTRUCTURE ONLY: the surrogate's GPU tests use this module as the
checker; the product path never imports it.

The surrogate has no counterpart in the reference (the reference estimates
nucleation by running lattices); this file restates the network's own
mathematics so that the hand-written tensor-core kernels can be checked:

* layers 16 -> 128 -> 128 -> 128 -> 32 (6 input features zero-padded to 16,
  17 outputs zero-padded to 32), SiLU after the three hidden layers;
* parameters in one float32 vector, per layer W[in][out] then b[out];
* the GPU kernels multiply BF16 operands (round-to-nearest-even of the FP32
  activations, weights and output gradients) and accumulate in FP32;
  ``bf16=True`` reproduces those roundings here while accumulating in FP64;
* loss per row (targets row t = [event, exposure, w_gamma, w_curve, f_1..f_16]):
  w_gamma * (exp(l) * exposure - event * l) + w_curve / 16 * sum_k BCE(o_k, f_k)
  with l = y[0] clamped to [-40, 40] inside the exponential (the censored
  exponential negative log-likelihood of a first-passage time) and
  BCE(o, f) = softplus(o) - f o on the 16 converted-fraction logits y[1..16];
  the mean is taken over ``norm`` rows;
* Adam with bias correction and decoupled weight decay.

``grad_fd`` (central finite differences of the FP64 loss) pins the analytic
gradient ``loss_and_grad``.
"""
from __future__ import annotations

import numpy as np

IN_FEATURES = 6
N_OUT = 17
DIMS = (16, 128, 128, 128, 32)
N_CURVE = 16
TGT_COLS = 4 + N_CURVE
L_CLAMP = 40.0


def layout():
    """[(W offset, b offset, in, out)] per layer and the total parameter count."""
    out, off = [], 0
    for i in range(4):
        fi, fo = DIMS[i], DIMS[i + 1]
        out.append((off, off + fi * fo, fi, fo))
        off += fi * fo + fo
    return out, off


def bf16(x):
    """Round float values to bfloat16 (nearest, ties to even) and back to float64."""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    r = r.astype(np.uint32)
    nan = np.isnan(f)
    r = np.where(nan, np.uint32(0x7FC00000), r)
    return r.view(np.float32).astype(np.float64)


def f32(x):
    return np.asarray(x, dtype=np.float32).astype(np.float64)


def unpack(params):
    lay, _ = layout()
    p = np.asarray(params, dtype=np.float64)
    return [(p[w:b].reshape(fi, fo), p[b:b + fo]) for (w, b, fi, fo) in lay]


def sigmoid(z):
    return 0.5 * (1.0 + np.tanh(0.5 * z))


def silu(z):
    return z * sigmoid(z)


def pad_x(x):
    x = np.asarray(x, dtype=np.float64)
    xp = np.zeros((x.shape[0], DIMS[0]))
    xp[:, :IN_FEATURES] = x
    return xp


def forward(params, x, *, bf16_ops=True):
    """Returns (y[rows][17], cache).  With bf16_ops the matrix operands are rounded as on
    the GPU (inputs and SiLU outputs from FP32 values, weights from FP32)."""
    layers = unpack(params)
    rnd = bf16 if bf16_ops else (lambda a: a)
    h = rnd(f32(pad_x(x)))
    zs, hs = [], [h]
    for li, (W, b) in enumerate(layers):
        z = h @ rnd(W) + b
        if bf16_ops:
            z = f32(z)
        zs.append(z)
        if li < 3:
            h = rnd(f32(silu(z))) if bf16_ops else silu(z)
            hs.append(h)
    y = zs[-1][:, :N_OUT]
    return y, {"zs": zs, "hs": hs}


def row_loss_and_dy(y, tgt, norm):
    """Per-row loss and dL/dy (mean over norm rows) of the surrogate objective."""
    y = np.asarray(y, dtype=np.float64)
    t = np.asarray(tgt, dtype=np.float64)
    ev, ex, wg, wc = t[:, 0], t[:, 1], t[:, 2], t[:, 3]
    f = t[:, 4:4 + N_CURVE]
    l = y[:, 0]
    lc = np.clip(l, -L_CLAMP, L_CLAMP)
    E = np.exp(lc)
    inside = np.abs(l) < L_CLAMP
    lg = wg * (E * ex - ev * l)
    o = y[:, 1:1 + N_CURVE]
    sp = np.maximum(o, 0.0) + np.log1p(np.exp(-np.abs(o)))
    lcurve = wc / N_CURVE * (sp - f * o).sum(axis=1)
    dy = np.zeros_like(y)
    dy[:, 0] = wg * (np.where(inside, E, 0.0) * ex - ev) / norm
    dy[:, 1:1 + N_CURVE] = (wc / N_CURVE)[:, None] * (sigmoid(o) - f) / norm
    return lg + lcurve, dy


def loss_and_grad(params, x, tgt, norm=None, *, bf16_ops=True):
    """(mean loss, per-row losses, gradient vector) by reverse-mode differentiation.

    With bf16_ops the backward pass rounds its matrix operands as the GPU kernels do:
    dW = bf16(H)^T bf16(dZ), dH = bf16(dZ) bf16(W)^T, db = sum dZ (FP32 values)."""
    rows = np.asarray(x).shape[0]
    norm = rows if norm is None else norm
    layers = unpack(params)
    rnd = bf16 if bf16_ops else (lambda a: a)
    y, cache = forward(params, x, bf16_ops=bf16_ops)
    lrow, dy = row_loss_and_dy(y, tgt, norm)
    lay, total = layout()
    g = np.zeros(total)
    dz = np.zeros((rows, DIMS[4]))
    dz[:, :N_OUT] = dy
    if bf16_ops:
        dz = f32(dz)
    for li in range(3, -1, -1):
        w_off, b_off, fi, fo = lay[li]
        W, _ = layers[li]
        h_in = cache["hs"][li]
        g[w_off:b_off] = (h_in.T @ rnd(dz)).reshape(-1)
        g[b_off:b_off + fo] = dz.sum(axis=0)
        if li > 0:
            dh = rnd(dz) @ rnd(W).T
            z = cache["zs"][li - 1]
            s = sigmoid(z)
            dz = dh * (s * (1.0 + z * (1.0 - s)))
            if bf16_ops:
                dz = f32(dz)
    return float(lrow.sum() / norm), lrow, g


def grad_fd(params, x, tgt, idx, eps=1e-6, norm=None):
    """Central finite differences of the FP64 loss (no BF16 rounding) at parameter idx."""
    out = []
    p = np.asarray(params, dtype=np.float64)
    for i in idx:
        a = p.copy()
        a[i] += eps
        b = p.copy()
        b[i] -= eps
        la, _, _ = loss_and_grad(a, x, tgt, norm, bf16_ops=False)
        lb, _, _ = loss_and_grad(b, x, tgt, norm, bf16_ops=False)
        out.append((la - lb) / (2 * eps))
    return np.array(out)


def adam(params, grad, m, v, step, lr, beta1=0.9, beta2=0.999, eps=1e-8, wd=0.0):
    """One Adam update (step counts from 1); returns new (params, m, v)."""
    p = np.asarray(params, np.float64)
    g = np.asarray(grad, np.float64)
    m = beta1 * np.asarray(m, np.float64) + (1 - beta1) * g
    v = beta2 * np.asarray(v, np.float64) + (1 - beta2) * g * g
    mh = m / (1 - beta1 ** step)
    vh = v / (1 - beta2 ** step)
    p = p - lr * (mh / (np.sqrt(vh) + eps) + wd * p)
    return p, m, v


def init_params(seed=0, out_bias=None):
    """He-normal hidden weights, small output weights; padded rows/columns zero."""
    rng = np.random.default_rng(seed)
    lay, total = layout()
    p = np.zeros(total, np.float32)
    for li, (w, b, fi, fo) in enumerate(lay):
        fan_in = IN_FEATURES if li == 0 else fi
        W = np.zeros((fi, fo))
        scale = np.sqrt(2.0 / fan_in) if li < 3 else 0.1 / np.sqrt(fan_in)
        W[:fan_in if li == 0 else fi, :N_OUT if li == 3 else fo] = rng.normal(
            0.0, scale, (fan_in if li == 0 else fi, N_OUT if li == 3 else fo))
        p[w:b] = W.reshape(-1)
        if li == 3 and out_bias is not None:
            p[b:b + N_OUT] = out_bias
    return p
