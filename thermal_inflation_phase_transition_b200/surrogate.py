"""Surrogate of the nucleation rate and the converted-fraction curve.

No reference counterpart: the reference estimates nucleation only by running
lattices.  ``SurrogateNet`` is a 6 -> 128 -> 128 -> 128 -> 17 SiLU network whose
forward, backward and Adam kernels are this library's own (``tipt_mlp_*``:
BF16 tensor-core products, FP32 accumulation, deterministic reductions).

Inputs (``features``): T/T0, E, D, lam, log lattice volume, dimension, each
mapped to about [-1, 1].  Outputs: y[0] = log(Gamma * u) with Gamma the
nucleation rate per unit volume and time and u = ``exposure_unit`` (volume x
time), and y[1..16] = logits of the converted fraction at 16 fixed times
t_k = (k + 1) / 16 * horizon.

Training rows come from the ensemble engine (one row per replica): the event
flag and exposure (volume x time to first passage, or to censoring) enter the
censored exponential likelihood of the rate, the replica's converted-fraction
curve the cross-entropy of the curve logits.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from . import _lib as L
from ._common import ptr, stream_handle

__all__ = ["SurrogateNet", "features", "init_params", "N_CURVE", "PARAM_BOX"]

N_IN = 6
N_OUT = 17
N_CURVE = 16
TGT_COLS = 4 + N_CURVE
DIMS = (16, 128, 128, 128, 32)

# parameter box of the scan and the centring/scaling of the features
PARAM_BOX = {"T": (0.97, 1.02), "E": (0.03, 0.07), "D": (0.05, 0.15), "lam": (0.05, 0.2)}
_LOGV_CENTRE, _LOGV_SCALE = 12.0, 2.0


def features(T_over_T0, E, D, lam, volume, dim):
    """Normalised network inputs [rows][6] (float32) from physical parameters."""
    cols = []
    for v, key in ((T_over_T0, "T"), (E, "E"), (D, "D"), (lam, "lam")):
        lo, hi = PARAM_BOX[key]
        cols.append((np.asarray(v, np.float64) - 0.5 * (lo + hi)) / (0.5 * (hi - lo)))
    cols.append((np.log(np.asarray(volume, np.float64)) - _LOGV_CENTRE) / _LOGV_SCALE)
    cols.append(np.asarray(dim, np.float64) - 2.5)
    n = max(np.size(c) for c in cols)
    return np.stack([np.broadcast_to(c, (n,)) for c in cols], axis=1).astype(np.float32)


def layout():
    out, off = [], 0
    for i in range(4):
        fi, fo = DIMS[i], DIMS[i + 1]
        out.append((off, off + fi * fo, fi, fo))
        off += fi * fo + fo
    return out, off


def init_params(seed=0, out_bias=None):
    """He-normal hidden layers, small output layer; padding rows/columns are zero."""
    rng = np.random.default_rng(seed)
    lay, total = layout()
    p = np.zeros(total, np.float32)
    for li, (w, b, fi, fo) in enumerate(lay):
        rows = N_IN if li == 0 else fi
        cols = N_OUT if li == 3 else fo
        scale = math.sqrt(2.0 / rows) if li < 3 else 0.1 / math.sqrt(rows)
        W = np.zeros((fi, fo), np.float32)
        W[:rows, :cols] = rng.normal(0.0, scale, (rows, cols))
        p[w:b] = W.reshape(-1)
        if li == 3 and out_bias is not None:
            p[b:b + N_OUT] = np.asarray(out_bias, np.float32)
    return p


class SurrogateNet:
    """Parameters, Adam state and step counter on the device."""

    def __init__(self, params=None, *, seed=0, exposure_unit=1.0, horizon=1.0, device="cuda"):
        self.dev = torch.device(device)
        n = int(L.lib().tipt_mlp_param_count())
        p = init_params(seed) if params is None else np.asarray(params, np.float32)
        if p.shape != (n,):
            raise ValueError(f"expected {n} parameters, got {p.shape}")
        self.params = torch.from_numpy(p.copy()).to(self.dev)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.grad_buf = torch.zeros_like(self.params)
        self.counter = torch.zeros(1, dtype=torch.int64, device=self.dev)
        self.exposure_unit = float(exposure_unit)
        self.horizon = float(horizon)
        self._ws = None
        self._graphs = {}

    # ------------------------------------------------------------ kernels
    def forward(self, x):
        """y[rows][17] for x[rows][6] (device or host array)."""
        x = self._dev32(x, N_IN)
        y = torch.empty((x.shape[0], N_OUT), dtype=torch.float32, device=self.dev)
        L.call("tipt_mlp_forward", ptr(self.params), ptr(x), x.shape[0], ptr(y), stream_handle())
        return y

    def _workspace(self, rows):
        need = int(L.lib().tipt_mlp_workspace_size(rows))
        if self._ws is None or self._ws.numel() * 4 < need:
            self._ws = torch.empty(need // 4 + 4, dtype=torch.float32, device=self.dev)
        return self._ws

    def grad(self, x, tgt, norm=None, *, loss_rows=None, out=None):
        """Gradient of the mean loss (over norm rows, default all) into out (or grad_buf)."""
        x = self._dev32(x, N_IN)
        tgt = self._dev32(tgt, TGT_COLS)
        rows = x.shape[0]
        ws = self._workspace(rows)
        g = self.grad_buf if out is None else out
        L.call("tipt_mlp_grad", ptr(self.params), ptr(x), ptr(tgt), rows,
               float(rows if norm is None else norm), ptr(g),
               ptr(loss_rows) if loss_rows is not None else None, ptr(ws), ws.numel() * 4,
               stream_handle())
        return g

    def adam(self, grad, lr, *, lr_schedule=None, beta1=0.9, beta2=0.999, eps=1e-8,
             weight_decay=0.0, use_counter=True):
        """One Adam step; the step number comes from the device counter (advanced here)."""
        L.call("tipt_mlp_adam", ptr(self.params), ptr(grad), ptr(self.m), ptr(self.v),
               ptr(self.counter) if use_counter else None, 0, float(lr),
               ptr(lr_schedule) if lr_schedule is not None else None,
               int(lr_schedule.numel()) if lr_schedule is not None else 0, float(beta1),
               float(beta2), float(eps), float(weight_decay), stream_handle())
        if use_counter:
            L.call("tipt_counter_add", ptr(self.counter), 1, stream_handle())

    # ------------------------------------------------------------ training
    def fit(self, x, tgt, *, iters=2000, lr=2e-3, lr_final=1e-4, batch=4096, seed=0,
            weight_decay=0.0, graph_iters=50):
        """Adam on minibatches (a fresh random permutation per pass over the rows, drawn
        on the host); the learning rate decays geometrically from lr to lr_final through
        a device schedule indexed by the step counter, so one CUDA graph of graph_iters
        iterations is captured once and replayed.  Returns the mean loss per chunk."""
        x = self._dev32(x, N_IN)
        tgt = self._dev32(tgt, TGT_COLS)
        n = x.shape[0]
        batch = min(batch, n)
        iters = max(graph_iters, (iters // graph_iters) * graph_iters)
        rng = np.random.default_rng(seed)
        start = int(self.counter.item())
        sched = np.geomspace(1.0, lr_final / lr, iters).astype(np.float32)
        self._lr_sched = torch.from_numpy(np.concatenate([np.ones(start, np.float32), sched])
                                          ).to(self.dev)
        xb = torch.empty((graph_iters, batch, N_IN), dtype=torch.float32, device=self.dev)
        tb = torch.empty((graph_iters, batch, TGT_COLS), dtype=torch.float32, device=self.dev)
        loss_rows = torch.zeros((graph_iters, batch), dtype=torch.float32, device=self.dev)
        self._workspace(batch)
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.graph(g, stream=s):
            for q in range(graph_iters):
                self.grad(xb[q], tb[q], loss_rows=loss_rows[q])
                self.adam(self.grad_buf, lr, lr_schedule=self._lr_sched,
                          weight_decay=weight_decay)
        torch.cuda.current_stream().wait_stream(s)
        history = []
        perm = rng.permutation(n)
        pos = 0
        for _ in range(iters // graph_iters):
            idx = np.empty((graph_iters, batch), np.int64)
            for q in range(graph_iters):
                if pos + batch > n:
                    perm = rng.permutation(n)
                    pos = 0
                idx[q] = perm[pos:pos + batch]
                pos += batch
            it = torch.from_numpy(idx.reshape(-1)).to(self.dev)
            xb.copy_(x.index_select(0, it).view(graph_iters, batch, N_IN))
            tb.copy_(tgt.index_select(0, it).view(graph_iters, batch, TGT_COLS))
            g.replay()
            history.append(float(loss_rows.mean()))
        torch.cuda.synchronize(self.dev)
        del g
        return np.array(history)

    def loss(self, x, tgt):
        x = self._dev32(x, N_IN)
        lr = torch.empty(x.shape[0], dtype=torch.float32, device=self.dev)
        tmp = torch.empty_like(self.params)
        self.grad(x, tgt, loss_rows=lr, out=tmp)
        return float(lr.mean())

    # ------------------------------------------------------------ predictions
    def log_gamma(self, T_over_T0, E, D, lam, volume, dim):
        """log Gamma (per unit volume and time) at the given physical parameters."""
        y = self.forward(features(T_over_T0, E, D, lam, volume, dim)).cpu().numpy()
        return y[:, 0].astype(np.float64) - math.log(self.exposure_unit)

    def curve(self, T_over_T0, E, D, lam, volume, dim):
        """Converted fraction at the 16 fixed times, [rows][16]."""
        y = self.forward(features(T_over_T0, E, D, lam, volume, dim)).cpu().numpy()
        return 1.0 / (1.0 + np.exp(-y[:, 1:].astype(np.float64)))

    def state_dict(self):
        return {"params": self.params.cpu().numpy(), "exposure_unit": self.exposure_unit,
                "horizon": self.horizon}

    # ------------------------------------------------------------ helpers
    def _dev32(self, a, cols):
        if isinstance(a, torch.Tensor):
            t = a.to(self.dev, torch.float32)
        else:
            t = torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(self.dev)
        if t.dim() != 2 or t.shape[1] != cols:
            raise ValueError(f"expected [rows][{cols}], got {tuple(t.shape)}")
        return t.contiguous()
