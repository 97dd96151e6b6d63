"""Observable reductions on device (FP64, deterministic order).

``observables`` returns a CUDA float64 tensor of 10 values without a host
sync; index with ``OBS_INDEX``.  Covers compute_energy_densities (R:2270-2319)
plus the per-step reductions of the host loop.
"""
from __future__ import annotations

import torch

from . import _lib as L
from ._common import dims_of, need_cuda, ptr, storage_of, stream_handle

OBS_NAMES = ("E_kin", "E_grad", "E_pot", "phi_mean", "phi2_mean", "pi2_mean", "frac_above",
             "phi_min", "phi_max", "n_nonfinite")
OBS_INDEX = {n: q for q, n in enumerate(OBS_NAMES)}


def workspace_bytes(shape) -> int:
    nx, ny, nz = shape
    return int(L.lib().tipt_observables_workspace_size(nx, ny, nz))


def observables(phi, pi=None, *, dx=1.0, inv_a2=1.0, lam=0.0, mphi=0.0, mu=1.0, thr=1.0,
                out=None, workspace=None, stream=None):
    """Reduce (phi, pi) to E_kin, E_grad, E_pot, <phi>, <phi^2>, <pi^2>,
    fraction(phi > thr), min, max, non-finite count (device float64[10])."""
    need_cuda(phi, pi, names=["phi", "pi"])
    st = storage_of(phi)
    shape = dims_of(phi)
    if out is None:
        out = torch.empty(10, dtype=torch.float64, device=phi.device)
    wb = workspace_bytes(shape)
    if workspace is None:
        workspace = torch.empty(max(wb, 8) // 8 + 1, dtype=torch.float64, device=phi.device)
    L.call("tipt_observables", st, ptr(phi), ptr(pi), *shape, float(dx), float(inv_a2),
           float(lam), float(mphi), float(mu), float(thr), ptr(out), ptr(workspace),
           workspace.numel() * workspace.element_size(), stream_handle(stream))
    return out
