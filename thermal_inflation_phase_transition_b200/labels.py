"""Connected-component labelling of bubbles and string voxels on the GPU.

Replaces ``scipy.ndimage.label`` and the per-cluster measurements of the
reference's post-processing: ``_identify_bubbles`` (postprocess/
revisualize_snapshots.py:171-214) and ``_identify_strings`` (:360-392).  The
label array equals scipy's (face connectivity, raster-order numbering); the
per-label statistics come from one pass of device sums.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from . import _lib as L
from ._common import dims_of, need_cuda, ptr, storage_of, stream_handle

__all__ = ["label", "label_stats", "identify_bubbles", "identify_strings"]


def label(field, threshold, *, periodic=False):
    """Components of |field| > threshold: (int32 labels with the lattice shape, n)."""
    need_cuda(field, names=["field"])
    st = storage_of(field)
    shape = dims_of(field)
    dev = field.device
    ws = torch.empty(int(L.lib().tipt_label_workspace_size(*shape)) // 4 + 1, dtype=torch.int32,
                     device=dev)
    lab = torch.empty(shape, dtype=torch.int32, device=dev)
    n = torch.zeros(1, dtype=torch.int32, device=dev)
    L.call("tipt_label_components", st, ptr(field), float(threshold), *shape, int(bool(periodic)),
           ptr(lab), ptr(n), ptr(ws), ws.numel() * 4, stream_handle())
    return lab, int(n.item())


def label_stats(field, labels, n):
    """Per-label (count, sum_xyz[n+1][3], sum_sq, sum_val, max_abs) as host arrays."""
    shape = tuple(labels.shape)
    dev = labels.device
    st = storage_of(field) if field is not None else L.TIPT_F64
    count = torch.empty(n + 1, dtype=torch.int64, device=dev)
    sxyz = torch.empty((n + 1, 3), dtype=torch.int64, device=dev)
    ssq = torch.empty(n + 1, dtype=torch.int64, device=dev)
    sval = torch.empty(n + 1, dtype=torch.float64, device=dev)
    mx = torch.empty(n + 1, dtype=torch.float64, device=dev)
    L.call("tipt_label_stats", st, ptr(field), ptr(labels), *shape, int(n), ptr(count), ptr(sxyz),
           ptr(ssq), ptr(sval), ptr(mx), stream_handle())
    return (count.cpu().numpy(), sxyz.cpu().numpy(), ssq.cpu().numpy(), sval.cpu().numpy(),
            mx.cpu().numpy())


def identify_bubbles(phi, escape_phi, *, dx_phys=None, periodic=False):
    """_identify_bubbles(|phi| > escape_phi, phi): dicts with centroid, volume, r_eff,
    r_rms, sign, peak (and r_phys), sorted by volume, largest first."""
    lab, n = label(phi, escape_phi, periodic=periodic)
    if n == 0:
        return []
    count, sxyz, ssq, sval, mx = label_stats(phi, lab, n)
    out = []
    for c in range(1, n + 1):
        vol = int(count[c])
        centroid = sxyz[c] / vol
        r_eff = (3.0 * vol / (4.0 * np.pi)) ** (1.0 / 3.0)
        r_rms = math.sqrt(max(ssq[c] / vol - float(np.dot(centroid, centroid)), 0.0))
        e = dict(centroid=centroid, volume=vol, r_eff=r_eff, r_rms=r_rms,
                 sign=1 if sval[c] / vol >= 0 else -1, peak=float(mx[c]))
        if dx_phys is not None:
            e["r_phys"] = r_eff * dx_phys
        out.append(e)
    out.sort(key=lambda b: b["volume"], reverse=True)
    return out


def identify_strings(winding, threshold=0.5, *, periodic=False):
    """_identify_strings: (labels as a host array, dicts with loop_id, n_voxels,
    centroid, winding_sign, max_winding), sorted by n_voxels, longest first."""
    lab, n = label(winding, threshold, periodic=periodic)
    if n == 0:
        return lab.cpu().numpy(), []
    count, sxyz, _, sval, mx = label_stats(winding, lab, n)
    out = []
    for c in range(1, n + 1):
        v = int(count[c])
        out.append(dict(loop_id=c, n_voxels=v, centroid=sxyz[c] / v,
                        winding_sign=1 if sval[c] / v >= 0 else -1, max_winding=float(mx[c])))
    out.sort(key=lambda s: s["n_voxels"], reverse=True)
    return lab.cpu().numpy(), out
