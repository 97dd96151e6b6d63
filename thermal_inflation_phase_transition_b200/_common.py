"""Tensor checks and C-ABI argument packing shared by the field modules."""
from __future__ import annotations

import ctypes as C

import torch

from . import _lib as L


def storage_of(t: torch.Tensor) -> int:
    """float64 (nx,ny,nz) -> F64; float32 (nx,ny,nz) -> F32; float32 (2,nx,ny,nz) -> F32C
    (compensated pair: plane 0 = hi, plane 1 = lo, value hi + lo)."""
    if t.dtype == torch.float64 and t.dim() == 3:
        return L.TIPT_F64
    if t.dtype == torch.float32 and t.dim() == 3:
        return L.TIPT_F32
    if t.dtype == torch.float32 and t.dim() == 4 and t.shape[0] == 2:
        return L.TIPT_F32C
    raise TypeError(f"unsupported field tensor: dtype={t.dtype}, shape={tuple(t.shape)} "
                    "(want float64/float32 (nx,ny,nz) or float32 (2,nx,ny,nz) hi/lo planes)")


def dims_of(t: torch.Tensor) -> tuple[int, int, int]:
    return tuple(int(x) for x in (t.shape[1:] if t.dim() == 4 else t.shape))


def need_cuda(*ts, names=None):
    for n, t in enumerate(ts):
        if t is None:
            continue
        nm = names[n] if names else f"argument {n}"
        if not isinstance(t, torch.Tensor) or not t.is_cuda:
            raise TypeError(f"{nm} must be a CUDA tensor")
        if not t.is_contiguous():
            raise ValueError(f"{nm} must be contiguous (C-order)")


def same_layout(ref: torch.Tensor, *ts, names=None):
    for n, t in enumerate(ts):
        if t is None:
            continue
        if t.dtype != ref.dtype or t.shape != ref.shape:
            nm = names[n] if names else f"argument {n}"
            raise ValueError(f"{nm} must match the field's dtype/shape {ref.dtype}"
                             f"{tuple(ref.shape)}, got {t.dtype}{tuple(t.shape)}")


def ptr(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def stream_handle(stream=None):
    s = torch.cuda.current_stream() if stream is None else stream
    return C.c_void_p(s.cuda_stream)


def step_params(dt, dx, eta_eff, mu, inv_a2, noise_scale=0.0, noise_step=0, seed=0):
    return L.StepParams(float(dt), float(dx), float(eta_eff), float(mu), float(inv_a2),
                        float(noise_scale), int(noise_step) & (2 ** 64 - 1),
                        int(seed) & (2 ** 64 - 1))


def table_source(vp_table, vp_tmin, vp_dinv, vp_npts, T=None, T_min=None, T_dinv=None):
    """V' source from the reference's table arguments (R:1885-1888).

    A 1-D float64 CUDA tensor is the reference's table; a 2-D [nT][npts] tensor
    is the (phi, T) table, blended at T (T_min, T_dinv give its T grid).  The
    source holds a reference to the table tensor, so a source kept for later
    launches never points at freed memory."""
    need_cuda(vp_table, names=["vp_table"])
    if vp_table.dtype != torch.float64:
        raise TypeError("vp_table must be float64 (the table is built in FP64)")
    npts = int(vp_npts)
    if vp_table.dim() == 1:
        if vp_table.numel() < npts or npts < 2:
            raise ValueError("vp_npts out of range for vp_table")
        vs = L.VSource(L.VP_TABLE, npts, vp_table.data_ptr(), float(vp_tmin), float(vp_dinv),
                       0, 0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0)
        vs._keep = vp_table
        return vs
    if vp_table.dim() == 2:
        if T is None or T_min is None or T_dinv is None:
            raise ValueError("a 2-D table needs T, T_min and T_dinv")
        if vp_table.shape[1] != npts:
            raise ValueError("vp_npts must equal the table's phi extent")
        vs = L.VSource(L.VP_TABLE2D, npts, vp_table.data_ptr(), float(vp_tmin), float(vp_dinv),
                       int(vp_table.shape[0]), 0, float(T_min), float(T_dinv), float(T), 0.0,
                       0.0, 0.0)
        vs._keep = vp_table
        return vs
    raise ValueError("vp_table must be 1-D or 2-D")


def poly_source(c1, c2, c3):
    return L.VSource(L.VP_POLY, 0, None, 0.0, 0.0, 0, 0, 0.0, 0.0, 0.0, float(c1), float(c2),
                     float(c3))


def swap_storage(a: torch.Tensor, b: torch.Tensor) -> None:
    """Exchange the storages of a and b in place (tensor objects keep their identity).

    This gives the fused ping-pong kernels the reference's in-place call
    semantics without a copy; views taken of a or b before the call keep
    pointing at the old buffers."""
    sa, oa, za, ta = a.untyped_storage(), a.storage_offset(), a.size(), a.stride()
    sb, ob, zb, tb = b.untyped_storage(), b.storage_offset(), b.size(), b.stride()
    with torch.no_grad():
        a.set_(sb, ob, zb, tb)
        b.set_(sa, oa, za, ta)
