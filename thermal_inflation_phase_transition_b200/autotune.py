"""Tile-shape autotuner of the marching stage kernels, with a persisted JSON cache.

A marching kernel's tile is (rows per tile, planes per work item, ring
stages), plus the row segment for the complex kernel; ``field="real"`` tunes
the real-field kernel, ``field="complex"`` the complex-field one (compensated
FP32).  The built-in heuristic scores candidates by occupancy and halo share;
``tune`` instead times every admissible candidate on the device (CUDA events,
inputs larger than L2 where the lattice is) and keeps the fastest.  Results are
cached per (GPU name, field, storage, lattice shape, V' table size) in a JSON file
(``$TIPT_AUTOTUNE_CACHE``, else ``~/.cache/tipt_b200/autotune.json``);
``apply`` installs a cached shape, or the heuristic when there is none.

No reference counterpart: the reference's only knob is the CPU tile size
(R:1969-1970).
"""
from __future__ import annotations

import json
import os
import time

import torch

from . import _lib as L
from . import complex_field as CF
from . import real_field as RF
from ._common import table_source

__all__ = ["cache_path", "cache_key", "candidates", "tune", "apply", "load_cache"]

STAGES = (3, 4, 5)
PLANES = (8, 16, 32, 64, 128, 256, 512)


def cache_path() -> str:
    p = os.environ.get("TIPT_AUTOTUNE_CACHE")
    if p:
        return p
    return os.path.join(os.path.expanduser("~"), ".cache", "tipt_b200", "autotune.json")


def cache_key(shape, storage, table_points, device=None, field="real") -> str:
    dev = torch.device(device or "cuda")
    name = torch.cuda.get_device_name(dev).replace(" ", "_")
    cc = "%d.%d" % torch.cuda.get_device_capability(dev)
    nx, ny, nz = shape
    tag = "" if field == "real" else f"{field}|"
    return f"{name}|sm{cc}|{tag}{storage}|{nx}x{ny}x{nz}|table{int(table_points)}"


def load_cache() -> dict:
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _save_cache(c: dict) -> None:
    p = cache_path()
    os.makedirs(os.path.dirname(p), exist_ok=True)
    tmp = p + ".tmp"
    with open(tmp, "w") as f:
        json.dump(c, f, indent=1, sort_keys=True)
    os.replace(tmp, p)


def candidates(shape, field="real"):
    """Tile shapes the kernel may accept for this lattice: (rows, planes, stages) for the
    real kernel, (rows, planes, stages, row segment) for the complex one (the kernel still
    rejects those that do not fit shared memory)."""
    nx, ny, nz = shape
    if field == "real":
        n0, n1, n2 = (1, nx, ny) if nz == 1 else (nx, ny, nz)
        segs, planes = [None], PLANES
    else:
        n0, n1, n2 = nx, ny, nz
        segs = [n2] + [k for k in range(n2 - 1, 127, -1) if n2 % k == 0 and k % 32 == 0]
        planes = (32, 64, 128, 256)
    out = []
    for ks in segs:
        tpr = n2 // 4 if ks is None else ks // 2
        for tj in range(1, 65):
            if n1 % tj or (tj * tpr) % 32 or tj * tpr > 512:
                continue
            for ci in planes:
                if ci > n0 and ci != planes[0]:
                    continue
                for st in STAGES:
                    out.append((tj, ci, st) if ks is None else (tj, ci, st, ks))
    return out


def _state(shape, storage, device, field="real"):
    nx, ny, nz = shape
    g = torch.Generator(device=device)
    g.manual_seed(1)
    if field == "complex":
        f = [torch.zeros((2, nx, ny, nz), dtype=torch.float32, device=device) for _ in range(4)]
        for a in f[:2]:
            a[0] = 0.5 + 0.01 * torch.randn((nx, ny, nz), generator=g, device=device)
        return [f, [torch.empty_like(a) for a in f]]
    if storage == "f32c":
        phi = torch.zeros((2, nx, ny, nz), dtype=torch.float32, device=device)
        phi[0] = 0.01 * torch.randn((nx, ny, nz), generator=g, device=device)
        pi = torch.zeros_like(phi)
    else:
        phi = 0.01 * torch.randn((nx, ny, nz), dtype=torch.float64, generator=g, device=device)
        pi = torch.zeros_like(phi)
    return [phi, pi, torch.empty_like(phi), torch.empty_like(pi)]


def _time(state, table, steps, warmup, field="real"):
    """Mean ms per stage launch (ping-pong between the two state sets)."""
    vs = table_source(table, 0.0, (table.numel() - 1) / 3.0, table.numel())
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    for n in range(warmup + steps):
        if n == warmup:
            torch.cuda.synchronize()
            e0.record()
        if field == "complex":
            a, b = state[n % 2], state[(n + 1) % 2]
            CF.rk2_step_table_into(a, b, 0.05, 1.0, 1.0, 1.0, 1.0, vs, eps4=1e-3, noise_scale=0.3,
                                   noise_step=n, seed=2)
            continue
        bufs = ((state[0], state[1]), (state[2], state[3]))
        (phi, pi), (po, qo) = bufs[n % 2], bufs[(n + 1) % 2]
        RF.rk2_step_table_into(phi, pi, po, qo, 0.05, 1.0, 1.0, 1.0, 1.0, vs, noise_scale=0.3,
                               noise_step=n, seed=1)
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def tune(shape, storage="f32c", *, table_points=4096, steps=10, warmup=3, persist=True,
         device="cuda", log=None, field="real"):
    """Time every admissible tile shape; returns {"best": [rows, planes, stages], "ms": t,
    "default_ms": t0, "tried": n} and stores it in the cache."""
    if storage not in ("f32c", "f64") or (field == "complex" and storage != "f32c"):
        raise ValueError("the marching kernels run F32C and F64 (real) / F32C (complex)")
    dev = torch.device(device)
    state = _state(shape, storage, dev, field)
    table = torch.linspace(-0.1, 0.1, table_points, dtype=torch.float64, device=dev)
    L.set_kernel_policy(2)
    try:
        L.set_march_tiles(0, 0, 0)
        default_ms = _time(state, table, steps, warmup, field)
        best, best_ms, tried = None, float("inf"), 0
        t_start = time.perf_counter()
        for c in candidates(shape, field):
            L.set_march_tiles(*c[:3])
            L.set_march_kseg(c[3] if len(c) > 3 else 0)
            try:
                ms = _time(state, table, steps, warmup, field)
            except L.TiptError:
                continue
            tried += 1
            if log:
                log(f"  tile {c}: {ms:.4f} ms")
            if ms < best_ms:
                best, best_ms = c, ms
    finally:
        L.set_march_tiles(0, 0, 0)
        L.set_march_kseg(0)
        L.set_kernel_policy(0)
    if best is None:
        raise RuntimeError(f"no marching tile shape accepted for {shape} {storage}")
    res = {"best": list(best), "ms": best_ms, "default_ms": default_ms, "tried": tried,
           "seconds": time.perf_counter() - t_start}
    if persist:
        c = load_cache()
        c[cache_key(shape, storage, table_points, dev, field)] = res
        _save_cache(c)
    return res


def apply(shape, storage="f32c", *, table_points=4096, tune_if_missing=False, device="cuda",
          field="real"):
    """Install the cached tile shape for this workload (tuning first if asked and absent).
    Returns the installed (rows, planes, stages), or None for the built-in heuristic.  The
    tile shape is a library-wide setting: apply it before the runs of that workload."""
    key = cache_key(shape, storage, table_points, device, field)
    entry = load_cache().get(key)
    if entry is None and tune_if_missing:
        entry = tune(shape, storage, table_points=table_points, device=device, field=field)
    if entry is None or entry["ms"] >= entry.get("default_ms", float("inf")):
        L.set_march_tiles(0, 0, 0)
        L.set_march_kseg(0)
        return None
    b = entry["best"]
    L.set_march_tiles(*b[:3])
    L.set_march_kseg(b[3] if len(b) > 3 else 0)
    return tuple(b)
