"""Field snapshots, checkpoints and resume in the reference's ``.npz`` layout.

The reference saves ``state_step_{n:010d}.npz`` every snapshot interval
(R:3997-4018; complex C:4624-4654) and ``simulation_metadata.npz`` at the end
(R:4126-4167); ``--resume`` takes the newest snapshot that has ``pi`` and no
NaN (R:2963-3010).  This module writes and reads the same files from device
state, so the reference's post-processing reads GPU runs unchanged:

* real field: ``phi, step, time, temperature, phi_min, phi_max`` (+ ``E_kin,
  E_grad, E_pot`` when given, ``scale_factor, hubble`` when given) and ``pi`` on
  every ``checkpoint_every``-th save (the reference's CHECKPOINT_EVERY = 10,
  R:395);
* complex field: ``phi1, phi2, rho, theta (float32), winding (float32, per-site
  plaquette sum), step, time, temperature, rho_min, rho_max, zn_active`` and
  ``pi1, pi2`` on checkpoints.

Compensated-FP32 fields are written as float64 (hi + lo, exact) and their lo
planes are added under ``<name>_lo`` so that a resume rebuilds the exact
planes; the reference ignores the extra keys.  The device-to-host copies
happen on the caller's stream at the call; the file write runs on a
background thread (``wait()`` joins it).

The container is the reference's npz.  The reference deflates it
(``np.savez_compressed``); lattice fields are noise-dominated floats that
deflate by about 1 % at some 30 MB/s, so the writer stores the members
uncompressed by default (``np.savez``: the same keys and arrays for
``np.load``, 40x faster to write) and deflates on request (``compress=True``).
"""
from __future__ import annotations

import glob
import os
import threading

import numpy as np
import torch

__all__ = ["SnapshotWriter", "latest_checkpoint", "load_fields", "write_metadata",
           "snapshot_name"]


def snapshot_name(state_path, step):
    return os.path.join(state_path, f"state_step_{int(step):010d}.npz")


def _is_f32c(t):
    """The compensated-FP32 layout: float32 (2, nx, ny, nz), hi plane then lo plane."""
    return t.dtype == torch.float32 and t.dim() == 4 and t.shape[0] == 2


def _host(t):
    """Device or host tensor -> (numpy value array, numpy lo plane or None)."""
    if _is_f32c(t):
        hi = t[0].detach().to("cpu", torch.float64)
        lo = t[1].detach().to("cpu")
        return (hi + lo.double()).numpy(), lo.numpy()
    return t.detach().cpu().numpy(), None


class SnapshotWriter:
    """Writes snapshots into ``state_path`` with the reference's cadence of full
    checkpoints (``pi`` on saves 0, checkpoint_every, 2*checkpoint_every, ...)."""

    def __init__(self, state_path, *, checkpoint_every=10, background=True, compress=False):
        os.makedirs(state_path, exist_ok=True)
        self.state_path = state_path
        self.checkpoint_every = int(checkpoint_every)
        self.background = background
        self.compress = bool(compress)
        self.total_saves = 0
        self._threads = []

    def _write(self, path, d):
        def run():
            tmp = path[:-4] + ".tmp.npz"
            (np.savez_compressed if self.compress else np.savez)(tmp, **d)
            os.replace(tmp, path)
        if self.background:
            th = threading.Thread(target=run, daemon=False)
            th.start()
            self._threads.append(th)
        else:
            run()

    def wait(self):
        for th in self._threads:
            th.join()
        self._threads = []

    def _next_is_checkpoint(self):
        c = self.total_saves % self.checkpoint_every == 0
        self.total_saves += 1
        return c

    def save_real(self, step, time, temperature, phi, pi=None, *, energies=None,
                  scale_factor=None, hubble=None):
        """R:3997-4018.  ``energies`` = (E_kin, E_grad, E_pot) or None.  Returns the path."""
        ckpt = self._next_is_checkpoint()
        ph, ph_lo = _host(phi)
        d = dict(phi=ph, step=int(step), time=float(time), temperature=float(temperature),
                 phi_min=ph.min(), phi_max=ph.max())
        if ph_lo is not None:
            d["phi_lo"] = ph_lo
        if energies is not None:
            d["E_kin"], d["E_grad"], d["E_pot"] = (float(e) for e in energies)
        if ckpt and pi is not None:
            pv, pv_lo = _host(pi)
            d["pi"] = pv
            if pv_lo is not None:
                d["pi_lo"] = pv_lo
        if scale_factor is not None:
            d["scale_factor"] = float(scale_factor)
            d["hubble"] = float(hubble if hubble is not None else 0.0)
        path = snapshot_name(self.state_path, step)
        self._write(path, d)
        return path

    def save_complex(self, step, time, temperature, phi1, phi2, pi1=None, pi2=None, *,
                     zn_active=0.0, winding=None, scale_factor=None, hubble=None):
        """C:4624-4654.  ``winding`` (per-site plaquette sum, float32) is computed with
        the library's winding kernel when the fields are on the GPU and it is not given."""
        ckpt = self._next_is_checkpoint()
        if winding is None:
            if not phi1.is_cuda:
                raise ValueError("host fields need the winding array passed in")
            from .complex_field import compute_winding_number_full
            w = compute_winding_number_full(phi1, phi2, w_site=True, w3=False).w_site
            winding = w.cpu().numpy()
        a, a_lo = _host(phi1)
        b, b_lo = _host(phi2)
        a64, b64 = a.astype(np.float64), b.astype(np.float64)
        rho = np.sqrt(a64 ** 2 + b64 ** 2)
        theta = np.arctan2(b64, a64)
        d = dict(phi1=a, phi2=b, rho=rho.astype(np.float32), theta=theta.astype(np.float32),
                 winding=np.asarray(winding, np.float32).copy(), step=int(step), time=float(time),
                 temperature=float(temperature), rho_min=float(rho.min()),
                 rho_max=float(rho.max()), zn_active=float(zn_active))
        if a_lo is not None:
            d["phi1_lo"], d["phi2_lo"] = a_lo, b_lo
        if ckpt and pi1 is not None:
            u, u_lo = _host(pi1)
            v, v_lo = _host(pi2)
            d["pi1"], d["pi2"] = u, v
            if u_lo is not None:
                d["pi1_lo"], d["pi2_lo"] = u_lo, v_lo
        if scale_factor is not None:
            d["scale_factor"] = float(scale_factor)
            d["hubble"] = float(hubble if hubble is not None else 0.0)
        path = snapshot_name(self.state_path, step)
        self._write(path, d)
        return path


def latest_checkpoint(state_path, *, need_pi=True, keys=("phi",), pi_keys=("pi",)):
    """R:2963-2990: the newest ``state_step_*.npz`` (not ``*_NaN_debug*``) whose fields
    (and, with need_pi, momenta) are present and free of NaN.  Returns (path, dict) or
    (None, None).  Complex runs pass keys=("phi1", "phi2"), pi_keys=("pi1", "pi2")."""
    files = sorted(glob.glob(os.path.join(state_path, "state_step_*.npz")))
    files = [f for f in files if "_NaN_debug" not in f and ".tmp." not in f]
    for f in reversed(files):
        with np.load(f) as z:
            d = {k: z[k] for k in z.files}
        if need_pi and not all(k in d for k in pi_keys):
            continue
        names = list(keys) + (list(pi_keys) if need_pi else [])
        if any(np.isnan(d[k]).any() for k in names):
            continue
        return f, d
    return None, None


def load_fields(d, names, storage, device="cuda"):
    """Checkpoint arrays -> device tensors in the given storage ("f64", "f32", "f32c").
    Compensated fields saved with ``<name>_lo`` planes are rebuilt exactly."""
    out = []
    for n in names:
        x = np.asarray(d[n])
        if storage == "f32c":
            if n + "_lo" in d:
                lo = np.asarray(d[n + "_lo"], np.float32)
                hi = (x.astype(np.float64) - lo.astype(np.float64)).astype(np.float32)
            else:
                hi = x.astype(np.float32)
                lo = (x.astype(np.float64) - hi.astype(np.float64)).astype(np.float32)
            out.append(torch.from_numpy(np.stack([hi, lo])).to(device))
        else:
            dt = torch.float64 if storage == "f64" else torch.float32
            out.append(torch.from_numpy(np.ascontiguousarray(x)).to(device, dt))
    return out


def write_metadata(save_path, **fields):
    """R:4126-4167 ``simulation_metadata.npz`` (the caller passes the reference's keys:
    Nx, Ny, Nz, dx_phys, dt_phys, mphi, lam, eta_phys, nb, nf, T0, cooling_rate, Nt,
    steps, total_time, mu, dx, dt, eta, vev, integrator, ...)."""
    os.makedirs(save_path, exist_ok=True)
    path = os.path.join(save_path, "simulation_metadata.npz")
    np.savez(path, **fields)
    return path
