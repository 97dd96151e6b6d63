"""Thermal one-loop V' (the reference's physics-default potential) on the GPU.

R:432-496 tabulates dJ_B/du and dJ_F/du (u = m/T) on a uniform grid by
quadrature (cosmoTransitions' finiteT) and fits not-a-knot cubic splines; the
lattice counterterm (R:461-490, R:755-797) subtracts the soft modes below
k = pi/dx_phys; V' is assembled per site (R:1435 Vprime_field) or tabulated
over phi at a temperature (R:805-849 build_vprime_table).  Here the quadrature
and the V' evaluation run on the GPU (``tipt_thermal_*``) and the 256-point
spline is solved on the host.

``ThermalPotential(...).table_2d(...)`` gives a ``driver.Table2D`` for the
graph-captured stepper, so a thermal run steps with the same fused kernels as
the table runs.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from . import _lib as L
from ._common import dims_of, need_cuda, ptr, storage_of, stream_handle

__all__ = ["dj_grid", "not_a_knot_spline", "ThermalPotential", "counterterm_x_cut",
           "default_potential"]

YMAX = 100.0
N_Y = 256


def counterterm_x_cut(dx_phys, T0):
    """R:759 dimensionless cutoff k_max / T = pi / (dx_phys T0)."""
    return math.pi / (dx_phys * T0)


def dj_grid(u, *, fermion=False, x_cut=None, device="cuda"):
    """dJ_B (or dJ_F) at the points u (FP64, GPU quadrature); with x_cut the lattice
    counterterm's soft-mode part is subtracted."""
    u = np.ascontiguousarray(u, np.float64)
    ud = torch.from_numpy(u).to(device)
    out = torch.empty_like(ud)
    x, w = np.polynomial.legendre.leggauss(16)
    x = np.ascontiguousarray(x, np.float64)
    w = np.ascontiguousarray(w, np.float64)
    L.call("tipt_thermal_dj", int(bool(fermion)), ptr(ud), int(u.size),
           x.ctypes.data_as(L.C.c_void_p), w.ctypes.data_as(L.C.c_void_p),
           float(x_cut or 0.0), ptr(out), stream_handle())
    return out.cpu().numpy()


def not_a_knot_spline(x, y):
    """Cubic spline with not-a-knot ends (third derivative continuous at the second and
    second-to-last knots).  Returns c[4][n-1]: coefficients of dx^3, dx^2, dx, 1 on each
    segment (the layout of scipy's CubicSpline.c, which the reference uses)."""
    x = np.asarray(x, np.float64)
    y = np.asarray(y, np.float64)
    n = x.size
    if n < 4:
        raise ValueError("need at least 4 knots")
    h = np.diff(x)
    A = np.zeros((n, n))
    r = np.zeros(n)
    # second derivatives M: interior continuity of the first derivative
    for i in range(1, n - 1):
        A[i, i - 1] = h[i - 1]
        A[i, i] = 2.0 * (h[i - 1] + h[i])
        A[i, i + 1] = h[i]
        r[i] = 6.0 * ((y[i + 1] - y[i]) / h[i] - (y[i] - y[i - 1]) / h[i - 1])
    # not-a-knot: (M1 - M0)/h0 = (M2 - M1)/h1 and the same at the right end
    A[0, 0], A[0, 1], A[0, 2] = h[1], -(h[0] + h[1]), h[0]
    A[-1, -3], A[-1, -2], A[-1, -1] = h[-1], -(h[-2] + h[-1]), h[-2]
    M = np.linalg.solve(A, r)
    c = np.empty((4, n - 1))
    c[0] = (M[1:] - M[:-1]) / (6.0 * h)
    c[1] = 0.5 * M[:-1]
    c[2] = (y[1:] - y[:-1]) / h - h * (2.0 * M[:-1] + M[1:]) / 6.0
    c[3] = y[:-1]
    return c


class ThermalPotential:
    """V'(phi, T) of R:805-849 / R:1435 with the reference's parameter names; defaults are
    the script's (R:642-643, R:744-748).  ``counterterm=(dx_phys, T0)`` applies the lattice
    counterterm.  Splines can also be given directly (``splines=(cb, cf)``, each c[4][n-1]
    on the grid u = linspace(0, ymax, n_y))."""

    def __init__(self, *, lam=1e-24, mphi=1000.0, bosonMassSquared=1.0e6, bosonCoupling=1.09,
                 bosonGaugeCoupling=1.05, fermionCoupling=1.09, fermionGaugeCoupling=1.05,
                 pot_coeffs=(1.0, 1.0), n_y=N_Y, ymax=YMAX, counterterm=None, splines=None,
                 device="cuda"):
        self.dev = torch.device(device)
        self.u = np.linspace(0.0, ymax, n_y, dtype=np.float64)
        if splines is None:
            xc = counterterm_x_cut(*counterterm) if counterterm else None
            self.djb = dj_grid(self.u, fermion=False, x_cut=xc, device=self.dev)
            self.djf = dj_grid(self.u, fermion=True, x_cut=xc, device=self.dev)
            cb, cf = not_a_knot_spline(self.u, self.djb), not_a_knot_spline(self.u, self.djf)
        else:
            cb, cf = (np.asarray(c, np.float64) for c in splines)
        self.cb, self.cf = cb, cf
        self._spl = torch.from_numpy(np.ascontiguousarray(np.concatenate([cb, cf]))).to(self.dev)
        self.params = L.Thermal(lam, mphi, bosonMassSquared, bosonCoupling, bosonGaugeCoupling,
                                fermionCoupling, fermionGaugeCoupling, float(pot_coeffs[0]),
                                float(pot_coeffs[1]), float(self.u[0]),
                                float(self.u[1] - self.u[0]), n_y - 1, 0, self._spl.data_ptr())

    def source(self, T, *, lam=None, mphi=None, bosonMassSquared=None, bosonCoupling=None,
               bosonGaugeCoupling=None, fermionCoupling=None, fermionGaugeCoupling=None,
               form="inline"):
        """V' source of the steppers that evaluates this potential per site at T, as the
        reference's inline V' (R:2201-2266 _vprime_inline, ``form="inline"``) or as its
        Vprime_field (R:1435-1485, ``form="field"``, the V' of rk2_step /
        rk2_step_fused); couplings default to this object's.  The returned structure
        keeps its parameters alive."""
        if form not in ("inline", "field"):
            raise ValueError("form must be 'inline' or 'field'")
        q = self.params
        pick = lambda v, d: float(d if v is None else v)  # noqa: E731
        th = L.Thermal(pick(lam, q.lam), pick(mphi, q.mphi), pick(bosonMassSquared, q.boson_mass_sq),
                       pick(bosonCoupling, q.boson_coupling),
                       pick(bosonGaugeCoupling, q.boson_gauge_coupling),
                       pick(fermionCoupling, q.fermion_coupling),
                       pick(fermionGaugeCoupling, q.fermion_gauge_coupling), q.coeff_b, q.coeff_f,
                       q.x_min, q.h, q.nseg, 1 if form == "field" else 0, self._spl.data_ptr())
        vs = L.VSource(L.VP_THERMAL, 0, None, 0.0, 0.0, 0, 0, 0.0, 0.0, float(T), 0.0, 0.0, 0.0,
                       C.addressof(th))
        vs._keep = (th, self._spl)
        return vs

    def vprime_field(self, phi, T, out=None):
        """R:1435 Vprime_field(out, phi, T, ...): V' per site (FP64; into ``out`` with
        phi's dtype when given, as the reference's out array)."""
        need_cuda(phi, names=["phi"])
        shape = dims_of(phi)
        o = torch.empty(shape, dtype=torch.float64, device=phi.device)
        L.call("tipt_thermal_vprime_field", storage_of(phi), ptr(phi), float(T), self.params,
               ptr(o), *shape, stream_handle())
        if out is not None:
            out.copy_(o)
            return out
        return o

    def table(self, T, phi_min, phi_max, n_table):
        """R:840 build_vprime_table(T, phi_min, phi_max, n): (table, tmin, dinv)."""
        t = self._table(phi_min, phi_max, n_table, [T])[0]
        return t, float(phi_min), 1.0 / ((phi_max - phi_min) / (n_table - 1))

    def _table(self, phi_lo, phi_hi, nphi, Ts):
        Td = torch.from_numpy(np.ascontiguousarray(Ts, np.float64)).to(self.dev)
        out = torch.empty((len(Ts), nphi), dtype=torch.float64, device=self.dev)
        L.call("tipt_thermal_vprime_table", float(phi_lo), float(phi_hi), int(nphi), ptr(Td),
               int(len(Ts)), self.params, ptr(out), stream_handle())
        return out

    def table_2d(self, phi_lo, phi_hi, nphi, T_lo, T_hi, nT):
        """A driver.Table2D of V'(phi, T) on uniform grids, built on the GPU."""
        from .driver import Table2D
        Ts = np.linspace(T_lo, T_hi, nT, dtype=np.float64)
        v = self._table(phi_lo, phi_hi, nphi, Ts).cpu().numpy()
        return Table2D(np.ascontiguousarray(v), float(phi_lo),
                       1.0 / ((phi_hi - phi_lo) / (nphi - 1)), float(T_lo),
                       1.0 / ((T_hi - T_lo) / (nT - 1)))


_DEFAULT = {}


def default_potential(device="cuda", pot_coeffs=(1.0, 1.0)):
    """The reference script's module-level splines (R:432-455: dJ_B, dJ_F on the
    256-point grid, no counterterm) with its _POT_COEFFS (real script (1, 1),
    complex script (2, -1), C:215), built once per device on the GPU."""
    dev = torch.device(device)
    key = (dev.type, dev.index if dev.index is not None else torch.cuda.current_device(),
           tuple(float(c) for c in pot_coeffs))
    if key not in _DEFAULT:
        _DEFAULT[key] = ThermalPotential(device=dev, pot_coeffs=pot_coeffs)
    return _DEFAULT[key]


def Vprime_scalar(phi_val, T_val, *, potential=None):
    """R:805 Vprime_scalar(phi, T): V'(phi, T) as a Python float, evaluated on the GPU
    as build_vprime_table evaluates each point; the potential defaults to the
    reference script's (default_potential)."""
    tp = potential if potential is not None else default_potential()
    x = float(phi_val)
    # the first point of a two-point grid is phi itself
    return float(tp._table(x, x + max(1.0, abs(x)), 2, [float(T_val)])[0, 0])


def build_vprime_table(T_val, phi_min, phi_max, n_table, *, potential=None):
    """R:840 build_vprime_table(T, phi_min, phi_max, n): (table as a float64 CUDA
    tensor, phi_min, 1/dphi); the potential defaults to the reference script's."""
    tp = potential if potential is not None else default_potential()
    return tp.table(T_val, phi_min, phi_max, n_table)
