"""numpy/ctypes front end of the CPU oracle (``oracle/tipt_oracle.c``).

TEST INFRASTRUCTURE ONLY: the parity tests, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` use this module as the checker.  The product
path never imports it.

Also holds the FP64 potential/table builders for the benchmark workloads (the
toy polynomial V' = 2D(T^2-T0^2)phi - 3E T phi^2 + lam phi^3) restated from the
table construction in R:805-849 (``build_vprime_table``): a uniform grid,
``table[i] = V'(lo + i*(hi-lo)/(n-1), T)``, ``dinv = 1/((hi-lo)/(n-1))``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtipt_oracle.so")

K_PASS2 = 73856093
K_PASS4 = 19349669

_lib = None


def build(force: bool = False) -> str:
    if force or not os.path.exists(LIB_PATH) or (
        os.path.getmtime(LIB_PATH) < os.path.getmtime(os.path.join(HERE, "tipt_oracle.c"))
    ):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = C.CDLL(LIB_PATH)
        _declare(_lib)
    return _lib


_d, _i64, _u64, _i = C.c_double, C.c_int64, C.c_uint64, C.c_int
_p = C.c_void_p


def _declare(L):
    L.orc_hash_pair.argtypes = [_p, _i64, _p, _p, _p]
    L.orc_noise_key.argtypes = [_i64, _u64, _u64, _u64]
    L.orc_noise_key.restype = _u64
    L.orc_noise_fill.argtypes = [_p, _i64, _i64, _i64, _u64, _u64, _u64, _d, _i]
    L.orc_table_blend_row.argtypes = [_p, _i64, _i64, _d, _d, _d, _p]
    base = [_p, _p, _p, _p, _i64, _i64, _i64, _d, _d, _d, _d, _d]
    L.orc_rk2_step_table_f64.argtypes = base + [_p, _d, _d, _i64, _p, _d, _u64, _u64]
    L.orc_rk2_step_table_f32.argtypes = base + [_p, _d, _d, _i64, _p, _d, _u64, _u64]
    L.orc_rk2_fused_table_f64.argtypes = base + [_p, _d, _d, _i64, _p, _d, _d, _i64, _p, _d, _u64, _u64]
    L.orc_rk2_fused_table_f32.argtypes = base + [_p, _d, _d, _i64, _p, _d, _d, _i64, _p, _d, _u64, _u64]
    L.orc_rk2_fused_poly_f64.argtypes = base + [_d, _d, _d, _u64, _u64]
    L.orc_rk2_step_poly_f64.argtypes = base + [_d, _d, _d, _d, _u64, _u64]
    L.orc_rk2_step_table_complex_f64.argtypes = (
        [_p] * 8 + [_i64, _i64, _i64, _d, _d, _d, _d, _d, _p, _d, _d, _i64, _d, _d, _d, _d,
                    _p, _p, _d, _u64, _u64])
    L.orc_winding.argtypes = [_p, _p, _i64, _i64, _i64, _p, _p, _p]
    L.orc_observables_f64.argtypes = [_p, _p, _i64, _i64, _i64, _d, _d, _d, _d, _d, _d, _p]
    L.orc_num_threads.restype = _i


def _ptr(a):
    return None if a is None else a.ctypes.data


def _c(a, dtype):
    assert a.dtype == dtype and a.flags.c_contiguous, (a.dtype, a.flags)
    return a


def num_threads() -> int:
    return int(lib().orc_num_threads())


# ------------------------------------------------------------------ noise
def hash_pair(seeds):
    seeds = np.ascontiguousarray(seeds, dtype=np.uint64)
    u1 = np.empty(seeds.shape, np.float64)
    u2 = np.empty(seeds.shape, np.float64)
    z = np.empty(seeds.shape, np.float64)
    lib().orc_hash_pair(_ptr(seeds), seeds.size, _ptr(u1), _ptr(u2), _ptr(z))
    return u1, u2, z


def noise_key(site, step, mul, seed=0):
    return int(lib().orc_noise_key(site, step, mul, seed))


def noise_field(shape, step, mul=K_PASS2, seed=0, scale=1.0, component=0):
    out = np.empty(shape, np.float64)
    nx, ny, nz = shape
    lib().orc_noise_fill(_ptr(out), nx, ny, nz, step, mul, seed, scale, component)
    return out


# ------------------------------------------------------------------ tables
def toy_vprime(phi, T, D=0.1, E=0.05, lam=0.1, T0=1.0):
    """V'(phi) of V = D(T^2-T0^2)phi^2 - E T phi^3 + (lam/4) phi^4."""
    phi = np.asarray(phi, np.float64)
    return 2.0 * D * (T * T - T0 * T0) * phi - 3.0 * E * T * phi * phi + lam * phi * phi * phi


def toy_vprime_rho(rho, T, D=0.1, E=0.05, lam=0.1, T0=1.0):
    """dV/d|Phi| of the complex toy potential (same polynomial in |Phi|)."""
    return toy_vprime(rho, T, D, E, lam, T0)


def build_table(fn, lo, hi, n):
    """R:840-849 build_vprime_table: (table, tmin, dinv)."""
    x = np.linspace(lo, hi, n, dtype=np.float64)
    return np.ascontiguousarray(fn(x), np.float64), float(lo), 1.0 / ((hi - lo) / (n - 1))


def build_table_2d(fn, lo, hi, n_phi, T_lo, T_hi, n_T):
    """[n_T][n_phi] FP64 table of fn(phi, T); returns (table, tmin, dinv, T_min, T_dinv)."""
    x = np.linspace(lo, hi, n_phi, dtype=np.float64)
    Ts = np.linspace(T_lo, T_hi, n_T, dtype=np.float64)
    t2 = np.stack([fn(x, T) for T in Ts]).astype(np.float64)
    return (np.ascontiguousarray(t2), float(lo), 1.0 / ((hi - lo) / (n_phi - 1)), float(T_lo),
            1.0 / ((T_hi - T_lo) / (n_T - 1)))


def table_blend_row(t2d, T_min, T_dinv, T):
    t2d = _c(t2d, np.float64)
    out = np.empty(t2d.shape[1], np.float64)
    lib().orc_table_blend_row(_ptr(t2d), t2d.shape[0], t2d.shape[1], T_min, T_dinv, T, _ptr(out))
    return out


# ------------------------------------------------------------------ steppers
def rk2_step_table(phi, pi, dt, dx, eta_eff, mu, noise, phi_tmp, pi_tmp, inv_a2, vp_table,
                   vp_tmin, vp_dinv, vp_npts, *, noise_scale=0.0, noise_step=0, noise_seed=0):
    """R:1875 rk2_step_table, in place; noise=None selects inline hash noise."""
    nx, ny, nz = phi.shape
    f = lib().orc_rk2_step_table_f64 if phi.dtype == np.float64 else lib().orc_rk2_step_table_f32
    dt_ = phi.dtype
    for a in (phi, pi, phi_tmp, pi_tmp):
        _c(a, dt_)
    if noise is not None:
        _c(noise, dt_)
    f(_ptr(phi), _ptr(pi), _ptr(phi_tmp), _ptr(pi_tmp), nx, ny, nz, dt, dx, eta_eff, mu, inv_a2,
      _ptr(_c(vp_table, np.float64)), vp_tmin, vp_dinv, vp_npts, _ptr(noise), noise_scale,
      noise_step, noise_seed)


def rk2_fused_table(phi, pi, dt, dx, eta_eff, mu, noise, phi_tmp, pi_tmp, inv_a2, vp_table_T,
                    vp_tmin_T, vp_dinv_T, vp_npts_T, vp_table_Tm, vp_tmin_Tm, vp_dinv_Tm,
                    vp_npts_Tm, *, noise_scale=0.0, noise_step=0, noise_seed=0):
    """R:1708 rk2_fused_table (two dt/2 halves), in place."""
    nx, ny, nz = phi.shape
    f = lib().orc_rk2_fused_table_f64 if phi.dtype == np.float64 else lib().orc_rk2_fused_table_f32
    dt_ = phi.dtype
    for a in (phi, pi, phi_tmp, pi_tmp):
        _c(a, dt_)
    if noise is not None:
        _c(noise, dt_)
    f(_ptr(phi), _ptr(pi), _ptr(phi_tmp), _ptr(pi_tmp), nx, ny, nz, dt, dx, eta_eff, mu, inv_a2,
      _ptr(_c(vp_table_T, np.float64)), vp_tmin_T, vp_dinv_T, vp_npts_T,
      _ptr(_c(vp_table_Tm, np.float64)), vp_tmin_Tm, vp_dinv_Tm, vp_npts_Tm, _ptr(noise),
      noise_scale, noise_step, noise_seed)


def rk2_step_poly(phi, pi, dt, dx, eta_eff, mu, inv_a2, c1, c2, c3, *, noise_scale=0.0,
                  noise_step=0, noise_seed=0):
    """R:1875 rk2_step_table with V'(x) = c1 x + c2 x^2 + c3 x^3 instead of the table (the
    batched replicas' toy potential), FP64, in place, inline hash noise."""
    nx, ny, nz = phi.shape
    for a in (phi, pi):
        _c(a, np.float64)
    tmp = [np.empty_like(phi), np.empty_like(pi)]
    lib().orc_rk2_step_poly_f64(_ptr(phi), _ptr(pi), _ptr(tmp[0]), _ptr(tmp[1]), nx, ny, nz, dt,
                                dx, eta_eff, mu, inv_a2, c1, c2, c3, noise_scale, noise_step,
                                noise_seed)


def rk2_fused_single_pass_poly(phi, pi, dt, dx, eta_eff, mu, lam, mphi, noise_scale, noise_step,
                               phi_tmp, pi_tmp, inv_a2, noise_seed=0):
    """R:2339 rk2_fused_single_pass with zero thermal couplings (V' = lam phi^3 - mphi^2 phi)."""
    nx, ny, nz = phi.shape
    for a in (phi, pi, phi_tmp, pi_tmp):
        _c(a, np.float64)
    lib().orc_rk2_fused_poly_f64(_ptr(phi), _ptr(pi), _ptr(phi_tmp), _ptr(pi_tmp), nx, ny, nz, dt,
                                 dx, eta_eff, mu, inv_a2, lam, mphi, noise_scale, noise_step,
                                 noise_seed)


def rk2_step_table_complex(phi1, phi2, pi1, pi2, dt, dx, eta_eff, mu, noise1, noise2, phi1_tmp,
                           phi2_tmp, pi1_tmp, pi2_tmp, inv_a2, vp_table, vp_tmin, vp_dinv, vp_npts,
                           *, zn=(0.0, 0.0, 0.0), eps4=0.0, noise_scale=0.0, noise_step=0,
                           noise_seed=0):
    """C:2067 complex rk2_step_table (FP64), in place."""
    nx, ny, nz = phi1.shape
    for a in (phi1, phi2, pi1, pi2, phi1_tmp, phi2_tmp, pi1_tmp, pi2_tmp):
        _c(a, np.float64)
    lib().orc_rk2_step_table_complex_f64(
        _ptr(phi1), _ptr(phi2), _ptr(pi1), _ptr(pi2), _ptr(phi1_tmp), _ptr(phi2_tmp),
        _ptr(pi1_tmp), _ptr(pi2_tmp), nx, ny, nz, dt, dx, eta_eff, mu, inv_a2,
        _ptr(_c(vp_table, np.float64)), vp_tmin, vp_dinv, vp_npts, float(zn[0]), float(zn[1]),
        float(zn[2]), eps4, _ptr(noise1), _ptr(noise2), noise_scale, noise_step, noise_seed)


def winding(phi1, phi2):
    """C:2683 compute_winding_number on FP64 arrays -> (w_site f32, w3 int8[3,...], counts[4])."""
    phi1 = _c(np.ascontiguousarray(phi1, np.float64), np.float64)
    phi2 = _c(np.ascontiguousarray(phi2, np.float64), np.float64)
    nx, ny, nz = phi1.shape
    w = np.empty(phi1.shape, np.float32)
    w3 = np.empty((3,) + phi1.shape, np.int8)
    cnt = np.zeros(4, np.int64)
    lib().orc_winding(_ptr(phi1), _ptr(phi2), nx, ny, nz, _ptr(w), _ptr(w3), _ptr(cnt))
    return w, w3, cnt


OBS_NAMES = ("E_kin", "E_grad", "E_pot", "phi_mean", "phi2_mean", "pi2_mean", "frac_above",
             "phi_min", "phi_max", "n_nonfinite")


def observables(phi, pi, dx=1.0, inv_a2=1.0, lam=0.0, mphi=0.0, mu=1.0, thr=1.0):
    phi = _c(np.ascontiguousarray(phi, np.float64), np.float64)
    pi = None if pi is None else _c(np.ascontiguousarray(pi, np.float64), np.float64)
    nx, ny, nz = phi.shape
    out = np.zeros(10, np.float64)
    lib().orc_observables_f64(_ptr(phi), _ptr(pi), nx, ny, nz, dx, inv_a2, lam, mphi, mu, thr,
                              _ptr(out))
    return dict(zip(OBS_NAMES, out.tolist()))
