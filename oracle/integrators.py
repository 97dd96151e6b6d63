"""CPU oracle of the alternative integrators: BAOAB and overdamped Euler-Maruyama
for the real field (R:1973-2108, R:2115-2193) and the complex field
(C:2222-2414, C:2422-2528).

TEST INFRASTRUCTURE ONLY: the GPU tests use it as the checker; the product path
never imports it.

Two sweep orders:
  * ``sweep="serial"`` restates the reference kernels run on one thread: the
    field is updated in place in the order i, 16 x 16 (j, k) tiles, j, k, so a
    site sees the already-advanced values of the neighbours visited before it.
    Pure Python loops, for the small golden cases (tests/golden/integrators.npz).
  * ``sweep="jacobi"`` (numpy) is the simultaneous update the CUDA kernels
    implement: every sub-step reads the previous sub-step's field only.
Both use the same per-site arithmetic, in the reference's order of operations.

Noise: the reference draws numpy Mersenne-Twister normals (not reproducible
across thread counts); here z (and z2 for the complex field, the sine branch of
the same pair) is the counter-based hash of (site, step) at the pass-2
multiplier, as in the RK2 stepper.
"""
from __future__ import annotations

import math

import numpy as np

from . import oracle as O

TILE_J = 16
TILE_K = 16


def _lerp(tab, tmin, dinv, npts, x):
    """R:1923-1930 lookup (vectorised): trunc toward zero, clamp, unclamped fraction."""
    x = np.asarray(x, np.float64)
    fidx = (x - tmin) * dinv
    idx = np.clip(np.trunc(np.nan_to_num(fidx, nan=0.0)), 0, npts - 2).astype(np.int64)
    frac = fidx - idx
    return tab[idx] + frac * (tab[idx + 1] - tab[idx])


def _lerp1(tab, tmin, dinv, npts, x):
    fidx = (x - tmin) * dinv
    idx = int(fidx)
    idx = 0 if idx < 0 else (npts - 2 if idx > npts - 2 else idx)
    frac = fidx - idx
    return tab[idx] + frac * (tab[idx + 1] - tab[idx])


def _lap(f, inv_dx2):
    """Periodic 7-point Laplacian summed in the reference order ip, im, jp, jm, kp, km."""
    s = np.roll(f, -1, 0) + np.roll(f, 1, 0)
    s = s + np.roll(f, -1, 1)
    s = s + np.roll(f, 1, 1)
    s = s + np.roll(f, -1, 2)
    s = s + np.roll(f, 1, 2)
    return (s - 6.0 * f) * inv_dx2


def _sites(shape):
    nx, ny, nz = shape
    for i in range(nx):
        for jj in range(0, ny, TILE_J):
            for kk in range(0, nz, TILE_K):
                for j in range(jj, min(jj + TILE_J, ny)):
                    for k in range(kk, min(kk + TILE_K, nz)):
                        yield i, j, k


def _lap1(f, i, j, k, inv_dx2):
    nx, ny, nz = f.shape
    ip, im = (i + 1) % nx, (i - 1) % nx
    jp, jm = (j + 1) % ny, (j - 1) % ny
    kp, km = (k + 1) % nz, (k - 1) % nz
    return (f[ip, j, k] + f[im, j, k] + f[i, jp, k] + f[i, jm, k] + f[i, j, kp] + f[i, j, km]
            - 6.0 * f[i, j, k]) * inv_dx2


def _noise(shape, step, seed, component=0):
    return O.noise_field(shape, step, O.K_PASS2, seed, 1.0, component)


# ------------------------------------------------------------------ real
def overdamped_step_table(phi, dt, dx, eta_eff, mu, inv_a2, tab, tmin, dinv, npts, noise_scale,
                          step, *, seed=0, sweep="jacobi"):
    """R:2115 overdamped_euler_step_table: phi += dt/eta F(phi) + ns z (returns phi)."""
    inv_dx2, inv_mu2, dto = 1.0 / (dx * dx), 1.0 / (mu * mu), dt / eta_eff
    z = _noise(phi.shape, step, seed) if noise_scale != 0.0 else np.zeros(phi.shape)
    if sweep == "serial":
        phi = phi.copy()
        for i, j, k in _sites(phi.shape):
            ph = phi[i, j, k]
            force = inv_a2 * _lap1(phi, i, j, k, inv_dx2) - _lerp1(tab, tmin, dinv, npts, ph) * inv_mu2
            phi[i, j, k] = ph + dto * force + noise_scale * z[i, j, k]
        return phi
    force = inv_a2 * _lap(phi, inv_dx2) - _lerp(tab, tmin, dinv, npts, phi) * inv_mu2
    return phi + dto * force + noise_scale * z


def baoab_step_table(phi, pi, dt, dx, gamma, mu, inv_a2, tab, tmin, dinv, npts, noise_scale,
                     step, *, seed=0, sweep="jacobi"):
    """R:1974 baoab_step_table: B A O A B with c1 = exp(-gamma dt),
    c2 = sqrt(1 - c1^2) ns.  Returns (phi, pi)."""
    inv_dx2, inv_mu2, h = 1.0 / (dx * dx), 1.0 / (mu * mu), 0.5 * dt
    c1 = math.exp(-gamma * dt)
    c2 = math.sqrt(1.0 - c1 * c1) * noise_scale
    z = _noise(phi.shape, step, seed) if noise_scale != 0.0 else np.zeros(phi.shape)
    phi, pi = phi.copy(), pi.copy()
    if sweep == "serial":
        for i, j, k in _sites(phi.shape):
            ph = phi[i, j, k]
            force = inv_a2 * _lap1(phi, i, j, k, inv_dx2) - _lerp1(tab, tmin, dinv, npts, ph) * inv_mu2
            pv = pi[i, j, k] + h * force
            phi[i, j, k] = ph + h * pv
            pi[i, j, k] = pv
        pi = c1 * pi + c2 * z
        for i, j, k in _sites(phi.shape):
            pv = pi[i, j, k]
            ph = phi[i, j, k] + h * pv
            phi[i, j, k] = ph
            force = inv_a2 * _lap1(phi, i, j, k, inv_dx2) - _lerp1(tab, tmin, dinv, npts, ph) * inv_mu2
            pi[i, j, k] = pv + h * force
        return phi, pi
    force = inv_a2 * _lap(phi, inv_dx2) - _lerp(tab, tmin, dinv, npts, phi) * inv_mu2
    pv = pi + h * force
    phi = phi + h * pv
    pi = c1 * pv + c2 * z
    phi = phi + h * pi
    force = inv_a2 * _lap(phi, inv_dx2) - _lerp(tab, tmin, dinv, npts, phi) * inv_mu2
    return phi, pi + h * force


# ---------------------------------------------------------------- complex
def _cforce1(p1, p2, tab, tmin, dinv, npts, zn):
    rho = math.sqrt(p1 * p1 + p2 * p2)
    rs = max(rho, 1e-30)
    dvr = _lerp1(tab, tmin, dinv, npts, rho)
    d1, d2 = dvr * p1 / rs, dvr * p2 / rs
    n, dv, act = zn
    if act > 0.5 and n > 0.5 and rho > 1e-20:
        s = math.sin(n * math.atan2(p2, p1))
        ir2 = (1.0 / rs) * (1.0 / rs)
        d1 += -n * dv * s * p2 * ir2
        d2 += n * dv * s * p1 * ir2
    return d1, d2


def _cforce(p1, p2, tab, tmin, dinv, npts, zn):
    rho = np.sqrt(p1 * p1 + p2 * p2)
    rs = np.maximum(rho, 1e-30)
    dvr = _lerp(tab, tmin, dinv, npts, rho)
    d1, d2 = dvr * p1 / rs, dvr * p2 / rs
    n, dv, act = zn
    if act > 0.5 and n > 0.5:
        s = np.sin(n * np.arctan2(p2, p1))
        ir2 = (1.0 / rs) * (1.0 / rs)
        on = rho > 1e-20
        d1 = d1 + np.where(on, -n * dv * s * p2 * ir2, 0.0)
        d2 = d2 + np.where(on, n * dv * s * p1 * ir2, 0.0)
    return d1, d2


def complex_overdamped_step_table(phi1, phi2, dt, dx, eta_eff, mu, inv_a2, tab, tmin, dinv,
                                  npts, noise_scale, step, *, seed=0, zn=(0.0, 0.0, 0.0),
                                  sweep="jacobi"):
    """C:2422 overdamped_euler_step_table (complex): both components, one noise pair."""
    inv_dx2, inv_mu2, dto = 1.0 / (dx * dx), 1.0 / (mu * mu), dt / eta_eff
    shp = phi1.shape
    z1 = _noise(shp, step, seed, 0) if noise_scale != 0.0 else np.zeros(shp)
    z2 = _noise(shp, step, seed, 1) if noise_scale != 0.0 else np.zeros(shp)
    if sweep == "serial":
        a, b = phi1.copy(), phi2.copy()
        for i, j, k in _sites(shp):
            p1, p2 = a[i, j, k], b[i, j, k]
            l1, l2 = _lap1(a, i, j, k, inv_dx2), _lap1(b, i, j, k, inv_dx2)
            d1, d2 = _cforce1(p1, p2, tab, tmin, dinv, npts, zn)
            a[i, j, k] = p1 + dto * (inv_a2 * l1 - d1 * inv_mu2) + noise_scale * z1[i, j, k]
            b[i, j, k] = p2 + dto * (inv_a2 * l2 - d2 * inv_mu2) + noise_scale * z2[i, j, k]
        return a, b
    d1, d2 = _cforce(phi1, phi2, tab, tmin, dinv, npts, zn)
    f1 = inv_a2 * _lap(phi1, inv_dx2) - d1 * inv_mu2
    f2 = inv_a2 * _lap(phi2, inv_dx2) - d2 * inv_mu2
    return phi1 + dto * f1 + noise_scale * z1, phi2 + dto * f2 + noise_scale * z2


def complex_baoab_step_table(phi1, phi2, pi1, pi2, dt, dx, gamma, mu, inv_a2, tab, tmin, dinv,
                             npts, noise_scale, step, *, seed=0, zn=(0.0, 0.0, 0.0),
                             sweep="jacobi"):
    """C:2223 baoab_step_table (complex).  Returns (phi1, phi2, pi1, pi2)."""
    inv_dx2, inv_mu2, h = 1.0 / (dx * dx), 1.0 / (mu * mu), 0.5 * dt
    c1 = math.exp(-gamma * dt)
    c2 = math.sqrt(1.0 - c1 * c1) * noise_scale
    shp = phi1.shape
    z1 = _noise(shp, step, seed, 0) if noise_scale != 0.0 else np.zeros(shp)
    z2 = _noise(shp, step, seed, 1) if noise_scale != 0.0 else np.zeros(shp)
    a, b, u, v = phi1.copy(), phi2.copy(), pi1.copy(), pi2.copy()
    if sweep == "serial":
        for i, j, k in _sites(shp):
            p1, p2 = a[i, j, k], b[i, j, k]
            l1, l2 = _lap1(a, i, j, k, inv_dx2), _lap1(b, i, j, k, inv_dx2)
            d1, d2 = _cforce1(p1, p2, tab, tmin, dinv, npts, zn)
            pv1 = u[i, j, k] + h * (inv_a2 * l1 - d1 * inv_mu2)
            pv2 = v[i, j, k] + h * (inv_a2 * l2 - d2 * inv_mu2)
            a[i, j, k], b[i, j, k] = p1 + h * pv1, p2 + h * pv2
            u[i, j, k], v[i, j, k] = pv1, pv2
        u, v = c1 * u + c2 * z1, c1 * v + c2 * z2
        for i, j, k in _sites(shp):
            pv1, pv2 = u[i, j, k], v[i, j, k]
            p1, p2 = a[i, j, k] + h * pv1, b[i, j, k] + h * pv2
            a[i, j, k], b[i, j, k] = p1, p2
            l1, l2 = _lap1(a, i, j, k, inv_dx2), _lap1(b, i, j, k, inv_dx2)
            d1, d2 = _cforce1(p1, p2, tab, tmin, dinv, npts, zn)
            u[i, j, k] = pv1 + h * (inv_a2 * l1 - d1 * inv_mu2)
            v[i, j, k] = pv2 + h * (inv_a2 * l2 - d2 * inv_mu2)
        return a, b, u, v
    d1, d2 = _cforce(a, b, tab, tmin, dinv, npts, zn)
    u = u + h * (inv_a2 * _lap(a, inv_dx2) - d1 * inv_mu2)
    v = v + h * (inv_a2 * _lap(b, inv_dx2) - d2 * inv_mu2)
    a, b = a + h * u, b + h * v
    u, v = c1 * u + c2 * z1, c1 * v + c2 * z2
    a, b = a + h * u, b + h * v
    d1, d2 = _cforce(a, b, tab, tmin, dinv, npts, zn)
    u = u + h * (inv_a2 * _lap(a, inv_dx2) - d1 * inv_mu2)
    v = v + h * (inv_a2 * _lap(b, inv_dx2) - d2 * inv_mu2)
    return a, b, u, v
