"""CPU oracle of the complex field's fused and inline RK2 steppers.

TEST INFRASTRUCTURE ONLY: the tests use it as the checker; the product path never
imports it.

numpy restatements, FP64, vectorised over the lattice in the reference's order of
operations:
* ``rk2_fused_table`` -- C:1789-2064: two dt/2 midpoint halves with the V'(rho)
  tables at T, then T_mid (R:1923-1930 lookup rule on rho), Z_N term of
  C:1850-1856, 0.5 * noise array in each half;
* ``rk2_fused_single_pass`` -- C:2765-3132: the same two halves with the inline
  thermal V'(rho) (_vprime_complex_inline, C:2606-2680, radial part
  oracle.thermal.vprime_inline at rho_safe = max(rho, 1e-30)) and the inline hash
  pair per site, key (site * 73856093) ^ step in the first half and
  (site * 19349669) ^ step in the second, 0.5 * noise_scale * (r cos, r sin);
* ``rk2_step_inline`` -- C:3140-: one midpoint step (dt/2 predictor, dt
  corrector) with the inline thermal V'(rho) and noise arrays;
* ``field_force`` / ``rk2_step`` / ``rk2_step_fused`` -- C:1452-1737: the
  un-fused forms with Vprime_field (the radial V' of oracle.thermal.vprime_field at
  rho_safe, projected, plus the Z_N term).
"""
from __future__ import annotations

import numpy as np

from . import oracle as O
from .thermal import vprime_field, vprime_inline


def _lap(f, inv_dx2):
    # (ip + im + jp + jm + kp + km - 6 f) * inv_dx2, periodic (C:1840-1848)
    return (np.roll(f, -1, 0) + np.roll(f, 1, 0) + np.roll(f, -1, 1) + np.roll(f, 1, 1) +
            np.roll(f, -1, 2) + np.roll(f, 1, 2) - 6.0 * f) * inv_dx2


def _lerp(tab, tmin, dinv, npts, x):
    # R:1923-1930: idx = trunc((x - tmin) dinv) clamped to [0, npts - 2], weight unclamped
    fidx = (x - tmin) * dinv
    last = npts - 2
    idx = np.where(fidx > 0.0, np.minimum(fidx, float(last)), 0.0).astype(np.int64)
    frac = fidx - idx
    return tab[idx] + frac * (tab[idx + 1] - tab[idx])


def _zn(p1, p2, rho, rho_safe, zn, d1, d2):
    # C:1850-1856 / C:2670-2678
    n, dv, active = zn
    if active > 0.5 and n > 0.5:
        on = rho > 1e-20
        sn = np.sin(n * np.arctan2(p2, p1))
        ir = 1.0 / rho_safe
        ir2 = ir * ir
        d1 = np.where(on, d1 + (-n * dv * sn * p2 * ir2), d1)
        d2 = np.where(on, d2 + (n * dv * sn * p1 * ir2), d2)
    return d1, d2


def table_force(tab, tmin, dinv, npts, zn=(0.0, 0.0, 0.0)):
    """C:1833-1856: dV_a = V'(rho) phi_a / rho_safe (+ Z_N)."""
    def f(p1, p2):
        rho = np.sqrt(p1 * p1 + p2 * p2)
        rho_safe = np.maximum(rho, 1e-30)
        dvdr = _lerp(tab, tmin, dinv, npts, rho)
        return _zn(p1, p2, rho, rho_safe, zn, dvdr * p1 / rho_safe, dvdr * p2 / rho_safe)
    return f


def thermal_force(T, cb, cf, x_min, h, couplings, pot_coeffs=(2.0, -1.0), zn=(0.0, 0.0, 0.0)):
    """C:2606-2680: V'(rho_safe) phi_a (1 / rho_safe) (+ Z_N)."""
    def f(p1, p2):
        rho = np.sqrt(p1 * p1 + p2 * p2)
        rho_safe = np.maximum(rho, 1e-30)
        dvdr = vprime_inline(rho_safe, T, cb, cf, x_min, h, pot_coeffs=pot_coeffs, **couplings)
        inv_rho = 1.0 / rho_safe
        return _zn(p1, p2, rho, rho_safe, zn, dvdr * p1 * inv_rho, dvdr * p2 * inv_rho)
    return f


def midpoint(s, h1, h2, dx, eta, mu, inv_a2, force, n1, n2):
    """One midpoint stage on s = [phi1, phi2, pi1, pi2] (in place): predictor
    phi + h1 pi, pi + h1 k at the state, corrector phi += h2 pi~,
    pi += h2 k~ + n at the predicted state."""
    inv_dx2, inv_mu2 = 1.0 / (dx * dx), 1.0 / (mu * mu)

    def kicks(p1, p2, v1, v2):
        d1, d2 = force(p1, p2)
        return (inv_a2 * _lap(p1, inv_dx2) - eta * v1 - d1 * inv_mu2,
                inv_a2 * _lap(p2, inv_dx2) - eta * v2 - d2 * inv_mu2)

    p1, p2, v1, v2 = s
    k1, k2 = kicks(p1, p2, v1, v2)
    t1, t2, u1, u2 = p1 + h1 * v1, p2 + h1 * v2, v1 + h1 * k1, v2 + h1 * k2
    k1, k2 = kicks(t1, t2, u1, u2)
    s[0] = p1 + h2 * u1
    s[1] = p2 + h2 * u2
    s[2] = v1 + (h2 * k1 + n1)
    s[3] = v2 + (h2 * k2 + n2)


def rk2_fused_table(s, dt, dx, eta, mu, noise1, noise2, inv_a2, tab_T, tmin_T, dinv_T, npts_T,
                    tab_Tm, tmin_Tm, dinv_Tm, npts_Tm, zn=(0.0, 0.0, 0.0)):
    """C:1789-2064 on s = [phi1, phi2, pi1, pi2], in place."""
    h = 0.5 * dt
    for tab, tmin, dinv, npts in ((tab_T, tmin_T, dinv_T, npts_T),
                                  (tab_Tm, tmin_Tm, dinv_Tm, npts_Tm)):
        midpoint(s, h, h, dx, eta, mu, inv_a2, table_force(tab, tmin, dinv, npts, zn),
                 0.5 * noise1, 0.5 * noise2)


def rk2_fused_single_pass(s, dt, dx, eta, T, T_mid, mu, couplings, noise_scale, step, inv_a2,
                          cb, cf, x_min, h_y, pot_coeffs=(2.0, -1.0)):
    """C:2765-3132 on s = [phi1, phi2, pi1, pi2], in place (seed 0)."""
    h = 0.5 * dt
    shape = s[0].shape
    for TT, mul in ((T, O.K_PASS2), (T_mid, O.K_PASS4)):
        z1 = O.noise_field(shape, step, mul, 0, noise_scale, 0)
        z2 = O.noise_field(shape, step, mul, 0, noise_scale, 1)
        midpoint(s, h, h, dx, eta, mu, inv_a2,
                 thermal_force(TT, cb, cf, x_min, h_y, couplings, pot_coeffs), 0.5 * z1, 0.5 * z2)


def rk2_step_inline(s, dt, dx, eta, T, mu, couplings, noise1, noise2, inv_a2, cb, cf, x_min, h_y,
                    pot_coeffs=(2.0, -1.0)):
    """C:3140- on s = [phi1, phi2, pi1, pi2], in place."""
    midpoint(s, 0.5 * dt, dt, dx, eta, mu, inv_a2,
             thermal_force(T, cb, cf, x_min, h_y, couplings, pot_coeffs), noise1, noise2)


def field_force(T, cb, cf, x_min, h, couplings, pot_coeffs=(2.0, -1.0), zn=(0.0, 0.0, 0.0)):
    """C:1452-1530 Vprime_field: V'(rho_safe) phi_a * (1 / rho_safe) (+ Z_N)."""
    def f(p1, p2):
        rho = np.sqrt(p1 * p1 + p2 * p2)
        rho_safe = np.maximum(rho, 1e-30)
        inv_rho = 1.0 / rho_safe
        dv = vprime_field(rho_safe, T, cb, cf, x_min, h, pot_coeffs=pot_coeffs, **couplings)
        return _zn(p1, p2, rho, rho_safe, zn, dv * p1 * inv_rho, dv * p2 * inv_rho)
    return f


def rk2_step(s, dt, dx, eta, T, mu, couplings, noise1, noise2, inv_a2, cb, cf, x_min, h_y,
             pot_coeffs=(2.0, -1.0), zn=(0.0, 0.0, 0.0)):
    """C:1533-1607 on s = [phi1, phi2, pi1, pi2], in place."""
    midpoint(s, 0.5 * dt, dt, dx, eta, mu, inv_a2,
             field_force(T, cb, cf, x_min, h_y, couplings, pot_coeffs, zn), noise1, noise2)


def rk2_step_fused(s, dt, dx, eta, T, T_mid, mu, couplings, noise1, noise2, inv_a2, cb, cf,
                   x_min, h_y, pot_coeffs=(2.0, -1.0), zn=(0.0, 0.0, 0.0)):
    """C:1610-1737 on s = [phi1, phi2, pi1, pi2], in place."""
    for TT in (T, T_mid):
        midpoint(s, 0.5 * dt, 0.5 * dt, dx, eta, mu, inv_a2,
                 field_force(TT, cb, cf, x_min, h_y, couplings, pot_coeffs, zn),
                 0.5 * noise1, 0.5 * noise2)
