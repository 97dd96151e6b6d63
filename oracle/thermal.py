"""CPU oracle of the thermal one-loop V' of the real field's inline steppers and of
the un-fused stepper rk2_step / rk2_step_fused (R:1489-1656).

TEST INFRASTRUCTURE ONLY: the tests use it as the checker; the product path never
imports it.

``vprime_inline`` restates the reference's ``_vprime_inline`` (R:2201-2266), the
V' that ``rk2_fused_single_pass`` (R:2339-2647) evaluates per site: the polynomial
part lam phi^3 - mphi^2 phi plus T^4/(2 pi^2) times the dJ_B / dJ_F spline terms
(arguments x_b, x_f clamped to [x_min, x_min + h nseg - 1e-12], segment
trunc((x - x_min) / h) clamped to [0, nseg - 1], Horner in dx), vectorised over phi,
FP64 in the reference's order of operations.  ``vprime_field`` is the
Vprime_field form (R:1435-1485): x above x_min + h nseg lowered to that bound
minus 1e-12 (values between the two bounds are left), segment
trunc((x - x_min) / h) (cubic_eval_uniform, R:1415-1426).  ``laplacian``,
``rk2_step`` and ``rk2_step_fused`` restate laplacian_periodic (R:1364-1385) and
the two un-fused steppers as whole-array numpy expressions.
"""
from __future__ import annotations

import math

import numpy as np


def vprime_inline(phi, T, cb, cf, x_min, h, *, lam, mphi, bosonMassSquared, bosonCoupling,
                  bosonGaugeCoupling, fermionCoupling, fermionGaugeCoupling,
                  pot_coeffs=(1.0, 1.0)):
    """R:2201-2266 for an array of field values at temperature T.  cb, cf: spline
    coefficients [4][nseg] (dx^3, dx^2, dx, 1) of dJ_B and dJ_F on x_min + i h."""
    ph = np.asarray(phi, np.float64)
    nseg = cb.shape[1]
    T2 = T * T                                          # R:2381
    pref = T2 * T2 / (2.0 * math.pi * math.pi)          # R:2382
    gb2, gg2 = bosonCoupling * bosonCoupling, bosonGaugeCoupling * bosonGaugeCoupling
    gf2, gfg2 = fermionCoupling * fermionCoupling, fermionGaugeCoupling * fermionGaugeCoupling
    coef_b = 0.25 * gb2 + (2.0 / 3.0) * gg2             # R:2376
    inv_hy, xhi = 1.0 / h, x_min + h * nseg - 1e-12    # R:452-453
    dV = lam * ph * ph * ph - (mphi * mphi) * ph
    xb_sq = bosonMassSquared + 0.5 * gb2 * ph * ph + coef_b * T2
    xb = np.where(xb_sq > 0.0, np.sqrt(np.maximum(xb_sq, 0.0)) / T, 0.0)
    xf_sq = 0.5 * gf2 * ph * ph + (1.0 / 6.0) * gfg2 * T2
    xf = np.where(xf_sq > 0.0, np.sqrt(np.maximum(xf_sq, 0.0)) / T, 0.0)

    def dj(c, x):
        xc = np.minimum(np.maximum(x, x_min), xhi)
        si = np.clip(((xc - x_min) * inv_hy).astype(np.int64), 0, nseg - 1)
        d = xc - (x_min + si * h)
        return ((c[0][si] * d + c[1][si]) * d + c[2][si]) * d + c[3][si]

    dxb = 0.5 * gb2 * ph / (T2 * np.maximum(xb, 1e-20))
    dxf = 0.5 * gf2 * ph / (T2 * np.maximum(xf, 1e-20))
    return dV + pref * (pot_coeffs[0] * dj(cb, xb) * dxb + pot_coeffs[1] * dj(cf, xf) * dxf)


def cubic_eval_uniform(x, x_min, h, nseg, c0, c1, c2, c3):
    """R:1415-1426 for an array of points."""
    x = np.asarray(x, np.float64)
    t = (x - x_min) / h
    i = np.where(t > 0.0, np.minimum(t, float(nseg - 1)), 0.0).astype(np.int64)
    d = x - (x_min + i * h)
    return ((c0[i] * d + c1[i]) * d + c2[i]) * d + c3[i]


def vprime_field(phi, T, cb, cf, x_min, h, *, lam, mphi, bosonMassSquared, bosonCoupling,
                 bosonGaugeCoupling, fermionCoupling, fermionGaugeCoupling,
                 pot_coeffs=(1.0, 1.0)):
    """R:1435-1485 Vprime_field for an array of field values at T."""
    ph = np.asarray(phi, np.float64)
    nseg = cb.shape[1]
    T2 = T * T
    pref = (T2 * T2) / (2.0 * math.pi * math.pi)
    gb2, gg2 = bosonCoupling * bosonCoupling, bosonGaugeCoupling * bosonGaugeCoupling
    gf2, gfg2 = fermionCoupling * fermionCoupling, fermionGaugeCoupling * fermionGaugeCoupling
    coef_b_T = 0.25 * gb2 + (2.0 / 3.0) * gg2
    dV = lam * ph * ph * ph - mphi * mphi * ph
    xb_sq = bosonMassSquared + 0.5 * gb2 * ph * ph + coef_b_T * T2
    xb = np.where(xb_sq > 0.0, np.sqrt(np.maximum(xb_sq, 0.0)) / T, 0.0)
    xf_sq = 0.5 * gf2 * ph * ph + (1.0 / 6.0) * gfg2 * T2
    xf = np.where(xf_sq > 0.0, np.sqrt(np.maximum(xf_sq, 0.0)) / T, 0.0)
    top = x_min + h * nseg

    def clamp(x):
        return np.where(x < x_min, x_min, np.where(x > top, top - 1e-12, x))

    djb = cubic_eval_uniform(clamp(xb), x_min, h, nseg, *cb)
    djf = cubic_eval_uniform(clamp(xf), x_min, h, nseg, *cf)
    dxb = 0.5 * gb2 * ph / (T2 * np.maximum(xb, 1e-20))
    dxf = 0.5 * gf2 * ph / (T2 * np.maximum(xf, 1e-20))
    return dV + pref * (pot_coeffs[0] * djb * dxb + pot_coeffs[1] * djf * dxf)


def laplacian(a, dx):
    """R:1364-1385 laplacian_periodic (FP64)."""
    return (np.roll(a, -1, 0) + np.roll(a, 1, 0) + np.roll(a, -1, 1) + np.roll(a, 1, 1) +
            np.roll(a, -1, 2) + np.roll(a, 1, 2) - 6.0 * a) * (1.0 / (dx * dx))


def _half(phi, pi, h1, h2, dx, eta, T, mu, inv_a2, noise, vp):
    k1 = inv_a2 * laplacian(phi, dx) - eta * pi - vp(phi, T) / (mu * mu)
    pm, vm = phi + h1 * pi, pi + h1 * k1
    k2 = inv_a2 * laplacian(pm, dx) - eta * vm - vp(pm, T) / (mu * mu)
    return phi + h2 * vm, pi + h2 * k2 + noise


def rk2_step(phi, pi, dt, dx, eta, T, mu, couplings, noise, inv_a2, cb, cf, x_min, h,
             pot_coeffs=(1.0, 1.0)):
    """R:1489-1550: returns (phi, pi) after one midpoint step (FP64)."""
    vp = lambda x, TT: vprime_field(x, TT, cb, cf, x_min, h, pot_coeffs=pot_coeffs,  # noqa: E731
                                    **couplings)
    return _half(phi, pi, 0.5 * dt, dt, dx, eta, T, mu, inv_a2, noise, vp)


def rk2_step_fused(phi, pi, dt, dx, eta, T, T_mid, mu, couplings, noise, inv_a2, cb, cf, x_min,
                   h, pot_coeffs=(1.0, 1.0)):
    """R:1553-1656: two dt/2 halves at T then T_mid, 0.5 * noise each (FP64)."""
    vp = lambda x, TT: vprime_field(x, TT, cb, cf, x_min, h, pot_coeffs=pot_coeffs,  # noqa: E731
                                    **couplings)
    phi, pi = _half(phi, pi, 0.5 * dt, 0.5 * dt, dx, eta, T, mu, inv_a2, 0.5 * noise, vp)
    return _half(phi, pi, 0.5 * dt, 0.5 * dt, dx, eta, T_mid, mu, inv_a2, 0.5 * noise, vp)
