"""CPU oracle of the thermal one-loop V' of the real field's inline steppers.

TEST INFRASTRUCTURE ONLY: the tests use it as the checker; the product path never
imports it.

``vprime_inline`` restates the reference's ``_vprime_inline`` (R:2201-2266), the
V' that ``rk2_fused_single_pass`` (R:2339-2647) evaluates per site: the polynomial
part lam phi^3 - mphi^2 phi plus T^4/(2 pi^2) times the dJ_B / dJ_F spline terms
(arguments x_b, x_f clamped to [x_min, x_min + h nseg - 1e-12], segment
trunc((x - x_min) / h) clamped to [0, nseg - 1], Horner in dx), vectorised over phi,
FP64 in the reference's order of operations.
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
