"""Golden fixture of rk2_fused_single_pass with the thermal inline V'
(tests/golden/thermal_inline.npz), generated with the REFERENCE's own kernels:

    TIPT_REFERENCE_ROOT=<reference checkout> python tests/golden/make_golden_thermal_inline.py

The spline coefficients are those of tests/golden/thermal.npz (the reference's
dJ_B / dJ_F quadratures on its 256-point grid, not-a-knot splines; see
make_golden_thermal.py); they become the module globals (c0_b .. c3_f, x_min,
h_y, inv_hy, xhi_clamp, nseg) of the AST-extracted real-field kernels, which
are run unmodified:
* ``_vprime_inline`` (R:2201-2266) at sample fields and temperatures;
* five steps of ``rk2_fused_single_pass`` (R:2339-2647) with the script's
  default couplings (R:642-643, R:744-748) on two lattices;
* five steps of ``rk2_step_inline`` (R:2654-2822) on the same lattices, its noise
  array filled with the reference's hash and Box-Muller (make_golden.noise).
"""
from __future__ import annotations

import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import make_golden  # noqa: E402
import ref_extract  # noqa: E402


def main():
    th = np.load(os.path.join(HERE, "thermal.npz"))
    u, cb, cf = th["u"], th["cb"], th["cf"]
    h = float(u[1] - u[0])
    nseg = cb.shape[1]
    spl = {"c0_b": cb[0].copy(), "c1_b": cb[1].copy(), "c2_b": cb[2].copy(), "c3_b": cb[3].copy(),
           "c0_f": cf[0].copy(), "c1_f": cf[1].copy(), "c2_f": cf[2].copy(), "c3_f": cf[3].copy(),
           "x_min": float(u[0]), "h_y": h, "inv_hy": 1.0 / h,
           "xhi_clamp": float(u[0]) + h * nseg - 1e-12, "nseg": nseg}
    pot = (1.0, 1.0)
    R = ref_extract.load_real(pot_coeffs=pot, splines=spl)
    c = dict(lam=1e-24, mphi=1000.0, bosonMassSquared=1.0e6, bosonCoupling=1.09,
             bosonGaugeCoupling=1.05, fermionCoupling=1.09, fermionGaugeCoupling=1.05)
    gb2, gg2 = c["bosonCoupling"] ** 2, c["bosonGaugeCoupling"] ** 2
    gf2, gfg2 = c["fermionCoupling"] ** 2, c["fermionGaugeCoupling"] ** 2
    coef_b = 0.25 * gb2 + (2.0 / 3.0) * gg2
    # _vprime_inline at sample fields (both signs, the clamps, x = 0) and temperatures
    phs = np.concatenate([np.linspace(-9e4, 9e4, 61), [0.0, 1e-3, -1e-3, 3e5, -3e5]])
    Ts = np.array([500.0, 3000.0, 12000.0])
    vin = np.empty((Ts.size, phs.size))
    for a, T in enumerate(Ts):
        T2 = T * T
        pref = T2 * T2 / (2.0 * math.pi * math.pi)
        for b, ph in enumerate(phs):
            vin[a, b] = R["_vprime_inline"](
                ph, T, T2, pref, c["lam"], c["mphi"] ** 2, c["bosonMassSquared"], gb2, gf2, gg2,
                gfg2, coef_b, spl["x_min"], spl["h_y"], spl["inv_hy"], spl["xhi_clamp"], nseg,
                spl["c0_b"], spl["c1_b"], spl["c2_b"], spl["c3_b"], spl["c0_f"], spl["c1_f"],
                spl["c2_f"], spl["c3_f"])
    # five steps of rk2_fused_single_pass: program units with mu = mphi, T near the
    # transition, fields of thousands of GeV
    dt, dx, eta, mu, inv_a2, T, Tm, ns = 0.05, 1.0, 0.5, 1000.0, 1.0, 3000.0, 2999.7, 40.0
    out = {}
    for tag, shape in {"3d": (12, 10, 8), "odd": (17, 9, 5)}.items():
        rng = np.random.default_rng(500 + len(tag))
        phi = rng.normal(0.0, 4000.0, shape)
        pi = rng.normal(0.0, 300.0, shape)
        out[f"{tag}_phi0"], out[f"{tag}_pi0"] = phi.copy(), pi.copy()
        for n in range(5):
            R["rk2_fused_single_pass"](phi, pi, dt, dx, eta, T, Tm, mu, c["lam"], c["mphi"],
                                       c["bosonMassSquared"], c["bosonCoupling"],
                                       c["bosonGaugeCoupling"], c["fermionCoupling"],
                                       c["fermionGaugeCoupling"], ns, np.uint64(n),
                                       np.empty_like(phi), np.empty_like(pi), inv_a2)
        out[f"{tag}_phi5"], out[f"{tag}_pi5"] = phi, pi
        # rk2_step_inline from the same initial state, noise array at the pass-2 multiplier
        phi, pi = out[f"{tag}_phi0"].copy(), out[f"{tag}_pi0"].copy()
        for n in range(5):
            nf = make_golden.noise(shape, n, make_golden.K_PASS2, ns)
            out[f"{tag}_noise{n}"] = nf
            R["rk2_step_inline"](phi, pi, dt, dx, eta, T, mu, c["lam"], c["mphi"],
                                 c["bosonMassSquared"], c["bosonCoupling"],
                                 c["bosonGaugeCoupling"], c["fermionCoupling"],
                                 c["fermionGaugeCoupling"], nf, np.empty_like(phi),
                                 np.empty_like(pi), inv_a2)
        out[f"{tag}_inline_phi5"], out[f"{tag}_inline_pi5"] = phi, pi
    np.savez_compressed(os.path.join(HERE, "thermal_inline.npz"), u=u, cb=cb, cf=cf,
                        pot_coeffs=np.array(pot), phs=phs, Ts=Ts, vprime_inline=vin, dt=dt,
                        dx=dx, eta=eta, mu=mu, inv_a2=inv_a2, T=T, T_mid=Tm, ns=ns,
                        **{k: np.float64(v) for k, v in c.items()}, **out)
    print("wrote thermal_inline.npz", vin[1, :3], out["3d_phi5"].ravel()[:3])


if __name__ == "__main__":
    main()
