"""Golden fixture of the reference's un-fused stepper and its array helpers
(tests/golden/unfused.npz), generated with the REFERENCE's own kernels:

    TIPT_REFERENCE_ROOT=<reference checkout> python tests/golden/make_golden_unfused.py

AST-extracted real-field kernels (ref_extract.load_real) with the dJ splines of
tests/golden/thermal.npz as module globals, run unmodified:
* ``laplacian_periodic`` (R:1364-1385) on float64 and float32 fields;
* ``cubic_eval_uniform`` (R:1415-1426) at points inside, below and above the grid;
* five steps of ``rk2_step`` (R:1489-1550) and of ``rk2_step_fused`` (R:1553-1656)
  with the script's default couplings, float64 and float32 arrays, noise arrays
  filled with the reference's hash and Box-Muller (make_golden.noise).
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import make_golden  # noqa: E402
import ref_extract  # noqa: E402
from make_golden_complex_thermal import _spline_globals  # noqa: E402

SHAPES = {"3d": (12, 10, 8), "odd": (17, 9, 5), "2d": (24, 20, 1)}


def main():
    spl = _spline_globals()
    R = ref_extract.load_real(pot_coeffs=(1.0, 1.0), splines=spl)
    c = dict(lam=1e-24, mphi=1000.0, bosonMassSquared=1.0e6, bosonCoupling=1.09,
             bosonGaugeCoupling=1.05, fermionCoupling=1.09, fermionGaugeCoupling=1.05)
    cv = [c[k] for k in ("lam", "mphi", "bosonMassSquared", "bosonCoupling",
                         "bosonGaugeCoupling", "fermionCoupling", "fermionGaugeCoupling")]
    out = {}
    # laplacian_periodic
    for tag, shape in SHAPES.items():
        rng = np.random.default_rng(900 + len(tag))
        a = rng.normal(0.3, 1.1, shape)
        for dtype, dn in ((np.float64, "f64"), (np.float32, "f32")):
            x = a.astype(dtype)
            o = np.empty_like(x)
            R["laplacian_periodic"](o, x, 0.7)
            out[f"lap_{tag}_{dn}_in"], out[f"lap_{tag}_{dn}_out"] = x, o
    # cubic_eval_uniform at points over [x_min - 2, x_max + 3]
    nseg = spl["nseg"]
    lo, hi = spl["x_min"], spl["x_min"] + spl["h_y"] * nseg
    xs = np.concatenate([np.linspace(lo - 2.0, hi + 3.0, 397), [lo, hi, spl["xhi_clamp"]]])
    cub = np.array([R["cubic_eval_uniform"](x, spl["x_min"], spl["h_y"], nseg, spl["c0_b"],
                                            spl["c1_b"], spl["c2_b"], spl["c3_b"]) for x in xs])
    out["cubic_x"], out["cubic_out"] = xs, cub
    # rk2_step / rk2_step_fused
    dt, dx, eta, mu, inv_a2, T, Tm, ns = 0.05, 1.0, 0.5, 1000.0, 1.0, 3000.0, 2999.7, 40.0
    for tag, shape in SHAPES.items():
        rng = np.random.default_rng(950 + len(tag))
        phi0 = rng.normal(0.0, 4000.0, shape)
        pi0 = rng.normal(0.0, 300.0, shape)
        for dtype, dn in ((np.float64, "f64"), (np.float32, "f32")):
            for name in ("rk2_step", "rk2_step_fused"):
                phi, pi = phi0.astype(dtype), pi0.astype(dtype)
                key = f"{name}_{tag}_{dn}"
                out[f"{key}_phi0"], out[f"{key}_pi0"] = phi.copy(), pi.copy()
                for n in range(5):
                    nf = make_golden.noise(shape, n, make_golden.K_PASS2, ns, dtype=dtype)
                    scratch = [np.empty_like(phi) for _ in range(4)]
                    if name == "rk2_step":
                        R[name](phi, pi, dt, dx, eta, T, mu, *cv, nf, *scratch, inv_a2)
                    else:
                        R[name](phi, pi, dt, dx, eta, T, Tm, mu, *cv, nf, *scratch, inv_a2)
                out[f"{key}_phi5"], out[f"{key}_pi5"] = phi, pi
    make_golden.save("unfused.npz", dt=dt, dx=dx, eta=eta, mu=mu, inv_a2=inv_a2, T=T, T_mid=Tm,
                     ns=ns, lap_dx=0.7, **{k: np.float64(v) for k, v in c.items()}, **out)


if __name__ == "__main__":
    main()
