"""Golden fixture of the complex script's un-fused stepper
(tests/golden/complex_unfused.npz), generated with the REFERENCE's own kernels:

    TIPT_REFERENCE_ROOT=<reference checkout> python tests/golden/make_golden_complex_unfused.py

AST-extracted complex-field kernels (ref_extract.load_complex) with the dJ
splines of tests/golden/thermal.npz and the script's _POT_COEFFS = (2, -1), run
unmodified: ``Vprime_field`` (C:1452-1530) on a field, and five steps of
``rk2_step`` (C:1533-1607) and ``rk2_step_fused`` (C:1610-1737) with the
script's default couplings, U(1) and Z_4, noise arrays filled with the
reference's hash pairs (make_golden.noise, components cos and sin).
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import make_golden  # noqa: E402
import ref_extract  # noqa: E402
from make_golden_complex_thermal import _ring, _spline_globals  # noqa: E402

SHAPES = {"3d": (12, 10, 8), "odd": (9, 7, 5)}
ZN = {"u1": (0.0, 0.0, 0.0), "z4": (4.0, 1e11, 1.0)}


def main():
    c = dict(lam=1e-24, mphi=1000.0, bosonMassSquared=1.0e6, bosonCoupling=1.09,
             bosonGaugeCoupling=1.05, fermionCoupling=1.09, fermionGaugeCoupling=1.05)
    cv = [c[k] for k in ("lam", "mphi", "bosonMassSquared", "bosonCoupling",
                         "bosonGaugeCoupling", "fermionCoupling", "fermionGaugeCoupling")]
    dt, dx, eta, mu, inv_a2, T, Tm, ns = 0.05, 1.0, 0.5, 1000.0, 1.0, 3000.0, 2999.7, 40.0
    out = {}
    for zn_tag, zn in ZN.items():
        Ck = ref_extract.load_complex(zn_params=zn, pot_coeffs=(2.0, -1.0),
                                      splines=_spline_globals())
        rng = np.random.default_rng(1000 + len(zn_tag))
        p1, p2 = _ring((12, 10, 8), rng, 4000.0)
        o1, o2 = np.empty_like(p1), np.empty_like(p2)
        Ck["Vprime_field"](o1, o2, p1, p2, T, *cv)
        out[f"vf_{zn_tag}_phi1"], out[f"vf_{zn_tag}_phi2"] = p1, p2
        out[f"vf_{zn_tag}_out1"], out[f"vf_{zn_tag}_out2"] = o1, o2
        for tag, shape in SHAPES.items():
            rng = np.random.default_rng(1100 + len(tag) + len(zn_tag))
            q1, q2 = _ring(shape, rng, 4000.0)
            v1, v2 = rng.normal(0, 300.0, shape), rng.normal(0, 300.0, shape)
            for name in ("rk2_step", "rk2_step_fused"):
                key = f"{name}_{zn_tag}_{tag}"
                s = [q1.copy(), q2.copy(), v1.copy(), v2.copy()]
                for f, a in zip(("phi1", "phi2", "pi1", "pi2"), s):
                    out[f"{key}_{f}_0"] = a.copy()
                for n in range(5):
                    n1 = make_golden.noise(shape, n, make_golden.K_PASS2, ns, 0)
                    n2 = make_golden.noise(shape, n, make_golden.K_PASS2, ns, 1)
                    scratch = [np.empty(shape) for _ in range(8)]
                    if name == "rk2_step":
                        Ck[name](*s, dt, dx, eta, T, mu, *cv, n1, n2, *scratch, inv_a2)
                    else:
                        Ck[name](*s, dt, dx, eta, T, Tm, mu, *cv, n1, n2, *scratch, inv_a2)
                for f, a in zip(("phi1", "phi2", "pi1", "pi2"), s):
                    out[f"{key}_{f}_5"] = a
    make_golden.save("complex_unfused.npz", dt=dt, dx=dx, eta=eta, mu=mu, inv_a2=inv_a2, T=T,
                     T_mid=Tm, ns=ns, zn_z4=np.array(ZN["z4"]),
                     **{k: np.float64(v) for k, v in c.items()}, **out)


if __name__ == "__main__":
    main()
