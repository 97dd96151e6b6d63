"""Golden fixture of the complex-field fused and inline steppers
(tests/golden/complex_thermal.npz), generated with the REFERENCE's own kernels:

    TIPT_REFERENCE_ROOT=<reference checkout> python tests/golden/make_golden_complex_thermal.py

AST-extracted complex-field kernels (ref_extract.load_complex), run unmodified:
* five steps of ``rk2_fused_table`` (C:1789-2064) with V'(rho) tables at T and
  T_mid and the noise arrays make_golden.noise fills with the reference's hash
  and Box-Muller, with Z_N off (U(1)) and on (Z_4);
* five steps of ``rk2_fused_single_pass`` (C:2765-3132) with the inline thermal
  V'(rho) (_vprime_complex_inline, C:2606-2680) from the dJ splines of
  tests/golden/thermal.npz, the complex script's _POT_COEFFS = (2, -1) and the
  script's default couplings;
* five steps of ``rk2_step_inline`` (C:3140-) from the same states with noise
  arrays.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import make_golden  # noqa: E402
import ref_extract  # noqa: E402

SHAPES = {"3d": (12, 10, 8), "odd": (17, 9, 5)}


def _spline_globals():
    th = np.load(os.path.join(HERE, "thermal.npz"))
    u, cb, cf = th["u"], th["cb"], th["cf"]
    h = float(u[1] - u[0])
    nseg = cb.shape[1]
    return {"c0_b": cb[0].copy(), "c1_b": cb[1].copy(), "c2_b": cb[2].copy(),
            "c3_b": cb[3].copy(), "c0_f": cf[0].copy(), "c1_f": cf[1].copy(),
            "c2_f": cf[2].copy(), "c3_f": cf[3].copy(), "x_min": float(u[0]), "h_y": h,
            "inv_hy": 1.0 / h, "xhi_clamp": float(u[0]) + h * nseg - 1e-12, "nseg": nseg}


def _ring(shape, rng, scale):
    rho = np.abs(rng.normal(0.8, 0.6, shape)) * scale
    th = rng.uniform(-np.pi, np.pi, shape)
    return rho * np.cos(th), rho * np.sin(th)


def gen_fused_table(out):
    dt, dx, eta, mu, inv_a2 = 0.05, 1.0, 0.7, 1.0, 1.0
    T, Tm = 1.03, 1.029
    ns = float(np.sqrt(2.0 * eta * T * dt / dx ** 3))
    ta, tmin_a, dinv_a, na = make_golden.table(T, lo=0.0, hi=4.0, n=4096)
    tb, tmin_b, dinv_b, nb_ = make_golden.table(Tm, lo=0.0, hi=3.5, n=2048)
    for zn_tag, zn in (("u1", (0.0, 0.0, 0.0)), ("z4", (4.0, 1e-2, 1.0))):
        Ck = ref_extract.load_complex(zn_params=zn)
        for tag, shape in SHAPES.items():
            rng = np.random.default_rng(700 + len(tag))
            p1, p2 = _ring(shape, rng, 1.0)
            v1, v2 = rng.normal(0, 0.3, shape), rng.normal(0, 0.3, shape)
            key = f"ft_{zn_tag}_{tag}"
            out[f"{key}_phi1_0"], out[f"{key}_phi2_0"] = p1.copy(), p2.copy()
            out[f"{key}_pi1_0"], out[f"{key}_pi2_0"] = v1.copy(), v2.copy()
            for n in range(5):
                n1 = make_golden.noise(shape, n, make_golden.K_PASS2, ns, 0)
                n2 = make_golden.noise(shape, n, make_golden.K_PASS2, ns, 1)
                tmp = [np.empty(shape) for _ in range(4)]
                Ck["rk2_fused_table"](p1, p2, v1, v2, dt, dx, eta, mu, n1, n2, *tmp, inv_a2, ta,
                                      tmin_a, dinv_a, na, tb, tmin_b, dinv_b, nb_)
            out[f"{key}_phi1_5"], out[f"{key}_phi2_5"] = p1, p2
            out[f"{key}_pi1_5"], out[f"{key}_pi2_5"] = v1, v2
    out.update(ft_dt=dt, ft_dx=dx, ft_eta=eta, ft_mu=mu, ft_inv_a2=inv_a2, ft_ns=ns,
               ft_table_T=ta, ft_tmin_T=tmin_a, ft_dinv_T=dinv_a, ft_npts_T=na, ft_table_Tm=tb,
               ft_tmin_Tm=tmin_b, ft_dinv_Tm=dinv_b, ft_npts_Tm=nb_,
               ft_zn_z4=np.array((4.0, 1e-2, 1.0)))


def gen_thermal(out):
    pot = (2.0, -1.0)
    Ck = ref_extract.load_complex(pot_coeffs=pot, splines=_spline_globals())
    c = dict(lam=1e-24, mphi=1000.0, bosonMassSquared=1.0e6, bosonCoupling=1.09,
             bosonGaugeCoupling=1.05, fermionCoupling=1.09, fermionGaugeCoupling=1.05)
    cv = [c[k] for k in ("lam", "mphi", "bosonMassSquared", "bosonCoupling",
                         "bosonGaugeCoupling", "fermionCoupling", "fermionGaugeCoupling")]
    dt, dx, eta, mu, inv_a2, T, Tm, ns = 0.05, 1.0, 0.5, 1000.0, 1.0, 3000.0, 2999.7, 40.0
    for tag, shape in SHAPES.items():
        rng = np.random.default_rng(800 + len(tag))
        p1, p2 = _ring(shape, rng, 4000.0)
        v1, v2 = rng.normal(0, 300.0, shape), rng.normal(0, 300.0, shape)
        key = f"th_{tag}"
        init = (p1.copy(), p2.copy(), v1.copy(), v2.copy())
        out[f"{key}_phi1_0"], out[f"{key}_phi2_0"], out[f"{key}_pi1_0"], out[f"{key}_pi2_0"] = \
            (a.copy() for a in init)
        for n in range(5):
            tmp = [np.empty(shape) for _ in range(4)]
            Ck["rk2_fused_single_pass"](p1, p2, v1, v2, dt, dx, eta, T, Tm, mu, *cv, ns,
                                        np.uint64(n), *tmp, inv_a2)
        out[f"{key}_phi1_5"], out[f"{key}_phi2_5"] = p1, p2
        out[f"{key}_pi1_5"], out[f"{key}_pi2_5"] = v1, v2
        p1, p2, v1, v2 = (a.copy() for a in init)
        for n in range(5):
            n1 = make_golden.noise(shape, n, make_golden.K_PASS2, ns, 0)
            n2 = make_golden.noise(shape, n, make_golden.K_PASS2, ns, 1)
            tmp = [np.empty(shape) for _ in range(4)]
            Ck["rk2_step_inline"](p1, p2, v1, v2, dt, dx, eta, T, mu, *cv, n1, n2, *tmp, inv_a2)
        out[f"{key}_inline_phi1_5"], out[f"{key}_inline_phi2_5"] = p1, p2
        out[f"{key}_inline_pi1_5"], out[f"{key}_inline_pi2_5"] = v1, v2
    out.update(th_pot_coeffs=np.array(pot), th_dt=dt, th_dx=dx, th_eta=eta, th_mu=mu,
               th_inv_a2=inv_a2, th_T=T, th_T_mid=Tm, th_ns=ns,
               **{f"th_{k}": np.float64(v) for k, v in c.items()})


def main():
    out = {}
    gen_fused_table(out)
    gen_thermal(out)
    make_golden.save("complex_thermal.npz", **out)


if __name__ == "__main__":
    main()
