"""Thermal V' pieces that need no GPU: the library's not-a-knot spline against the
reference's spline (scipy CubicSpline, R:437-447) of the golden dJ grids."""
import numpy as np

from thermal_inflation_phase_transition_b200.thermal import counterterm_x_cut, not_a_knot_spline


def test_spline_matches_reference_coefficients(golden):
    g = golden("thermal.npz")
    for key, c in (("djb", "cb"), ("djf", "cf")):
        got = not_a_knot_spline(g["u"], g[key])
        scale = np.abs(g[c]).max(axis=1, keepdims=True)
        assert np.abs(got - g[c]).max(axis=1).max() <= 1e-9 * scale.max()
        np.testing.assert_allclose(got[3], g[c][3], rtol=0, atol=0)  # knot values exact


def test_spline_reproduces_a_cubic_exactly():
    x = np.linspace(-1.0, 2.0, 9)
    y = 2 * x ** 3 - x ** 2 + 0.5 * x - 3
    c = not_a_knot_spline(x, y)
    assert np.allclose(c[0], 2.0) and np.allclose(c[3], y[:-1])


def test_counterterm_cut():
    assert abs(counterterm_x_cut(0.5, 2.0) - np.pi) < 1e-15


def test_inline_vprime_oracle_matches_reference(golden):
    """The oracle's restatement of _vprime_inline (R:2201-2266) against the reference
    kernel's values at sample fields (both signs, the argument clamps, phi = 0) and
    three temperatures."""
    from oracle.thermal import vprime_inline
    g = golden("thermal_inline.npz")
    keys = ("lam", "mphi", "bosonMassSquared", "bosonCoupling", "bosonGaugeCoupling",
            "fermionCoupling", "fermionGaugeCoupling")
    kw = {k: float(g[k]) for k in keys}
    u = g["u"]
    for a, T in enumerate(g["Ts"]):
        got = vprime_inline(g["phs"], float(T), g["cb"], g["cf"], float(u[0]),
                            float(u[1] - u[0]), pot_coeffs=tuple(g["pot_coeffs"]), **kw)
        want = g["vprime_inline"][a]
        np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-12 * np.abs(want).max())


_COUPLINGS = ("lam", "mphi", "bosonMassSquared", "bosonCoupling", "bosonGaugeCoupling",
              "fermionCoupling", "fermionGaugeCoupling")


def _state(g, key, n):
    return [g[f"{key}_{f}_{n}"].copy() for f in ("phi1", "phi2", "pi1", "pi2")]


def _close(got, g, key, suffix, rtol):
    for a, f in zip(got, ("phi1", "phi2", "pi1", "pi2")):
        want = g[f"{key}_{f}{suffix}"]
        assert np.abs(a - want).max() <= rtol * np.abs(want).max(), (key, f)


def test_complex_fused_table_oracle_matches_reference(golden):
    """oracle.complex_steps.rk2_fused_table against five steps of the reference's
    complex rk2_fused_table (C:1789-2064), U(1) and Z_4, noise arrays."""
    from oracle import oracle as O
    from oracle.complex_steps import rk2_fused_table
    g = golden("complex_thermal.npz")
    p = {k: g[f"ft_{k}"] for k in ("dt", "dx", "eta", "mu", "inv_a2", "ns")}
    tabs = [g[f"ft_{k}"] for k in ("table_T", "tmin_T", "dinv_T", "npts_T", "table_Tm", "tmin_Tm",
                                  "dinv_Tm", "npts_Tm")]
    tabs = [t if t.ndim else t.item() for t in tabs]
    for zn_tag, zn in (("u1", (0.0, 0.0, 0.0)), ("z4", tuple(g["ft_zn_z4"]))):
        for tag in ("3d", "odd"):
            key = f"ft_{zn_tag}_{tag}"
            s = _state(g, key, 0)
            shape = s[0].shape
            for n in range(5):
                n1 = O.noise_field(shape, n, O.K_PASS2, 0, float(p["ns"]), 0)
                n2 = O.noise_field(shape, n, O.K_PASS2, 0, float(p["ns"]), 1)
                rk2_fused_table(s, float(p["dt"]), float(p["dx"]), float(p["eta"]), float(p["mu"]),
                                n1, n2, float(p["inv_a2"]), *tabs, zn=zn)
            _close(s, g, key, "_5", 1e-12)


def test_complex_thermal_oracle_matches_reference(golden):
    """oracle.complex_steps rk2_fused_single_pass / rk2_step_inline against five
    steps of the reference's complex kernels (C:2765-3132, C:3140-) with the
    inline thermal V'(rho) and the complex script's pot_coeffs (2, -1)."""
    from oracle import oracle as O
    from oracle.complex_steps import rk2_fused_single_pass, rk2_step_inline
    g = golden("complex_thermal.npz")
    th = golden("thermal.npz")
    u, cb, cf = th["u"], th["cb"], th["cf"]
    x_min, h = float(u[0]), float(u[1] - u[0])
    c = {k: float(g[f"th_{k}"]) for k in _COUPLINGS}
    pot = tuple(g["th_pot_coeffs"])
    dt, dx, eta, mu, inv_a2, T, Tm, ns = (float(g[f"th_{k}"]) for k in
                                          ("dt", "dx", "eta", "mu", "inv_a2", "T", "T_mid", "ns"))
    for tag in ("3d", "odd"):
        key = f"th_{tag}"
        s = _state(g, key, 0)
        for n in range(5):
            rk2_fused_single_pass(s, dt, dx, eta, T, Tm, mu, c, ns, n, inv_a2, cb, cf, x_min, h,
                                  pot)
        _close(s, g, key, "_5", 1e-12)
        s = _state(g, key, 0)
        shape = s[0].shape
        for n in range(5):
            n1 = O.noise_field(shape, n, O.K_PASS2, 0, ns, 0)
            n2 = O.noise_field(shape, n, O.K_PASS2, 0, ns, 1)
            rk2_step_inline(s, dt, dx, eta, T, mu, c, n1, n2, inv_a2, cb, cf, x_min, h, pot)
        for a, f in zip(s, ("phi1", "phi2", "pi1", "pi2")):
            want = g[f"{key}_inline_{f}_5"]
            assert np.abs(a - want).max() <= 1e-12 * np.abs(want).max(), (key, f)


def test_unfused_oracle_matches_reference(golden):
    """oracle.thermal laplacian / cubic_eval_uniform / rk2_step / rk2_step_fused
    against the reference's kernels (R:1364-1656), FP64 arrays."""
    from oracle import oracle as O
    from oracle import thermal as OT
    g = golden("unfused.npz")
    th = golden("thermal.npz")
    u, cb, cf = th["u"], th["cb"], th["cf"]
    x_min, h = float(u[0]), float(u[1] - u[0])
    got = OT.cubic_eval_uniform(g["cubic_x"], x_min, h, cb.shape[1], *cb)
    np.testing.assert_allclose(got, g["cubic_out"], rtol=1e-14, atol=0)
    for tag in ("3d", "odd", "2d"):
        lap = OT.laplacian(g[f"lap_{tag}_f64_in"], float(g["lap_dx"]))
        ref = g[f"lap_{tag}_f64_out"]
        assert np.abs(lap - ref).max() <= 1e-13 * np.abs(ref).max()
    c = {k: float(g[k]) for k in _COUPLINGS}
    dt, dx, eta, mu, inv_a2, T, Tm, ns = (float(g[k]) for k in
                                          ("dt", "dx", "eta", "mu", "inv_a2", "T", "T_mid", "ns"))
    for tag in ("3d", "odd", "2d"):
        for name in ("rk2_step", "rk2_step_fused"):
            key = f"{name}_{tag}_f64"
            phi, pi = g[f"{key}_phi0"], g[f"{key}_pi0"]
            for n in range(5):
                nf = O.noise_field(phi.shape, n, O.K_PASS2, 0, ns, 0)
                if name == "rk2_step":
                    phi, pi = OT.rk2_step(phi, pi, dt, dx, eta, T, mu, c, nf, inv_a2, cb, cf,
                                          x_min, h)
                else:
                    phi, pi = OT.rk2_step_fused(phi, pi, dt, dx, eta, T, Tm, mu, c, nf, inv_a2,
                                                cb, cf, x_min, h)
            for a, f in ((phi, "phi5"), (pi, "pi5")):
                ref = g[f"{key}_{f}"]
                assert np.abs(a - ref).max() <= 1e-12 * np.abs(ref).max(), (key, f)


def test_complex_unfused_oracle_matches_reference(golden):
    """oracle.complex_steps field_force / rk2_step / rk2_step_fused against the
    complex script's Vprime_field, rk2_step and rk2_step_fused (C:1452-1737),
    U(1) and Z_4."""
    from oracle import oracle as O
    from oracle import complex_steps as CS
    g = golden("complex_unfused.npz")
    th = golden("thermal.npz")
    u, cb, cf = th["u"], th["cb"], th["cf"]
    x_min, h = float(u[0]), float(u[1] - u[0])
    c = {k: float(g[k]) for k in _COUPLINGS}
    dt, dx, eta, mu, inv_a2, T, Tm, ns = (float(g[k]) for k in
                                          ("dt", "dx", "eta", "mu", "inv_a2", "T", "T_mid", "ns"))
    for zn_tag, zn in (("u1", (0.0, 0.0, 0.0)), ("z4", tuple(g["zn_z4"]))):
        d1, d2 = CS.field_force(T, cb, cf, x_min, h, c, zn=zn)(g[f"vf_{zn_tag}_phi1"],
                                                               g[f"vf_{zn_tag}_phi2"])
        for got, k in ((d1, "out1"), (d2, "out2")):
            ref = g[f"vf_{zn_tag}_{k}"]
            assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max(), (zn_tag, k)
        for tag in ("3d", "odd"):
            for name in ("rk2_step", "rk2_step_fused"):
                key = f"{name}_{zn_tag}_{tag}"
                s = _state(g, key, 0)
                shape = s[0].shape
                for n in range(5):
                    n1 = O.noise_field(shape, n, O.K_PASS2, 0, ns, 0)
                    n2 = O.noise_field(shape, n, O.K_PASS2, 0, ns, 1)
                    if name == "rk2_step":
                        CS.rk2_step(s, dt, dx, eta, T, mu, c, n1, n2, inv_a2, cb, cf, x_min, h,
                                    zn=zn)
                    else:
                        CS.rk2_step_fused(s, dt, dx, eta, T, Tm, mu, c, n1, n2, inv_a2, cb, cf,
                                          x_min, h, zn=zn)
                _close(s, g, key, "_5", 1e-12)
