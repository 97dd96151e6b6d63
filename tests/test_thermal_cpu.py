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
