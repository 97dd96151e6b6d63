"""Host-side schedule builders of the step driver (no GPU)."""
import math

import numpy as np

from thermal_inflation_phase_transition_b200 import driver as D


def test_hubble_param_matches_reference_form():
    # R:706-710: chi_g^2 = 30 / (pi^2 g*), H^2 = (T^4 / chi_g^2 + del_V) / (3 M_pl^2)
    for T in (10.0, 7350.0, 1e6):
        chig2 = 30.0 / (np.pi ** 2 * D.G_STAR)
        ref = math.sqrt((T ** 4 / chig2 + D.DEL_V) / (3.0 * D.M_PL ** 2))
        assert abs(D.hubble_param(T) - ref) <= 1e-14 * ref


def test_hubble_expansion_schedule():
    """Rows follow R:3621-3636 and R:3714-3718: T = T0/a, a_{n+1} = a_n (1 + H_n dt/mu),
    eta_eff = eta + 3H/mu, inv_a2 = 1/a^2, ns = sqrt(2 eta_eff T dt / a^3 / (mu^2 dx^3))."""
    T0, dt, eta, mu, dxp = 7350.0, 0.1, 7.35, 1000.0, 1e-3
    # a large vacuum energy makes the expansion visible within a few steps
    s, a_end = D.hubble_expansion(T0, 50, dt=dt, eta=eta, mu=mu, dx_phys=dxp, del_v=1e44)
    a = 1.0
    for n in range(50):
        T, ns, eta_eff, inv_a2 = s[n]
        H = D.hubble_param(T0 / a, del_v=1e44)
        assert abs(T - T0 / a) <= 1e-13 * T
        assert abs(eta_eff - (eta + 3.0 * H / mu)) <= 1e-13 * eta_eff
        assert abs(inv_a2 - 1.0 / a ** 2) <= 1e-13
        ref_ns = math.sqrt(2.0 * eta_eff * T * dt / a ** 3 / (mu ** 2 * dxp ** 3))
        assert abs(ns - ref_ns) <= 1e-13 * ref_ns
        a += a * H * (dt / mu)
    assert abs(a_end - a) <= 1e-13 * a and a > 1.0 + 1e-6
    assert np.all(np.diff(s[:, 0]) < 0)
    flat, _ = D.hubble_expansion(T0, 5, dt=dt, eta=eta, mu=mu, scale_factor=False,
                                 noise=False, del_v=1e44)
    assert np.all(flat[:, 2] == eta) and np.all(flat[:, 3] == 1.0) and np.all(flat[:, 1] == 0.0)
