"""Thermal V' on the GPU against fixtures from the reference's own code
(tests/golden/make_golden_thermal.py): dJ quadratures, the counterterm, the
Vprime_field kernel and build_vprime_table."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from thermal_inflation_phase_transition_b200 import thermal as TH  # noqa: E402

COUPLINGS = ("lam", "mphi", "bosonMassSquared", "bosonCoupling", "bosonGaugeCoupling",
             "fermionCoupling", "fermionGaugeCoupling")


def _pot(g, **kw):
    return TH.ThermalPotential(**{k: float(g[k]) for k in COUPLINGS}, **kw)


def test_dj_quadrature_matches_reference(golden):
    g = golden("thermal.npz")
    for fermion, key in ((False, "djb"), (True, "djf")):
        got = TH.dj_grid(g["u"], fermion=fermion)
        assert np.abs(got - g[key]).max() <= 2e-8 * np.abs(g[key]).max()
        assert got[0] == 0.0


def test_counterterm_soft_subtraction(golden):
    g = golden("thermal.npz")
    xc = float(g["x_cut"])
    for fermion, key, soft in ((False, "djb", "soft_b"), (True, "djf", "soft_f")):
        got = TH.dj_grid(g["u"], fermion=fermion, x_cut=xc)
        want = g[key] - g[soft]
        assert np.abs(got - want).max() <= 2e-8 * np.abs(want).max()


def test_vprime_field_with_reference_splines(golden):
    g = golden("thermal.npz")
    pot = _pot(g, splines=(g["cb"], g["cf"]))
    phi = torch.from_numpy(g["phi"]).cuda()
    got = pot.vprime_field(phi, float(g["T"])).cpu().numpy()
    ref = g["vprime_field"]
    np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())


def test_vprime_table_with_reference_splines(golden):
    g = golden("thermal.npz")
    pot = _pot(g, splines=(g["cb"], g["cf"]))
    tab, tmin, dinv = pot.table(float(g["T"]), -20000.0, 20000.0, 4096)
    ref = g["table"]
    assert tmin == float(g["tmin"]) and dinv == float(g["dinv"])
    np.testing.assert_allclose(tab.cpu().numpy(), ref, rtol=1e-11, atol=1e-11 * np.abs(ref).max())


def test_full_pipeline_matches_reference(golden):
    """Own quadrature and own spline, end to end, against the reference's V'."""
    g = golden("thermal.npz")
    pot = _pot(g)
    phi = torch.from_numpy(g["phi"]).cuda()
    got = pot.vprime_field(phi, float(g["T"])).cpu().numpy()
    ref = g["vprime_field"]
    assert np.abs(got - ref).max() <= 1e-7 * np.abs(ref).max()


def test_thermal_table_drives_the_stepper():
    from thermal_inflation_phase_transition_b200 import driver as D
    pot = TH.ThermalPotential()
    tab = pot.table_2d(-20000.0, 20000.0, 1024, 2000.0, 4000.0, 32)
    sched = D.constant_temperature(3000.0, 20, dt=0.05)
    sim = D.Simulation((16, 16, 16), storage="f64", table=tab, schedule=sched, seed=1,
                       init_sigma=100.0, graph_steps=10)
    obs = sim.run(20)
    assert np.isfinite(obs).all() and obs[-1, 9] == 0
