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


# ------------------------------------------ rk2_fused_single_pass, thermal V' ---
def _single_pass_run(g, tag, storage, policy=0):
    from thermal_inflation_phase_transition_b200 import _lib as L
    from thermal_inflation_phase_transition_b200 import real_field as RF
    from thermal_inflation_phase_transition_b200.thermal import ThermalPotential
    tp = ThermalPotential(splines=(g["cb"], g["cf"]), n_y=g["u"].size, ymax=float(g["u"][-1]),
                          pot_coeffs=tuple(g["pot_coeffs"]))
    phi = torch.from_numpy(g[f"{tag}_phi0"]).cuda()
    pi = torch.from_numpy(g[f"{tag}_pi0"]).cuda()
    if storage == "f32c":
        phi, pi = RF.to_f32c(phi), RF.to_f32c(pi)
    tmp = [torch.empty_like(phi), torch.empty_like(pi)]
    keys = ("lam", "mphi", "bosonMassSquared", "bosonCoupling", "bosonGaugeCoupling",
            "fermionCoupling", "fermionGaugeCoupling")
    L.set_kernel_policy(policy)
    try:
        for n in range(5):
            RF.rk2_fused_single_pass(phi, pi, float(g["dt"]), float(g["dx"]), float(g["eta"]),
                                     float(g["T"]), float(g["T_mid"]), float(g["mu"]),
                                     *[float(g[k]) for k in keys], float(g["ns"]), n, *tmp,
                                     float(g["inv_a2"]), splines=tp)
        torch.cuda.synchronize()
    finally:
        L.set_kernel_policy(0)
    if storage == "f32c":
        return RF.from_f32c(phi).cpu().numpy(), RF.from_f32c(pi).cpu().numpy(), phi, pi
    return phi.cpu().numpy(), pi.cpu().numpy(), phi, pi


@pytest.mark.parametrize("tag", ["3d", "odd"])
@pytest.mark.parametrize("storage", ["f64", "f32c"])
def test_fused_single_pass_thermal_vs_reference(golden, tag, storage):
    """rk2_fused_single_pass with the thermal inline V' (nonzero couplings, the
    reference's dJ splines) against the reference kernel's five-step trajectory."""
    g = golden("thermal_inline.npz")
    phi, pi, _, _ = _single_pass_run(g, tag, storage)
    tol = 1e-11 if storage == "f64" else 2e-6
    for got, key in ((phi, f"{tag}_phi5"), (pi, f"{tag}_pi5")):
        ref = g[key]
        assert np.abs(got - ref).max() <= tol * np.abs(ref).max(), (key, np.abs(got - ref).max())


def test_fused_single_pass_thermal_marching_equals_generic(golden):
    g = golden("thermal_inline.npz")
    a = _single_pass_run(g, "3d", "f32c", policy=1)
    b = _single_pass_run(g, "3d", "f32c", policy=0)
    assert torch.equal(a[2], b[2]) and torch.equal(a[3], b[3])


@pytest.mark.parametrize("tag", ["3d", "odd"])
@pytest.mark.parametrize("storage", ["f64", "f32c"])
def test_step_inline_thermal_vs_reference(golden, tag, storage):
    """rk2_step_inline (R:2654-2822: the midpoint step with the thermal V' inline),
    driven by the reference's noise arrays, against the reference kernel."""
    from thermal_inflation_phase_transition_b200 import real_field as RF
    from thermal_inflation_phase_transition_b200.thermal import ThermalPotential
    g = golden("thermal_inline.npz")
    tp = ThermalPotential(splines=(g["cb"], g["cf"]), n_y=g["u"].size, ymax=float(g["u"][-1]),
                          pot_coeffs=tuple(g["pot_coeffs"]))
    phi = torch.from_numpy(g[f"{tag}_phi0"]).cuda()
    pi = torch.from_numpy(g[f"{tag}_pi0"]).cuda()
    if storage == "f32c":
        phi, pi = RF.to_f32c(phi), RF.to_f32c(pi)
    tmp = [torch.empty_like(phi), torch.empty_like(pi)]
    keys = ("lam", "mphi", "bosonMassSquared", "bosonCoupling", "bosonGaugeCoupling",
            "fermionCoupling", "fermionGaugeCoupling")
    for n in range(5):
        RF.rk2_step_inline(phi, pi, float(g["dt"]), float(g["dx"]), float(g["eta"]),
                           float(g["T"]), float(g["mu"]), *[float(g[k]) for k in keys],
                           torch.from_numpy(g[f"{tag}_noise{n}"]).cuda(), *tmp,
                           float(g["inv_a2"]), splines=tp)
    torch.cuda.synchronize()
    if storage == "f32c":
        phi, pi = RF.from_f32c(phi), RF.from_f32c(pi)
    tol = 1e-11 if storage == "f64" else 2e-6
    for got, key in ((phi, f"{tag}_inline_phi5"), (pi, f"{tag}_inline_pi5")):
        ref = g[key]
        got = got.cpu().numpy()
        assert np.abs(got - ref).max() <= tol * np.abs(ref).max(), (key, np.abs(got - ref).max())


def test_module_level_reference_names(golden):
    """thermal.Vprime_scalar / build_vprime_table (R:805, R:840) with the reference's
    splines against the reference's table."""
    g = golden("thermal.npz")
    pot = _pot(g, splines=(g["cb"], g["cf"]))
    tab, tmin, dinv = TH.build_vprime_table(float(g["T"]), -20000.0, 20000.0, 4096, potential=pot)
    ref = g["table"]
    np.testing.assert_allclose(tab.cpu().numpy(), ref, rtol=1e-11, atol=1e-11 * np.abs(ref).max())
    x = np.linspace(-20000.0, 20000.0, 4096)
    for i in (0, 1000, 2048, 4095):
        v = TH.Vprime_scalar(x[i], float(g["T"]), potential=pot)
        assert abs(v - ref[i]) <= 1e-11 * np.abs(ref).max()
