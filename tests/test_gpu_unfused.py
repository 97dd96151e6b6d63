"""The reference's un-fused stepper and its array helpers on the GPU against the
reference's own kernels (tests/golden/make_golden_unfused.py): laplacian_periodic
(R:1364-1385), cubic_eval_uniform (R:1415-1426), Vprime_field (R:1435-1485),
rk2_step (R:1489-1550) and rk2_step_fused (R:1553-1656)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from thermal_inflation_phase_transition_b200 import real_field as RF  # noqa: E402

COUPLINGS = ("lam", "mphi", "bosonMassSquared", "bosonCoupling", "bosonGaugeCoupling",
             "fermionCoupling", "fermionGaugeCoupling")
TAGS = ("3d", "odd", "2d")


def _pot(th):
    from thermal_inflation_phase_transition_b200.thermal import ThermalPotential
    return ThermalPotential(splines=(th["cb"], th["cf"]), n_y=th["u"].size,
                            ymax=float(th["u"][-1]))


def _np(t):
    return (RF.from_f32c(t) if t.dim() == 4 else t).double().cpu().numpy()


@pytest.mark.parametrize("tag", TAGS)
@pytest.mark.parametrize("storage", ["f64", "f32", "f32c"])
def test_laplacian_periodic_vs_reference(golden, tag, storage):
    g = golden("unfused.npz")
    dn = "f32" if storage == "f32" else "f64"
    a = torch.from_numpy(g[f"lap_{tag}_{dn}_in"]).cuda()
    if storage == "f32c":
        a = RF.to_f32c(a)
    out = torch.empty_like(a)
    assert RF.laplacian_periodic(out, a, float(g["lap_dx"])) is out
    ref = g[f"lap_{tag}_{dn}_out"].astype(np.float64)
    # f32: the reference's float32 neighbour sum, rounded once more on the store
    tol = 1e-6 if storage == "f32" else 1e-13
    assert np.abs(_np(out) - ref).max() <= tol * np.abs(ref).max()


def test_cubic_eval_uniform_vs_reference(golden):
    g = golden("unfused.npz")
    th = golden("thermal.npz")
    u, cb = th["u"], th["cb"]
    c = [torch.from_numpy(np.ascontiguousarray(cb[q])).cuda() for q in range(4)]
    x = torch.from_numpy(g["cubic_x"]).cuda()
    got = RF.cubic_eval_uniform(x, float(u[0]), float(u[1] - u[0]), cb.shape[1], *c)
    # the spline's far tail is ~1e-43: bound the error by the values' scale
    ref = g["cubic_out"]
    np.testing.assert_allclose(got.cpu().numpy(), ref, rtol=1e-14, atol=1e-15 * np.abs(ref).max())
    s = RF.cubic_eval_uniform(float(g["cubic_x"][7]), float(u[0]), float(u[1] - u[0]),
                              cb.shape[1], *c)
    assert isinstance(s, float) and abs(s - g["cubic_out"][7]) <= 1e-14 * abs(g["cubic_out"][7])


def test_vprime_field_reference_signature(golden):
    g = golden("thermal.npz")
    phi = torch.from_numpy(g["phi"]).cuda()
    out = torch.empty_like(phi)
    RF.Vprime_field(out, phi, float(g["T"]), *[float(g[k]) for k in COUPLINGS],
                    splines=_pot(g))
    ref = g["vprime_field"]
    np.testing.assert_allclose(out.cpu().numpy(), ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())


def _run(g, tp, name, tag, storage):
    dn = "f32" if storage == "f32" else "f64"
    key = f"{name}_{tag}_{dn}"
    phi = torch.from_numpy(g[f"{key}_phi0"]).cuda()
    pi = torch.from_numpy(g[f"{key}_pi0"]).cuda()
    if storage == "f32c":
        phi, pi = RF.to_f32c(phi), RF.to_f32c(pi)
    ndt = torch.float32 if storage == "f32" else torch.float64
    p = {k: float(g[k]) for k in ("dt", "dx", "eta", "mu", "inv_a2", "T", "T_mid", "ns")}
    c = [float(g[k]) for k in COUPLINGS]
    shape = tuple(g[f"{key}_phi0"].shape)
    lap, vp = torch.empty_like(phi), torch.empty_like(phi)
    mid = [torch.empty_like(phi), torch.empty_like(pi)]
    phi_id = phi
    for n in range(5):
        noise = torch.empty(shape, dtype=ndt, device="cuda")
        RF.generate_noise_field(noise, p["ns"], n)
        if name == "rk2_step":
            RF.rk2_step(phi, pi, p["dt"], p["dx"], p["eta"], p["T"], p["mu"], *c, noise, lap, vp,
                        *mid, p["inv_a2"], splines=tp)
        else:
            RF.rk2_step_fused(phi, pi, p["dt"], p["dx"], p["eta"], p["T"], p["T_mid"], p["mu"],
                              *c, noise, lap, vp, *mid, p["inv_a2"], splines=tp)
    torch.cuda.synchronize()
    assert phi is phi_id  # updated in place, as the reference
    return key, _np(phi), _np(pi)


@pytest.mark.parametrize("name", ["rk2_step", "rk2_step_fused"])
@pytest.mark.parametrize("tag", TAGS)
@pytest.mark.parametrize("storage", ["f64", "f32", "f32c"])
def test_unfused_steppers_vs_reference(golden, name, tag, storage):
    """Five steps with the thermal V' (the reference's dJ splines and default
    couplings) and the reference's noise arrays, against the reference kernels.
    f32: the reference rounds the Laplacian and V' arrays to float32 between its
    passes, the fused kernel keeps them in FP64, hence 1e-5 of the field scale."""
    g = golden("unfused.npz")
    key, phi, pi = _run(g, _pot(golden("thermal.npz")), name, tag, storage)
    tol = {"f64": 1e-11, "f32": 1e-5, "f32c": 2e-6}[storage]
    for got, f in ((phi, "phi5"), (pi, "pi5")):
        ref = g[f"{key}_{f}"].astype(np.float64)
        assert np.abs(got - ref).max() <= tol * np.abs(ref).max(), (key, f,
                                                                   np.abs(got - ref).max())
