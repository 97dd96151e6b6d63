"""Complex-field fused and inline steppers on the GPU against the reference's own
kernels (tests/golden/make_golden_complex_thermal.py): rk2_fused_table
(C:1789-2064, V'(rho) tables at T and T_mid, noise arrays, U(1) and Z_4),
rk2_fused_single_pass (C:2765-3132) and rk2_step_inline (C:3140-) with the inline
thermal V'(rho) from the reference's dJ splines."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from thermal_inflation_phase_transition_b200 import _lib as L  # noqa: E402
from thermal_inflation_phase_transition_b200 import complex_field as CF  # noqa: E402
from thermal_inflation_phase_transition_b200 import real_field as RF  # noqa: E402

FIELDS = ("phi1", "phi2", "pi1", "pi2")
COUPLINGS = ("lam", "mphi", "bosonMassSquared", "bosonCoupling", "bosonGaugeCoupling",
             "fermionCoupling", "fermionGaugeCoupling")


def _state(g, key, storage):
    st = [torch.from_numpy(g[f"{key}_{f}_0"]).cuda() for f in FIELDS]
    return [RF.to_f32c(a) for a in st] if storage == "f32c" else st


def _np(t):
    return (RF.from_f32c(t) if t.dim() == 4 else t).double().cpu().numpy()


def _check(st, g, prefix, tol):
    for a, f in zip(st, FIELDS):
        ref = g[f"{prefix}_{f}_5"]
        err = np.abs(_np(a) - ref).max()
        assert err <= tol * np.abs(ref).max(), (prefix, f, err)


def _noise(shape, step, scale, component):
    out = torch.empty(shape, dtype=torch.float64, device="cuda")
    RF.generate_noise_field(out, scale, step, component=component)
    return out


def _pot(th):
    from thermal_inflation_phase_transition_b200.thermal import ThermalPotential
    return ThermalPotential(splines=(th["cb"], th["cf"]), n_y=th["u"].size,
                            ymax=float(th["u"][-1]), pot_coeffs=(2.0, -1.0))


def _fused_table_run(g, key, storage, zn, *, noise=True, policy=0):
    st = _state(g, key, storage)
    tmp = [torch.empty_like(a) for a in st]
    p = {k: float(g[f"ft_{k}"]) for k in ("dt", "dx", "eta", "mu", "inv_a2", "ns")}
    tabs = (torch.from_numpy(g["ft_table_T"]).cuda(), float(g["ft_tmin_T"]),
            float(g["ft_dinv_T"]), int(g["ft_npts_T"]), torch.from_numpy(g["ft_table_Tm"]).cuda(),
            float(g["ft_tmin_Tm"]), float(g["ft_dinv_Tm"]), int(g["ft_npts_Tm"]))
    shape = tuple(g[f"{key}_phi1_0"].shape)
    L.set_kernel_policy(policy)
    try:
        for n in range(5):
            if noise:
                n1 = _noise(shape, n, p["ns"], 0)
                n2 = _noise(shape, n, p["ns"], 1)
                kw = {}
            else:
                n1 = n2 = None
                kw = dict(noise_scale=p["ns"], noise_step=n)
            CF.rk2_fused_table(*st, p["dt"], p["dx"], p["eta"], p["mu"], n1, n2, *tmp,
                               p["inv_a2"], *tabs, zn=zn, **kw)
        torch.cuda.synchronize()
    finally:
        L.set_kernel_policy(0)
    return st


@pytest.mark.parametrize("zn", ["u1", "z4"])
@pytest.mark.parametrize("tag", ["3d", "odd"])
@pytest.mark.parametrize("storage", ["f64", "f32c"])
def test_complex_fused_table_vs_reference(golden, zn, tag, storage):
    """Five steps of the two-table fused step, noise arrays filled with the
    reference's hash pairs, against the reference kernel."""
    g = golden("complex_thermal.npz")
    znp = tuple(g["ft_zn_z4"]) if zn == "z4" else (0.0, 0.0, 0.0)
    st = _fused_table_run(g, f"ft_{zn}_{tag}", storage, znp)
    # f32c: FP32 forces (U(1)); the Z_N force grows like 1/rho at small rho (as
    # in the single-table complex step), hence the wider Z_4 bound
    tol = 1e-12 if storage == "f64" else (5e-5 if zn == "z4" else 5e-6)
    _check(st, g, f"ft_{zn}_{tag}", tol)


def test_complex_fused_table_marching_equals_generic(golden):
    """The compensated-FP32 marching kernel and the generic kernel give the same
    bits for the fused step with inline hash noise."""
    g = golden("complex_thermal.npz")
    a = _fused_table_run(g, "ft_u1_3d", "f32c", (0.0, 0.0, 0.0), noise=False, policy=0)
    b = _fused_table_run(g, "ft_u1_3d", "f32c", (0.0, 0.0, 0.0), noise=False, policy=1)
    assert all(torch.equal(x, y) for x, y in zip(a, b))


def test_complex_fused_table_hash_noise_vs_oracle(golden):
    """Inline hash noise: multiplier 73856093 in the first half, 19349669 in the
    second, 0.5 * noise_scale * (r cos, r sin) per half (C:2958-2974,
    C:3116-3132), against the oracle's restatement."""
    from oracle import oracle as O
    from oracle.complex_steps import midpoint, table_force
    g = golden("complex_thermal.npz")
    key = "ft_u1_odd"
    st = _fused_table_run(g, key, "f64", (0.0, 0.0, 0.0), noise=False)
    s = [g[f"{key}_{f}_0"].copy() for f in FIELDS]
    p = {k: float(g[f"ft_{k}"]) for k in ("dt", "dx", "eta", "mu", "inv_a2", "ns")}
    shape = s[0].shape
    for n in range(5):
        for tk, mul in (("T", O.K_PASS2), ("Tm", O.K_PASS4)):
            f = table_force(g[f"ft_table_{tk}"], float(g[f"ft_tmin_{tk}"]),
                            float(g[f"ft_dinv_{tk}"]), int(g[f"ft_npts_{tk}"]))
            z1 = O.noise_field(shape, n, mul, 0, p["ns"], 0)
            z2 = O.noise_field(shape, n, mul, 0, p["ns"], 1)
            midpoint(s, 0.5 * p["dt"], 0.5 * p["dt"], p["dx"], p["eta"], p["mu"], p["inv_a2"], f,
                     0.5 * z1, 0.5 * z2)
    for a, want in zip(st, s):
        assert np.abs(_np(a) - want).max() <= 1e-12 * np.abs(want).max()


@pytest.mark.parametrize("tag", ["3d", "odd"])
@pytest.mark.parametrize("storage", ["f64", "f32c"])
def test_complex_fused_single_pass_thermal_vs_reference(golden, tag, storage):
    """rk2_fused_single_pass with the inline thermal V'(rho) (the reference's dJ
    splines, pot_coeffs (2, -1)) against the reference kernel's five steps."""
    g = golden("complex_thermal.npz")
    tp = _pot(golden("thermal.npz"))
    key = f"th_{tag}"
    st = _state(g, key, storage)
    tmp = [torch.empty_like(a) for a in st]
    p = {k: float(g[f"th_{k}"]) for k in ("dt", "dx", "eta", "mu", "inv_a2", "T", "T_mid", "ns")}
    c = [float(g[f"th_{k}"]) for k in COUPLINGS]
    for n in range(5):
        CF.rk2_fused_single_pass(*st, p["dt"], p["dx"], p["eta"], p["T"], p["T_mid"], p["mu"], *c,
                                 p["ns"], n, *tmp, p["inv_a2"], splines=tp)
    torch.cuda.synchronize()
    _check(st, g, key, 1e-11 if storage == "f64" else 2e-6)


@pytest.mark.parametrize("tag", ["3d", "odd"])
@pytest.mark.parametrize("storage", ["f64", "f32c"])
def test_complex_step_inline_thermal_vs_reference(golden, tag, storage):
    """rk2_step_inline (the midpoint step with the inline thermal V'(rho)), driven
    by noise arrays of the reference's hash pairs, against the reference kernel."""
    g = golden("complex_thermal.npz")
    tp = _pot(golden("thermal.npz"))
    key = f"th_{tag}"
    st = _state(g, key, storage)
    tmp = [torch.empty_like(a) for a in st]
    p = {k: float(g[f"th_{k}"]) for k in ("dt", "dx", "eta", "mu", "inv_a2", "T", "ns")}
    c = [float(g[f"th_{k}"]) for k in COUPLINGS]
    shape = tuple(g[f"{key}_phi1_0"].shape)
    for n in range(5):
        n1 = _noise(shape, n, p["ns"], 0)
        n2 = _noise(shape, n, p["ns"], 1)
        CF.rk2_step_inline(*st, p["dt"], p["dx"], p["eta"], p["T"], p["mu"], *c, n1, n2, *tmp,
                           p["inv_a2"], splines=tp)
    torch.cuda.synchronize()
    _check(st, g, f"{key}_inline", 1e-11 if storage == "f64" else 2e-6)


def test_complex_thermal_rejects_mismatched_noise(golden):
    g = golden("complex_thermal.npz")
    st = _state(g, "th_3d", "f64")
    tmp = [torch.empty_like(a) for a in st]
    n1 = torch.zeros_like(st[0])
    with pytest.raises(ValueError):
        CF.rk2_step_inline(*st, 0.05, 1.0, 0.5, 3000.0, 1000.0, 1e-24, 1000.0, 1e6, 1.09, 1.05,
                           1.09, 1.05, n1, None, *tmp, 1.0, splines=_pot(golden("thermal.npz")))


# ------------------------------------- complex un-fused stepper (C:1452-1737) ---
ZN_TAGS = ("u1", "z4")


def _zn_of(g, zn_tag):
    return tuple(g["zn_z4"]) if zn_tag == "z4" else (0.0, 0.0, 0.0)


@pytest.mark.parametrize("zn_tag", ZN_TAGS)
def test_complex_vprime_field_vs_reference(golden, zn_tag):
    g = golden("complex_unfused.npz")
    tp = _pot(golden("thermal.npz"))
    p1 = torch.from_numpy(g[f"vf_{zn_tag}_phi1"]).cuda()
    p2 = torch.from_numpy(g[f"vf_{zn_tag}_phi2"]).cuda()
    o1, o2 = torch.empty_like(p1), torch.empty_like(p2)
    CF.Vprime_field(o1, o2, p1, p2, float(g["T"]), *[float(g[k]) for k in COUPLINGS],
                    zn=_zn_of(g, zn_tag), splines=tp)
    for got, k in ((o1, "out1"), (o2, "out2")):
        ref = g[f"vf_{zn_tag}_{k}"]
        assert np.abs(got.cpu().numpy() - ref).max() <= 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize("name", ["rk2_step", "rk2_step_fused"])
@pytest.mark.parametrize("zn_tag", ZN_TAGS)
@pytest.mark.parametrize("tag", ["3d", "odd"])
@pytest.mark.parametrize("storage", ["f64", "f32c"])
def test_complex_unfused_vs_reference(golden, name, zn_tag, tag, storage):
    """Five steps of the complex script's rk2_step / rk2_step_fused (Vprime_field
    with the reference's dJ splines, pot_coeffs (2, -1), noise arrays) against the
    reference kernels; f32c with Z_4 gets the wider bound of the Z_N force."""
    g = golden("complex_unfused.npz")
    tp = _pot(golden("thermal.npz"))
    key = f"{name}_{zn_tag}_{tag}"
    st = _state(g, key, storage)
    mid = [torch.empty_like(a) for a in st]
    p = {k: float(g[k]) for k in ("dt", "dx", "eta", "mu", "inv_a2", "T", "T_mid", "ns")}
    c = [float(g[k]) for k in COUPLINGS]
    shape = tuple(g[f"{key}_phi1_0"].shape)
    ids = [id(a) for a in st]
    for n in range(5):
        n1, n2 = _noise(shape, n, p["ns"], 0), _noise(shape, n, p["ns"], 1)
        if name == "rk2_step":
            CF.rk2_step(*st, p["dt"], p["dx"], p["eta"], p["T"], p["mu"], *c, n1, n2, None, None,
                        None, None, *mid, p["inv_a2"], zn=_zn_of(g, zn_tag), splines=tp)
        else:
            CF.rk2_step_fused(*st, p["dt"], p["dx"], p["eta"], p["T"], p["T_mid"], p["mu"], *c,
                              n1, n2, None, None, None, None, *mid, p["inv_a2"],
                              zn=_zn_of(g, zn_tag), splines=tp)
    torch.cuda.synchronize()
    assert [id(a) for a in st] == ids
    tol = 1e-11 if storage == "f64" else (5e-5 if zn_tag == "z4" else 2e-6)
    _check(st, g, key, tol)
