"""Pin the CPU oracle against the fixtures produced by the reference's own numba
kernels (tests/golden/make_golden.py).  CPU only."""
import numpy as np
import pytest

from oracle import oracle as O

CASES = ("2d", "3d", "odd")


def test_hash_pairs_bit_exact(golden):
    g = golden("hash_pairs.npz")
    u1, u2, z = O.hash_pair(g["seeds"])
    assert np.array_equal(u1, g["u1"])  # 53-bit integers: exact by construction
    assert np.array_equal(u2, g["u2"])
    # same libm on both sides -> Box-Muller agrees bit for bit here
    assert np.array_equal(z, g["z_cos"])


def test_hash_site0_step0_quirk(golden):
    # R:2334-2335: key 0 gives u1 = 1e-12, radius sqrt(-2 ln u1) ~ 7.4
    u1, u2, z = O.hash_pair(np.array([0], np.uint64))
    assert u1[0] == 1e-12
    assert abs(z[0]) > 6.0 and np.sqrt(-2.0 * np.log(u1[0])) > 7.4


def test_inline_noise_matches_reference_kernel(golden):
    # reference rk2_fused_single_pass with dt=0, pi=0, ns=2 leaves pi = z2 + z4
    g = golden("hash_pairs.npz")
    sh = tuple(int(x) for x in g["inline_shape"])
    step = int(g["inline_step"])
    z2 = O.noise_field(sh, step, O.K_PASS2)
    z4 = O.noise_field(sh, step, O.K_PASS4)
    # the fastmath kernel contracts pi + r*cos(theta) into an FMA, so its sum
    # differs from the rounded z2 + z4 by at most two ulps of the summands
    ulp = np.spacing(np.maximum(np.abs(z2), np.abs(z4)))
    assert np.all(np.abs(z2 + z4 - g["inline_pi"]) <= 2 * ulp)


def test_seed_zero_is_reference_key():
    for site, step in [(0, 0), (5, 7), (134217727, 19999)]:
        ref = ((site * O.K_PASS2) % 2 ** 64) ^ step
        assert O.noise_key(site, step, O.K_PASS2, 0) == ref
        assert O.noise_key(site, step, O.K_PASS2, 1) == (ref + 0x9E3779B97F4A7C15) % 2 ** 64


def _run_step_table(g, tag, dn, nsteps):
    dtype = np.float64 if dn == "f64" else np.float32
    phi = g[f"{tag}_{dn}_phi0"].copy()
    pi = g[f"{tag}_{dn}_pi0"].copy()
    tmp = [np.empty_like(phi), np.empty_like(phi)]
    for n in range(nsteps):
        O.rk2_step_table(phi, pi, float(g["dt"]), float(g["dx"]), float(g["eta"]), float(g["mu"]),
                         None if dtype == np.float64 else
                         O.noise_field(phi.shape, n, scale=float(g["ns"])).astype(np.float32),
                         *tmp, float(g["inv_a2"]), g["table"], float(g["tmin"]),
                         float(g["dinv"]), int(g["npts"]), noise_scale=float(g["ns"]),
                         noise_step=n)
    return phi, pi


@pytest.mark.parametrize("tag", CASES)
def test_rk2_step_table_f64(golden, tag):
    g = golden("rk2_step_table.npz")
    phi, pi = _run_step_table(g, tag, "f64", 1)
    np.testing.assert_allclose(phi, g[f"{tag}_f64_phi1"], rtol=0, atol=1e-14)
    np.testing.assert_allclose(pi, g[f"{tag}_f64_pi1"], rtol=0, atol=1e-14)
    phi, pi = _run_step_table(g, tag, "f64", 10)
    scale = np.abs(g[f"{tag}_f64_phi10"]).max()
    assert np.abs(phi - g[f"{tag}_f64_phi10"]).max() <= 1e-12 * scale
    assert np.abs(pi - g[f"{tag}_f64_pi10"]).max() <= 1e-12 * np.abs(g[f"{tag}_f64_pi10"]).max()


@pytest.mark.parametrize("tag", CASES)
def test_rk2_step_table_f32_mixed(golden, tag):
    g = golden("rk2_step_table.npz")
    phi, pi = _run_step_table(g, tag, "f32", 10)
    # float32 storage, FP64 arithmetic: differences are store-rounding flips
    np.testing.assert_allclose(phi, g[f"{tag}_f32_phi10"], rtol=0, atol=2e-6)
    np.testing.assert_allclose(pi, g[f"{tag}_f32_pi10"], rtol=0, atol=2e-6)


@pytest.mark.parametrize("tag", CASES)
@pytest.mark.parametrize("dn", ("f64", "f32"))
def test_rk2_fused_table(golden, tag, dn):
    g = golden("rk2_fused_table.npz")
    dtype = np.float64 if dn == "f64" else np.float32
    phi = g[f"{tag}_{dn}_phi0"].copy()
    pi = g[f"{tag}_{dn}_pi0"].copy()
    tmp = [np.empty_like(phi), np.empty_like(phi)]
    for n in range(5):
        nf = O.noise_field(phi.shape, n, scale=float(g["ns"])).astype(dtype)
        O.rk2_fused_table(phi, pi, float(g["dt"]), float(g["dx"]), float(g["eta"]), float(g["mu"]),
                          nf, *tmp, float(g["inv_a2"]), g["table_T"], float(g["tmin_T"]),
                          float(g["dinv_T"]), int(g["npts_T"]), g["table_Tm"], float(g["tmin_Tm"]),
                          float(g["dinv_Tm"]), int(g["npts_Tm"]))
    tol = 1e-13 if dn == "f64" else 2e-6
    np.testing.assert_allclose(phi, g[f"{tag}_{dn}_phi5"], rtol=0, atol=tol)
    np.testing.assert_allclose(pi, g[f"{tag}_{dn}_pi5"], rtol=0, atol=tol)


@pytest.mark.parametrize("tag", CASES)
def test_rk2_fused_single_pass_inline_hash(golden, tag):
    g = golden("rk2_fused_single_pass.npz")
    phi = g[f"{tag}_phi0"].copy()
    pi = g[f"{tag}_pi0"].copy()
    tmp = [np.empty_like(phi), np.empty_like(phi)]
    for n in range(5):
        O.rk2_fused_single_pass_poly(phi, pi, float(g["dt"]), float(g["dx"]), float(g["eta"]),
                                     float(g["mu"]), float(g["lam"]), float(g["mphi"]),
                                     float(g["ns"]), n, *tmp, float(g["inv_a2"]))
    np.testing.assert_allclose(phi, g[f"{tag}_phi5"], rtol=0, atol=1e-13)
    np.testing.assert_allclose(pi, g[f"{tag}_pi5"], rtol=0, atol=1e-13)


@pytest.mark.parametrize("zn", ("u1", "z4"))
@pytest.mark.parametrize("tag", CASES)
def test_complex_rk2_step_table(golden, zn, tag):
    g = golden("rk2_complex.npz")
    k = f"{zn}_{tag}"
    st = [g[f"{k}_{n}_0"].copy() for n in ("phi1", "phi2", "pi1", "pi2")]
    tmp = [np.empty_like(st[0]) for _ in range(4)]
    znp = tuple(g["zn_z4"]) if zn == "z4" else (0.0, 0.0, 0.0)
    for n in range(5):
        O.rk2_step_table_complex(*st, float(g["dt"]), float(g["dx"]), float(g["eta"]),
                                 float(g["mu"]), None, None, *tmp, float(g["inv_a2"]), g["table"],
                                 float(g["tmin"]), float(g["dinv"]), int(g["npts"]), zn=znp,
                                 noise_scale=float(g["ns"]), noise_step=n)
    for a, n in zip(st, ("phi1", "phi2", "pi1", "pi2")):
        np.testing.assert_allclose(a, g[f"{k}_{n}_5"], rtol=0, atol=1e-12)


@pytest.mark.parametrize("tag", ("a", "b", "c"))
def test_winding_matches_reference(golden, tag):
    g = golden("winding.npz")
    w, w3, cnt = O.winding(g[f"{tag}_phi1"], g[f"{tag}_phi2"])
    # the float output carries ~1e-16 rounding residue around the integers;
    # the integer windings and the string count are the exact quantities
    assert np.array_equal(np.round(w), np.round(g[f"{tag}_w"]))
    assert np.abs(w - g[f"{tag}_w"]).max() < 1e-12
    assert cnt[3] == int(g[f"{tag}_n_strings"])
    # per-site value is the sum of the three integer orientation windings
    assert np.array_equal(w3.sum(0).astype(np.float32), np.round(g[f"{tag}_w"]))
    assert cnt[0] + cnt[1] + cnt[2] > 0


@pytest.mark.parametrize("tag", ("a", "b"))
def test_winding_evolved_strings_match_reference(golden, tag):
    """String networks evolved by the reference's complex kernels (strings.npz):
    integer windings, per-orientation windings and counts are exact."""
    g = golden("strings.npz")
    w, w3, cnt = O.winding(g[f"{tag}_phi1"], g[f"{tag}_phi2"])
    assert np.array_equal(np.round(w), g[f"{tag}_w"].astype(np.float32))
    assert np.array_equal(w3, g[f"{tag}_w3"])
    assert cnt[3] == int(g[f"{tag}_n_strings"])
    assert list(cnt[:3]) == g[f"{tag}_n_pierced"].tolist()


@pytest.mark.parametrize("tag", CASES)
def test_energies(golden, tag):
    g = golden("energies.npz")
    o = O.observables(g[f"{tag}_phi"], g[f"{tag}_pi"], float(g["dx"]), float(g["inv_a2"]),
                      float(g["lam"]), float(g["mphi"]), float(g["mu"]))
    np.testing.assert_allclose([o["E_kin"], o["E_grad"], o["E_pot"]], g[f"{tag}_E"], rtol=1e-13)


def test_table_2d_blend_is_bilinear():
    t2, tmin, dinv, Tmin, Tdinv = O.build_table_2d(O.toy_vprime, 0.0, 3.0, 64, 0.95, 1.10, 16)
    row = O.table_blend_row(t2, Tmin, Tdinv, 1.0123)
    ft = (1.0123 - Tmin) * Tdinv
    it = int(ft)
    w = ft - it
    np.testing.assert_allclose(row, t2[it] + w * (t2[it + 1] - t2[it]), rtol=0, atol=0)
    # toy V' is linear in T^2 only approximately: blend error is O(dT^2)
    np.testing.assert_allclose(row, O.toy_vprime(np.linspace(0, 3, 64), 1.0123), atol=1e-4)


def test_trajectory_2d_256(golden):
    """2-D 256^2 FP64, 2000 steps: oracle vs the reference's rk2_step_table run."""
    g = golden("trajectory_2d_256.npz")
    phi = g["phi0"].copy()
    pi = np.zeros_like(phi)
    tmp = [np.empty_like(phi), np.empty_like(phi)]
    nz0 = O.noise_field(phi.shape, 0, scale=float(g["ns"]))
    assert np.array_equal(nz0, g["noise0"])
    p2 = np.empty(2000)
    for n in range(2000):
        O.rk2_step_table(phi, pi, float(g["dt"]), float(g["dx"]), float(g["eta"]), float(g["mu"]),
                         None, *tmp, float(g["inv_a2"]), g["table"], float(g["tmin"]),
                         float(g["dinv"]), int(g["npts"]), noise_scale=float(g["ns"]),
                         noise_step=n)
        p2[n] = np.mean(phi * phi)
    assert np.max(np.abs(p2 - g["phi2_mean"]) / g["phi2_mean"]) < 1e-12
    assert np.abs(phi - g["phi_final"]).max() < 1e-12
