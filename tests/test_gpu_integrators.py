"""BAOAB and overdamped Euler-Maruyama kernels (real and complex field, three
storages) against the oracle's simultaneous-update restatement, with hash noise."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from oracle import integrators as I  # noqa: E402
from oracle import oracle as O  # noqa: E402
from thermal_inflation_phase_transition_b200 import complex_field as CF  # noqa: E402
from thermal_inflation_phase_transition_b200 import real_field as RF  # noqa: E402

DEV = "cuda"
SHAPE = (6, 20, 18)
DT, DX, MU, IA2, GAMMA, ETA, NS = 0.05, 0.9, 1.1, 0.95, 0.8, 1.3, 0.3


def _table():
    tab, tmin, dinv = O.build_table(lambda x: O.toy_vprime(x, 1.01), 0.0, 4.0, 4096)
    return tab, tmin, dinv, 4096


def _dev(a, storage):
    t = torch.from_numpy(np.ascontiguousarray(a)).to(DEV)
    if storage == "f32c":
        return RF.to_f32c(t)
    return t.float() if storage == "f32" else t


def _host(t, storage):
    if storage == "f32c":
        return RF.from_f32c(t).cpu().numpy()
    return t.double().cpu().numpy()


TOL = {"f64": 1e-12, "f32": 3e-6, "f32c": 2e-6}


@pytest.mark.parametrize("storage", ["f64", "f32", "f32c"])
def test_real_overdamped(storage):
    tab, tmin, dinv, npts = _table()
    rng = np.random.default_rng(3)
    phi0 = rng.normal(0.4, 0.6, SHAPE)
    ref = phi0
    phi = _dev(phi0, storage)
    tabd = torch.from_numpy(tab).to(DEV)
    for n in range(3):
        ref = I.overdamped_step_table(ref, DT, DX, ETA, MU, IA2, tab, tmin, dinv, npts, NS, n, seed=4)
        RF.overdamped_euler_step_table(phi, DT, DX, ETA, MU, IA2, tabd, tmin, dinv, npts, NS, n,
                                       hash_seed=4)
    torch.cuda.synchronize()
    got = _host(phi, storage)
    assert np.abs(got - ref).max() <= TOL[storage] * np.abs(ref).max()


@pytest.mark.parametrize("storage", ["f64", "f32", "f32c"])
def test_real_baoab(storage):
    tab, tmin, dinv, npts = _table()
    rng = np.random.default_rng(4)
    phi0, pi0 = rng.normal(0.4, 0.6, SHAPE), rng.normal(0.0, 0.3, SHAPE)
    rp, rq = phi0, pi0
    phi, pi = _dev(phi0, storage), _dev(pi0, storage)
    tabd = torch.from_numpy(tab).to(DEV)
    for n in range(3):
        rp, rq = I.baoab_step_table(rp, rq, DT, DX, GAMMA, MU, IA2, tab, tmin, dinv, npts, NS, n,
                                    seed=5)
        RF.baoab_step_table(phi, pi, DT, DX, GAMMA, MU, IA2, tabd, tmin, dinv, npts, NS, n,
                            hash_seed=5)
    torch.cuda.synchronize()
    for t, r in ((phi, rp), (pi, rq)):
        assert np.abs(_host(t, storage) - r).max() <= TOL[storage] * np.abs(r).max()


@pytest.mark.parametrize("zn", [(0.0, 0.0, 0.0), (4.0, 0.01, 1.0)])
@pytest.mark.parametrize("storage", ["f64", "f32c"])
def test_complex_baoab_and_overdamped(storage, zn):
    tab, tmin, dinv, npts = _table()
    rng = np.random.default_rng(5)
    cs = (5, 18, 17)
    f0 = [rng.normal(0.5, 0.6, cs) for _ in range(2)] + [rng.normal(0.0, 0.3, cs) for _ in range(2)]
    tabd = torch.from_numpy(tab).to(DEV)
    ref = list(f0)
    dev = [_dev(a, storage) for a in f0]
    for n in range(2):
        ref = list(I.complex_baoab_step_table(*ref, DT, DX, GAMMA, MU, IA2, tab, tmin, dinv, npts,
                                              NS, n, seed=6, zn=zn))
        CF.baoab_step_table(*dev, DT, DX, GAMMA, MU, IA2, tabd, tmin, dinv, npts, NS, n, zn=zn,
                            hash_seed=6)
    ro = list(f0[:2])
    od = [_dev(a, storage) for a in f0[:2]]
    for n in range(2):
        ro = list(I.complex_overdamped_step_table(*ro, DT, DX, ETA, MU, IA2, tab, tmin, dinv, npts,
                                                  NS, n, seed=6, zn=zn))
        CF.overdamped_euler_step_table(*od, DT, DX, ETA, MU, IA2, tabd, tmin, dinv, npts, NS, n,
                                       zn=zn, hash_seed=6)
    torch.cuda.synchronize()
    tol = 1e-12 if storage == "f64" else (5e-5 if zn[2] else 5e-6)
    for t, r in list(zip(dev, ref)) + list(zip(od, ro)):
        assert np.abs(_host(t, storage) - r).max() <= tol * np.abs(r).max()


def test_baoab_without_noise_conserves_energy_at_zero_friction():
    """gamma -> 0, no noise: BAOAB is velocity Verlet, which keeps the energy of a
    harmonic lattice bounded (relative change < 1e-2 over 200 steps)."""
    from thermal_inflation_phase_transition_b200.observables import observables
    rng = np.random.default_rng(8)
    phi = torch.from_numpy(rng.normal(0, 0.1, (16, 16, 16))).to(DEV)
    pi = torch.zeros_like(phi)
    e = []
    for n in range(200):
        RF.baoab_step_table(phi, pi, 0.05, 1.0, 1e-12, 1.0, 1.0, None, 0.0, 1.0, 2, 0.0, n,
                            vpoly=(0.5, 0.0, 0.0))
        o = observables(phi, pi).cpu().numpy()
        # E = kin + grad + 0.25 phi^2 (V = 0.25 phi^2 for V' = 0.5 phi)
        e.append(o[0] + o[1] + 0.25 * o[4])
    e = np.array(e)
    assert np.abs(e / e[0] - 1).max() < 1e-2


# ----------------------------------------------- marching kernel (F32C) ----
from thermal_inflation_phase_transition_b200 import _lib as L  # noqa: E402


def _run_real(kind, shape, policy, vpoly, steps=3):
    tab, tmin, dinv, npts = _table()
    tabd = torch.from_numpy(tab).to(DEV)
    rng = np.random.default_rng(8)
    phi = _dev(rng.normal(0.4, 0.6, shape), "f32c")
    pi = _dev(rng.normal(0.0, 0.3, shape), "f32c")
    L.set_kernel_policy(policy)
    try:
        for n in range(steps):
            if kind == "overdamped":
                RF.overdamped_euler_step_table(phi, DT, DX, ETA, MU, IA2, tabd, tmin, dinv, npts,
                                               NS, n, hash_seed=4, vpoly=vpoly)
            else:
                RF.baoab_step_table(phi, pi, DT, DX, GAMMA, MU, IA2, tabd, tmin, dinv, npts, NS,
                                    n, hash_seed=4, vpoly=vpoly)
        torch.cuda.synchronize()
    finally:
        L.set_kernel_policy(0)
    return phi.clone(), pi.clone()


@pytest.mark.parametrize("kind", ["overdamped", "baoab"])
@pytest.mark.parametrize("shape", [(8, 12, 64), (5, 6, 32), (33, 8, 128), (3, 4, 8),
                                   (4, 8, 512)])  # 512-site rows: the fixed-geometry kernels
@pytest.mark.parametrize("vpoly", [None, (-0.02, -0.15, 0.1)])
def test_real_integrators_marching_equals_generic(kind, shape, vpoly):
    """Compensated FP32 with nz % 4 == 0 runs on the marching ring: bitwise the
    generic kernel's result (same per-site arithmetic)."""
    a = _run_real(kind, shape, 1, vpoly)
    b = _run_real(kind, shape, 0, vpoly)
    assert torch.equal(a[0], b[0]) and torch.equal(a[1], b[1])
    assert L.device_status() == 0


def test_real_overdamped_marching_vs_oracle():
    tab, tmin, dinv, npts = _table()
    shape = (10, 8, 32)
    rng = np.random.default_rng(3)
    ref = rng.normal(0.4, 0.6, shape)
    phi = _dev(ref, "f32c")
    tabd = torch.from_numpy(tab).to(DEV)
    for n in range(3):
        ref = I.overdamped_step_table(ref, DT, DX, ETA, MU, IA2, tab, tmin, dinv, npts, NS, n, seed=4)
        RF.overdamped_euler_step_table(phi, DT, DX, ETA, MU, IA2, tabd, tmin, dinv, npts, NS, n,
                                       hash_seed=4)
    torch.cuda.synchronize()
    got = _host(phi, "f32c")
    assert np.abs(got - ref).max() <= TOL["f32c"] * np.abs(ref).max()


def _run_complex(kind, shape, policy, vpoly, zn, eps4, steps=3):
    from oracle import oracle as O2
    tab, tmin, dinv = O2.build_table(lambda x: O2.toy_vprime_rho(x, 0.98), 0.0, 3.0, 2048)
    tabd = torch.from_numpy(tab).to(DEV)
    rng = np.random.default_rng(12)
    f = [_dev(rng.normal(0.3, 0.5, shape), "f32c") for _ in range(2)]
    v = [_dev(rng.normal(0.0, 0.3, shape), "f32c") for _ in range(2)]
    L.set_kernel_policy(policy)
    try:
        for n in range(steps):
            if kind == "overdamped":
                CF.overdamped_euler_step_table(f[0], f[1], DT, DX, ETA, MU, IA2, tabd, tmin, dinv,
                                               2048, NS, n, zn=zn, eps4=eps4, hash_seed=5,
                                               vpoly=vpoly)
            else:
                CF.baoab_step_table(f[0], f[1], v[0], v[1], DT, DX, GAMMA, MU, IA2, tabd, tmin,
                                    dinv, 2048, NS, n, zn=zn, eps4=eps4, hash_seed=5, vpoly=vpoly)
        torch.cuda.synchronize()
    finally:
        L.set_kernel_policy(0)
    return [a.clone() for a in f + v]


@pytest.mark.parametrize("kind", ["overdamped", "baoab"])
@pytest.mark.parametrize("shape", [(8, 12, 64), (5, 6, 32), (3, 4, 8), (4, 8, 512)])
@pytest.mark.parametrize("vpoly,zn,eps4", [(None, (0.0, 0.0, 0.0), 1e-3),
                                           ((-0.02, -0.15, 0.1), (0.0, 0.0, 0.0), 0.0),
                                           (None, (4.0, 0.01, 1.0), 0.0)])
def test_complex_integrators_marching_equals_generic(kind, shape, vpoly, zn, eps4):
    """The complex field's integrators on the marching ring (Z_N off) equal the generic
    kernel bit for bit; with Z_N on both calls take the generic kernel."""
    a = _run_complex(kind, shape, 1, vpoly, zn, eps4)
    b = _run_complex(kind, shape, 0, vpoly, zn, eps4)
    for x, y in zip(a, b):
        assert torch.equal(x, y)
    assert L.device_status() == 0
