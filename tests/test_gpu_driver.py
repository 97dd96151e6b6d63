"""The graph-captured host driver: device schedule + step counter, replayed chunks."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from thermal_inflation_phase_transition_b200 import driver as D  # noqa: E402


def test_driver_2d_trajectory_matches_reference(golden):
    """2-D 256^2 FP64, 2000 graph-replayed steps: the <phi^2> curve of the reference run."""
    g = golden("trajectory_2d_256.npz")
    tab = D.Table1D(g["table"], float(g["tmin"]), float(g["dinv"]))
    sched = D.constant_temperature(float(g["T"]), 2000, dt=float(g["dt"]), eta=float(g["eta"]))
    assert abs(sched[0, 1] - float(g["ns"])) < 1e-15
    sim = D.Simulation((256, 256, 1), storage="f64", dt=float(g["dt"]), dx=float(g["dx"]),
                       eta=float(g["eta"]), mu=float(g["mu"]), inv_a2=float(g["inv_a2"]),
                       table=tab, schedule=sched, seed=0, phi0=g["phi0"],
                       pi0=np.zeros_like(g["phi0"]), graph_steps=100)
    obs = sim.run(2000)
    rel = np.abs(obs[:, D.OBS_INDEX["phi2_mean"]] - g["phi2_mean"]) / g["phi2_mean"]
    assert rel.max() < 1e-11, rel.max()
    phi, _ = sim.fields()
    assert np.abs(phi.cpu().numpy() - g["phi_final"]).max() < 1e-11


@pytest.mark.parametrize("storage", ["f64", "f32c"])
def test_graphs_equal_eager(storage):
    tab = D.Table2D.build(D.toy_vprime, 0.0, 3.0, 4096, 0.97, 1.06, 64)
    sched = D.linear_cooling(1.05, 0.98, 10000, 130, dt=0.05)
    kw = dict(storage=storage, table=tab, schedule=sched, seed=1, init_seed=3, graph_steps=20)
    a = D.Simulation((16, 12, 32), **kw)
    b = D.Simulation((16, 12, 32), **kw)
    oa = a.run(130)                      # 6 graph chunks + an eager remainder of 10
    ob = b.run(130, use_graphs=False)
    assert np.array_equal(oa, ob)
    for x, y in zip(a.fields(), b.fields()):
        assert torch.equal(x, y)


@pytest.mark.parametrize("shape", [(64, 64, 64), (128, 128, 128), (256, 256, 256)])
def test_f32c_driver_tracks_fp64_cooling(shape):
    """T cooling 1.05 -> 0.98 on a 2-D table over the full 10^4 steps: <phi^2> of the
    compensated-FP32 run within 1e-6 of the FP64 run at every step (up to 256^3, the
    lattice of the two-storage cooling comparison)."""
    tab = D.Table2D.build(D.toy_vprime, 0.0, 3.0, 4096, 0.97, 1.06, 256)
    sched = D.linear_cooling(1.05, 0.98, 10000, 10000, dt=0.05)
    kw = dict(table=tab, schedule=sched, seed=1, init_seed=7, graph_steps=100)
    r64 = D.Simulation(shape, storage="f64", **kw).run(10000)
    r32 = D.Simulation(shape, storage="f32c", **kw).run(10000)
    k = D.OBS_INDEX["phi2_mean"]
    rel = np.abs(r32[:, k] - r64[:, k]) / r64[:, k]
    assert rel.max() < 1e-6, rel.max()


def _expanding_schedule(n):
    """(T, ns, eta_eff, inv_a2) rows with every column varying step to step."""
    s = np.empty((n, 4))
    k = np.arange(n)
    s[:, 0] = 1.04 - 0.002 * k
    s[:, 1] = 0.3 + 0.01 * np.sin(k)
    s[:, 2] = 1.0 + 0.05 * k
    s[:, 3] = 1.0 / (1.0 + 0.03 * k) ** 2
    return s


def test_expanding_schedule_vs_oracle():
    """Per-step eta_eff and inv_a2 from a 4-column schedule (the reference's
    expanding loop, R:3621-3636), 20 graph-replayed steps against the oracle's
    rk2_step_table called with each step's scalars."""
    from oracle import oracle as O
    shape = (12, 10, 8)
    sched = _expanding_schedule(20)
    tab = D.Table1D.build(D.toy_vprime, 1.02, -0.5, 3.0, 4096)
    rng = np.random.default_rng(4)
    phi0, pi0 = rng.normal(0.6, 0.5, shape), rng.normal(0.0, 0.3, shape)
    sim = D.Simulation(shape, storage="f64", dt=0.05, dx=1.0, eta=9.0, mu=1.0, inv_a2=9.0,
                       table=tab, schedule=sched, seed=3, phi0=phi0, pi0=pi0, graph_steps=10)
    sim.run(20, observe=False)
    phi, pi = phi0.copy(), pi0.copy()
    for n in range(20):
        T, ns, eta_eff, inv_a2 = sched[n]
        O.rk2_step_table(phi, pi, 0.05, 1.0, eta_eff, 1.0, None, np.empty(shape),
                         np.empty(shape), inv_a2, tab.values, tab.tmin, tab.dinv,
                         tab.values.size, noise_scale=ns, noise_step=n, noise_seed=3)
    g_phi, g_pi = sim.fields()
    assert np.abs(g_phi.cpu().numpy() - phi).max() <= 1e-12 * np.abs(phi).max()
    assert np.abs(g_pi.cpu().numpy() - pi).max() <= 1e-12 * np.abs(pi).max()


@pytest.mark.parametrize("storage", ["f64", "f32c"])
def test_expanding_graphs_equal_eager(storage):
    tab = D.Table2D.build(D.toy_vprime, 0.0, 3.0, 4096, 0.97, 1.06, 64)
    sched = _expanding_schedule(50)
    kw = dict(storage=storage, table=tab, schedule=sched, seed=1, init_seed=3, graph_steps=20)
    a = D.Simulation((16, 12, 32), **kw)
    b = D.Simulation((16, 12, 32), **kw)
    oa = a.run(50)
    ob = b.run(50, use_graphs=False)
    assert np.array_equal(oa, ob)
    for x, y in zip(a.fields(), b.fields()):
        assert torch.equal(x, y)
