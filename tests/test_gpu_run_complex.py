"""The complex-field command-line run end to end on the GPU."""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from thermal_inflation_phase_transition_b200 import run_complex as RC  # noqa: E402

BASE = ["--Nx", "12", "--Ny", "10", "--Nz", "8", "--quiet"]


def _snap(path, step):
    with np.load(os.path.join(path, "field_states", f"state_step_{step:010d}.npz")) as z:
        return {k: z[k] for k in z.files}


@pytest.mark.parametrize("integrator", [None] + RC.INTEGRATORS)
@pytest.mark.parametrize("storage", ["f32", "f32c", "f64"])
def test_every_integrator_runs_with_zn_turn_on(tmp_path, integrator, storage):
    """8 steps with Z_4 switched on below a T that the expanding background crosses
    at the first step (the flag reaches the kernels, unlike the reference's frozen
    global); snapshots carry rho, theta, windings, zn_active and the scale factor."""
    argv = BASE + ["--Nt", "8", "--steps", "4", "--out", str(tmp_path), "--storage", storage,
                   "--zn_order", "4", "--zn_strength", "1e9", "--zn_turn_on_T", "7349.9",
                   "--init_rho", "3000"]
    if integrator:
        argv += ["--integrator", integrator]
    r = RC.ComplexRun(RC.build_parser().parse_args(argv))
    assert r.run() == "completed"
    d0, d4 = _snap(r.save_path, 0), _snap(r.save_path, 4)
    assert float(d0["zn_active"]) == 0.0 and float(d4["zn_active"]) == 1.0
    for k in ("phi1", "phi2", "rho", "theta", "winding"):
        assert np.isfinite(d4[k]).all()
    assert ("pi1" in d0) == (r.integrator != "overdamped")
    assert float(d4["scale_factor"]) > 1.0
    with np.load(os.path.join(r.save_path, "simulation_metadata.npz")) as m:
        assert str(m["field_type"]) == "complex" and int(m["zn_order"]) == 4


def test_rk2_nonfused_vs_oracle(tmp_path):
    """Six steps of --integrator rk2_nonfused (FP64, U(1)) against the oracle's complex
    rk2_step_table with the run's table, scalars and the cos / sin hash noise pair."""
    from oracle import oracle as O
    argv = BASE + ["--Nt", "6", "--steps", "5", "--out", str(tmp_path), "--storage", "f64",
                   "--integrator", "rk2_nonfused", "--init_rho", "3000", "--init_seed", "2"]
    r = RC.ComplexRun(RC.build_parser().parse_args(argv))
    r.run()
    got = _snap(r.save_path, 5)
    rng = np.random.default_rng(2)
    th = 2.0 * np.pi * rng.random(r.shape)
    rr = 3000.0 * np.abs(rng.standard_normal(r.shape))
    s = [rr * np.cos(th), rr * np.sin(th), np.zeros(r.shape), np.zeros(r.shape)]
    q = RC.ComplexRun(RC.build_parser().parse_args(argv))
    T_last = None
    for n in range(6):
        T, T_mid, eta_eff, inv_a2, H = q.scalars(n)
        if T_last is None or abs(T - T_last) / T > 1e-4:     # the run's rebuild rule
            hi = np.sqrt(s[0] ** 2 + s[1] ** 2).max()
            tab, tmin, dinv = r.tp.table(T, 0.0, hi + max(hi, 20000.0), 16384)
            tab, T_last = tab.cpu().numpy(), T
        ns = np.sqrt(2.0 * eta_eff * T * r.dt / (r.mu ** 2 * r.dx_phys ** 3))
        n1 = O.noise_field(r.shape, n, O.K_PASS2, 0, ns, 0)
        n2 = O.noise_field(r.shape, n, O.K_PASS2, 0, ns, 1)
        O.rk2_step_table_complex(*s, r.dt, r.dx, eta_eff, r.mu, n1, n2,
                                 *[np.empty(r.shape) for _ in range(4)], inv_a2, tab, tmin, dinv,
                                 16384)
    for a, f in zip(s[:2], ("phi1", "phi2")):
        assert np.abs(got[f] - a).max() <= 1e-12 * np.abs(a).max()
