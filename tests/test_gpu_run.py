"""The command-line run end to end on the GPU: every --integrator for a few steps,
the default integrator's trajectory against the oracle, and --resume."""
import glob
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from thermal_inflation_phase_transition_b200 import run as RUN  # noqa: E402

BASE = ["--Nx", "12", "--Ny", "10", "--Nz", "8", "--quiet"]


def _snap(path, step):
    f = os.path.join(path, "field_states", f"state_step_{step:010d}.npz")
    with np.load(f) as z:
        return {k: z[k] for k in z.files}


@pytest.mark.parametrize("integrator", RUN.INTEGRATORS)
@pytest.mark.parametrize("hubble", [False, True])
@pytest.mark.parametrize("storage", ["f32", "f32c", "f64"])
def test_every_integrator_runs(tmp_path, integrator, hubble, storage):
    argv = BASE + ["--Nt", "8", "--steps", "4", "--integrator", integrator, "--out",
                   str(tmp_path), "--storage", storage, "--diag_energy"]
    if not hubble:
        argv.append("--no_hubble")
    r = RUN.Run(RUN.build_parser().parse_args(argv))
    assert r.run() == "completed"
    files = sorted(glob.glob(os.path.join(r.state_path, "state_step_*.npz")))
    assert [os.path.basename(f) for f in files] == ["state_step_0000000000.npz",
                                                    "state_step_0000000004.npz"]
    d = _snap(r.save_path, 4)
    assert np.isfinite(d["phi"]).all() and int(d["step"]) == 4
    assert ("scale_factor" in d) == hubble
    with np.load(os.path.join(r.save_path, "simulation_metadata.npz")) as m:
        assert str(m["integrator"]) == RUN.RECORDED_NAME[integrator]


def test_default_integrator_vs_oracle(tmp_path):
    """--no_hubble, FP64, the default rk2_nonfused: six steps of rk2_step_table with
    the table the run builds (T0, initial range +- 20000 margin, 16384 points) and
    the hash noise of generate_noise_field, against the oracle step by step."""
    from oracle import oracle as O
    argv = BASE + ["--Nt", "6", "--steps", "5", "--no_hubble", "--out", str(tmp_path),
                   "--storage", "f64", "--init_seed", "3"]
    r = RUN.Run(RUN.build_parser().parse_args(argv))
    r.run()
    d = _snap(r.save_path, 5)
    phi = 0.01 * np.random.default_rng(3).standard_normal(r.shape)
    pi = np.zeros(r.shape)
    lo, hi = phi.min() - 20000.0, phi.max() + 20000.0
    tab, tmin, dinv = r.tp.table(r.T0, lo, hi, RUN.TABLE_SIZE)
    tab = tab.cpu().numpy()
    ns = np.sqrt(2.0 * r.eta * r.T0 * r.dt / (r.mu ** 2 * r.dx_phys ** 3))
    for n in range(6):
        assert phi.min() >= lo and phi.max() <= hi   # no rebuild in the run either
        noise = O.noise_field(r.shape, n, O.K_PASS2, 0, ns, 0)
        O.rk2_step_table(phi, pi, r.dt, r.dx, r.eta, r.mu, noise, np.empty(r.shape),
                         np.empty(r.shape), 1.0, tab, tmin, dinv, RUN.TABLE_SIZE)
    assert np.abs(d["phi"] - phi).max() <= 1e-12 * np.abs(phi).max()


def test_resume_continues_the_run(tmp_path):
    """A run resumed from its step-10 checkpoint (pi on every 10th save) reaches
    the same step-14 state as the uninterrupted run: to the V' table's
    interpolation accuracy (1e-6 of the field scale), since the resumed run builds
    its table over the checkpoint's range, on another grid.  Applying a step twice
    (the reference's resume) would move the state by O(1) of its scale."""
    common = BASE + ["--steps", "1", "--no_hubble", "--storage", "f64"]
    a = RUN.Run(RUN.build_parser().parse_args(common + ["--Nt", "15", "--out",
                                                        str(tmp_path / "a")]))
    a.run()
    b_args = common + ["--Nt", "15", "--out", str(tmp_path / "b")]
    b = RUN.Run(RUN.build_parser().parse_args(b_args + ["--Nt", "12"]))
    b.run()
    c = RUN.Run(RUN.build_parser().parse_args(b_args + ["--resume"]))
    assert c.save_path == b.save_path
    c.run()
    assert c.n_start == 11
    ref, got = _snap(a.save_path, 14), _snap(c.save_path, 14)
    assert np.abs(got["phi"] - ref["phi"]).max() <= 1e-6 * np.abs(ref["phi"]).max()
