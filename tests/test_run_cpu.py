"""The command-line run's host logic (no GPU): flags and defaults of the reference
script (R:21-170), the potential coefficients (R:226-241), output naming
(R:2856-2877), replay parameters from a directory name (R:196-222) and the
expanding-background scalars against driver.hubble_expansion."""
import os

import numpy as np
import pytest

from thermal_inflation_phase_transition_b200 import driver as D
from thermal_inflation_phase_transition_b200 import run as RUN


def test_reference_flags_and_defaults():
    a = RUN.build_parser().parse_args([])
    assert (a.Nx, a.Ny, a.Nz, a.Nt, a.T0, a.steps) == (256, 256, 256, 100_000_000, 7350.0,
                                                        100_000)
    assert (a.nb, a.nf, a.dx_phys, a.dt_phys) == (20, 20, 1e-3, 1e-4)
    assert a.potential_type == "V_correct" and a.integrator is None
    assert (a.replay_steps, a.replay_save_every, a.dt_factor) == (3000, 10, 1.0)
    for flag in ("--resume", "--counterterm", "--no_scale_factor", "--no_hubble",
                 "--diag_energy"):
        assert getattr(RUN.build_parser().parse_args([flag]), flag[2:]) is True
    with pytest.raises(SystemExit):
        RUN.build_parser().parse_args(["--integrator", "leapfrog"])


def test_pot_coeffs_as_executed():
    assert RUN.pot_coeffs("V_correct", 20, 20) == (20.0, 20.0)
    assert RUN.pot_coeffs("V_p", 3, 2) == (3.0, 2.0)       # the code keeps (1, 1) for V_p
    assert RUN.pot_coeffs("fermion_only", 5, 7) == (0.0, 7.0)


def test_replay_params_from_directory_name(tmp_path):
    d = tmp_path / "64x32x16_T0_7350_dx_0.001_dtphys_0.0001_interval_500_3D_nohubble_eta_7350"
    d.mkdir()
    a = RUN.build_parser().parse_args(["--replay_dir", str(d), "--start_step", "10"])
    dxp, dtp, eta, hubble = RUN._replay_params(a)
    assert (a.Nx, a.Ny, a.Nz, a.T0) == (64, 32, 16, 7350.0)
    assert (dxp, dtp, eta, hubble) == (0.001, 0.0001, 7350.0, False)


def test_output_path_naming(tmp_path):
    a = RUN.build_parser().parse_args(["--Nx", "32", "--Ny", "32", "--Nz", "16", "--steps",
                                       "500", "--out", str(tmp_path), "--counterterm",
                                       "--device", "cpu"])
    r = RUN.Run.__new__(RUN.Run)
    r.args, r.replay, r.T0, r.dx_phys, r.dt_phys = a, False, a.T0, a.dx_phys, a.dt_phys
    r.steps, r.hubble, r.eta_phys, r.gb, r.gf = a.steps, True, a.T0, 1.09, 1.05
    r.overdamped, r.name = False, "rk2_nonfused_table"
    r._paths()
    assert r.save_path == os.path.join(
        str(tmp_path), "set8", "32x32x16_T0_7350_dx_0.001_dtphys_0.0001_interval_500_3D_hubble"
        "_eta_7350_gb_1.09_gf_1.05_nb_20_nf_20_rk2_nonfused_table_CT_V_correct")
    assert r.state_path.endswith("field_states")


def test_loop_scalars_match_hubble_schedule():
    r = RUN.Run.__new__(RUN.Run)
    r.hubble, r.T0, r.a, r.mu, r.dt, r.eta = True, 7350.0, 1.0, 1000.0, 0.1, 7.35
    r.args = RUN.build_parser().parse_args([])
    sched, a_end = D.hubble_expansion(7350.0, 40, dt=0.1, eta=7.35, mu=1000.0, dx_phys=1e-3)
    for n in range(40):
        T, T_mid, eta_eff, inv_a2, inv_a3, H = r.scalars(n)
        assert (T, eta_eff, inv_a2) == tuple(sched[n, [0, 2, 3]])
        assert T_mid == 7350.0 / r.a
    assert r.a == a_end
    ns = np.sqrt(2.0 * eta_eff * T * 0.1 * inv_a3 / (1000.0 ** 2 * 1e-3 ** 3))
    assert ns == sched[39, 1]
