"""Host logic of the complex-field command-line run (no GPU): flags and defaults
(C:21-158), potential coefficients (C:205-221), the automatic first-order
integrator (C:654-669), output naming (C:3355-3396) and the loop scalars."""
import os

import numpy as np

from thermal_inflation_phase_transition_b200 import driver as D
from thermal_inflation_phase_transition_b200 import run_complex as RC


def test_flags_and_defaults():
    a = RC.build_parser().parse_args([])
    assert (a.Nx, a.Ny, a.Nz, a.Nt, a.T0, a.steps) == (256, 256, 256, 100_000_000, 7350.0,
                                                        100_000)
    assert a.potential_type == "V_p" and (a.zn_order, a.zn_strength, a.zn_turn_on_T) == (0, 0.0,
                                                                                          0.0)
    assert a.init_rho == 0.01 and a.integrator is None


def test_pot_coeffs_and_integrator_choice():
    assert RC.pot_coeffs("V_p") == (2.0, -1.0)
    assert RC.pot_coeffs("V_correct") == (1.0, 1.0)
    assert RC.pot_coeffs("fermion_only") == (0.0, 1.0)
    a = RC.build_parser().parse_args([])
    assert RC.integrator_of(a, 1000.0) == "overdamped"      # eta_phys 1000 > 100
    assert RC.integrator_of(a, 50.0) == "rk2_nonfused"
    b = RC.build_parser().parse_args(["--integrator", "baoab"])
    assert RC.integrator_of(b, 1000.0) == "baoab"


def test_naming_and_scalars(tmp_path):
    a = RC.build_parser().parse_args(["--Nx", "32", "--Ny", "32", "--Nz", "16", "--steps", "500",
                                      "--zn_order", "4", "--out", str(tmp_path)])
    r = RC.ComplexRun.__new__(RC.ComplexRun)
    r.args, r.replay, r.T0, r.dx_phys, r.dt_phys = a, False, 7350.0, 1e-3, 2.5e-4
    r.steps, r.eta_phys, r.gb, r.gf, r.overdamped, r.name = 500, 1000.0, 1.09, 1.09, True, \
        "overdamped"
    r._paths()
    assert r.save_path == os.path.join(
        str(tmp_path), "set6", "32x32x16_T0_7350_complex_ZN4_dx_0.001_dtphys_0.00025_interval_500"
        "_3D_hubble_eta_1000_gb_1.09_gf_1.09_OD_overdamped")
    r.a, r.mu, r.dt, r.eta = 1.0, 1000.0, 0.25, 1.0
    sched, a_end = D.hubble_expansion(7350.0, 20, dt=0.25, eta=1.0, mu=1000.0)
    for n in range(20):
        T, T_mid, eta_eff, inv_a2, H = r.scalars(n)
        assert (T, eta_eff, inv_a2) == tuple(sched[n, [0, 2, 3]])
    assert r.a == a_end
