"""The surrogate-steered scan end to end on small lattices: training rows from the
ensemble engine, training through the library's own kernels, lam* proposals,
verification by plain 256-replica ensembles, and the cost against a dense scan.
This is the test of what the trained network gains over the plain method."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from thermal_inflation_phase_transition_b200 import scan as SC  # noqa: E402


def test_steered_scan_small():
    rep = SC.steered_scan(n_train=4000, train_shapes=((32, 32, 1), (16, 16, 16), (24, 24, 24)),
                          train_mix=(0.3, 0.3, 0.4), scan_shape=(24, 24, 24), n_points=27,
                          train_steps=1600, n_verify=256, fit_iters=1500, seed=3,
                          log=lambda *a: None)
    v, c = rep["verify"], rep["cost"]
    assert rep["proposals"]["bracketed"] >= 5
    # the surrogate's rate at its proposals against the plain ensembles
    assert v["median_abs_rel_err"] < 0.10, v
    assert v["frac_within_10pct_or_2sigma"] >= 0.8, v
    assert v["median_poisson_err"] < 0.08
    # the gain: a dense plain scan of the same points costs several times more
    assert c["ratio"] > 3.0, c
    assert rep["fit"]["loss_last"] < rep["fit"]["loss_first"]
    rows = v["rows"]
    assert all(0.05 <= r["lam"] <= 0.2 for r in rows)
    assert np.isfinite([r["gamma_plain"] for r in rows]).all()
