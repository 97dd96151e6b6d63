"""Batched ensemble engine: a replica stepped inside the batch equals the same
replica stepped alone through the single-lattice driver, bit for bit."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from thermal_inflation_phase_transition_b200 import ensemble as EN  # noqa: E402
from thermal_inflation_phase_transition_b200.driver import (Simulation,  # noqa: E402
                                                            constant_temperature)

SPECS = [EN.ReplicaSpec((16, 16, 1), 1.00, 0.05, 11), EN.ReplicaSpec((8, 8, 8), 0.99, 0.045, 12),
         EN.ReplicaSpec((12, 10, 8), 1.005, 0.055, 13), EN.ReplicaSpec((6, 4, 32), 0.985, 0.04, 14)]


@pytest.mark.parametrize("storage", ["f32c", "f64"])
def test_replica_in_batch_equals_alone(storage):
    ens = EN.Ensemble(SPECS, storage=storage, stop_frac=2.0, check_every=8, init_seed=5)
    ens.run(24)
    for r, sp in enumerate(SPECS):
        shape = EN._canonical(sp.shape)
        n = int(np.prod(shape))
        phi0 = EN.replica_initial_phi(n, sp.seed, 5, 0.01, "cuda").reshape(shape).cpu().numpy()
        sim = Simulation(shape, storage=storage, table=None,
                         vpoly=EN.toy_coefficients(sp.T, sp.E),
                         schedule=constant_temperature(sp.T, 1, dt=0.05), seed=sp.seed,
                         phi0=phi0, graph_steps=8)
        sim.run(24, observe=False)
        a = ens.replica_state(r)
        b = sim.fields()
        assert torch.equal(a[0], b[0]) and torch.equal(a[1], b[1]), r


def test_first_passage_batched_equals_plain():
    specs = [EN.ReplicaSpec((16, 16, 1), 0.98, 0.05, 21), EN.ReplicaSpec((8, 8, 8), 0.985, 0.045, 22),
             EN.ReplicaSpec((16, 8, 8), 0.98, 0.06, 23)]
    ens = EN.Ensemble(specs, check_every=10, init_seed=2)
    fs = ens.run(4000, poll_every=1)
    plain = EN.plain_first_passage(specs, 4000, check_every=10, init_seed=2)
    assert np.array_equal(fs, plain), (fs, plain)
    assert (fs > 0).all()
    steps, curves = ens.frac_curves()
    assert curves.shape[1] == 3 and (np.diff(steps) == 10).all()


def test_ensemble_mixed_lattice_shapes_step():
    """One check interval of a reduced mix of 2-D 128^2, 64^3 and 96^3 replicas."""
    specs = EN.mixed_lattice_specs(n128=8, n64=4, n96=2)
    ens = EN.Ensemble(specs, check_every=4)
    ens.run(4)
    for r in (0, 9, 13):
        phi, pi = ens.replica_state(r)
        assert torch.isfinite(phi).all() and torch.isfinite(pi).all()
        assert float(pi.abs().max()) > 0
