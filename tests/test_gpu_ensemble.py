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


# ---------------------------------------------------------------- vs the oracle
# The batched replicas (and the single lattice with the same polynomial V') against
# the CPU oracle's midpoint step with V'(x) = c1 x + c2 x^2 + c3 x^3 (R:1875-1966
# with the polynomial source), replica by replica: own extents, seed, T and E.
from oracle import oracle as O  # noqa: E402

# one replica of each size class of the 1792-replica mix, scaled down
# (128^2 -> 32^2 2-D, 64^3 -> 16^3, 96^3 -> 24^3), plus an odd extent
MIX = [EN.ReplicaSpec((32, 32, 1), 0.985, 0.052, 31), EN.ReplicaSpec((16, 16, 16), 1.004, 0.041, 32),
       EN.ReplicaSpec((24, 24, 24), 0.992, 0.058, 33), EN.ReplicaSpec((32, 32, 1), 1.009, 0.047, 34),
       EN.ReplicaSpec((10, 6, 14), 0.981, 0.06, 35)]
TOL = {"f64": 1e-12, "f32c": 2e-6}


def _oracle_replica(sp, phi0, nsteps, dt=0.05):
    c1, c2, c3 = EN.toy_coefficients(sp.T, sp.E, sp.D, sp.lam, sp.T0)
    ns = (2.0 * 1.0 * sp.T * dt / 1.0) ** 0.5
    phi = phi0.reshape(sp.shape).copy()
    pi = np.zeros_like(phi)
    for n in range(nsteps):
        O.rk2_step_poly(phi, pi, dt, 1.0, 1.0, 1.0, 1.0, c1, c2, c3, noise_scale=ns,
                        noise_step=n, noise_seed=sp.seed)
    return phi, pi


@pytest.mark.parametrize("storage", ["f64", "f32c"])
def test_ensemble_vs_oracle(storage):
    K = 8
    ens = EN.Ensemble(MIX, storage=storage, stop_frac=2.0, check_every=K, init_seed=3)
    phi0 = [EN.replica_initial_phi(int(np.prod(sp.shape)), sp.seed, 3, 0.01, "cuda")
            .cpu().numpy() for sp in MIX]
    ens.run(K)
    for r, sp in enumerate(MIX):
        ref_phi, ref_pi = _oracle_replica(sp, phi0[r], K)
        a, b = ens.replica_state(r)
        shape = EN._canonical(sp.shape)
        a = a.cpu().numpy().reshape(sp.shape)
        b = b.cpu().numpy().reshape(sp.shape)
        scale = max(np.abs(ref_phi).max(), np.abs(ref_pi).max())
        err = max(np.abs(a - ref_phi).max(), np.abs(b - ref_pi).max()) / scale
        assert err < TOL[storage], (r, shape, err)


@pytest.mark.parametrize("storage", ["f64", "f32c"])
def test_single_lattice_poly_vs_oracle(storage):
    """Simulation(vpoly=...) -- the per-replica plain path -- against the oracle."""
    sp = EN.ReplicaSpec((16, 12, 8), 0.99, 0.05, 41)
    rng = np.random.default_rng(2)
    phi0 = rng.normal(0.6, 0.5, sp.shape)
    sim = Simulation(sp.shape, storage=storage, table=None,
                     vpoly=EN.toy_coefficients(sp.T, sp.E), schedule=constant_temperature(sp.T, 1, dt=0.05),
                     seed=sp.seed, phi0=phi0, graph_steps=6)
    sim.run(6, observe=False)
    a, b = (t.cpu().numpy() for t in sim.fields())
    ref_phi, ref_pi = _oracle_replica(sp, phi0, 6)
    scale = max(np.abs(ref_phi).max(), np.abs(ref_pi).max())
    err = max(np.abs(a - ref_phi).max(), np.abs(b - ref_pi).max()) / scale
    assert err < TOL[storage], err


def test_marching_fixed_geometry_classes_equal_chunk_kernel():
    """The configuration's 3-D classes (64-site rows in 32-row tiles, 96-site rows in
    16-row tiles) run kernels compiled for their geometry: bitwise the chunk
    kernel's result."""
    specs = ([EN.ReplicaSpec((8, 64, 64), 0.99 + 0.004 * r, 0.05, 90 + r) for r in range(2)]
             + [EN.ReplicaSpec((6, 96, 96), 1.0, 0.045, 95 + r) for r in range(2)])
    kw = dict(storage="f32c", stop_frac=0.5, retire_frac=0.5, check_every=5, init_seed=6)
    a = EN.Ensemble(specs, use_march=True, **kw)
    b = EN.Ensemble(specs, use_march=False, **kw)
    assert len(a._march) == 2
    fa = a.run(20, poll_every=1)
    fb = b.run(20, poll_every=1)
    assert np.array_equal(fa, fb)
    for r in range(len(specs)):
        x, y = a.replica_state(r), b.replica_state(r)
        assert torch.equal(x[0], y[0]) and torch.equal(x[1], y[1]), r
    from thermal_inflation_phase_transition_b200 import _lib as L
    assert L.device_status() == 0


@pytest.mark.parametrize("storage", ["f32c"])
def test_marching_classes_equal_chunk_kernel(storage):
    """Replicas of the 3-D shape classes step on the marching stage (shared-memory
    tiles), one launch per class; bitwise the chunk work-list kernel's result,
    retired replicas included (their items are skipped by both warp roles)."""
    specs = ([EN.ReplicaSpec((16, 16, 16), 0.99 + 0.003 * r, 0.05, 60 + r) for r in range(5)]
             + [EN.ReplicaSpec((24, 12, 32), 1.0, 0.045, 70 + r) for r in range(3)]
             + [EN.ReplicaSpec((32, 32, 1), 0.985, 0.05, 80), EN.ReplicaSpec((10, 6, 14), 0.98, 0.06, 81)])
    kw = dict(storage=storage, stop_frac=0.02, retire_frac=0.02, check_every=6, init_seed=4)
    a = EN.Ensemble(specs, use_march=True, **kw)
    b = EN.Ensemble(specs, use_march=False, **kw)
    assert len(a._march) == 2 and len(b._march) == 0
    fa = a.run(60, poll_every=1)
    fb = b.run(60, poll_every=1)
    assert np.array_equal(fa, fb)
    for r in range(len(specs)):
        x, y = a.replica_state(r), b.replica_state(r)
        assert torch.equal(x[0], y[0]) and torch.equal(x[1], y[1]), r
    from thermal_inflation_phase_transition_b200 import _lib as L
    assert L.device_status() == 0
