"""x-slab decomposition host logic on CPU: plane split, halo exchange and a whole
decomposed step, with world sizes 1-3 over gloo (127.0.0.1 rendezvous).

The decomposed step uses the oracle as the per-slab stepper (array noise cut
from the lattice's noise field), so this checks the decomposition, the ghost
planes and the exchange end to end against the single-lattice oracle step; the
GPU slab kernel is checked against the single-lattice kernel in
tests/test_gpu_slab.py."""
import os
import socket
import sys

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from thermal_inflation_phase_transition_b200.slab import Slab, split_planes  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _run(world, fn, *args):
    port = _free_port()
    mp.start_processes(_worker, args=(world, port, fn, args), nprocs=world, join=True,
                       start_method="spawn")


def _worker(rank, world, port, fn, args):
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        fn(rank, world, *args)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_split_planes_cover_lattice():
    for nx in (1, 2, 7, 64, 513):
        for world in range(1, min(nx, 9) + 1):
            spans = [split_planes(nx, world, r) for r in range(world)]
            assert spans[0][0] == 0
            for (a, n), (b, _) in zip(spans, spans[1:]):
                assert a + n == b
            assert spans[-1][0] + spans[-1][1] == nx
            sizes = [n for _, n in spans]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        split_planes(3, 4, 0)


def _lattice(shape, compensated):
    rng = np.random.default_rng(5)
    a = torch.from_numpy(rng.normal(0.5, 0.4, shape))
    if not compensated:
        return a
    hi = a.float()
    lo = (a - hi.double()).float()
    return torch.stack([hi, lo])


def _exchange_case(rank, world, shape):
    for compensated in (False, True):
        g = _lattice(shape, compensated)
        sl = Slab(shape, rank=rank, world=world)
        want = sl.scatter(g)
        loc = want.clone()
        if loc.dim() == 4:
            loc[:, 0] = -7.0
            loc[:, -1] = -7.0
        else:
            loc[0] = -7.0
            loc[-1] = -7.0
        sl.exchange(loc)
        assert torch.equal(loc, want), (rank, compensated)
        assert torch.equal(sl.gather(loc), g)


@pytest.mark.parametrize("world,shape", [(1, (5, 4, 6)), (2, (8, 3, 4)), (2, (5, 3, 4)),
                                         (3, (7, 2, 4))])
def test_halo_exchange(world, shape):
    """Ghost planes after the exchange equal the periodic neighbours' planes."""
    if world == 1:
        _exchange_case(0, 1, shape)
    else:
        _run(world, _exchange_case, shape)


def _oracle_stepper(slab, phi, pi, phi_out, pi_out, dt, dx, eta, mu, inv_a2, vs, ns, step,
                    seed):
    """Per-slab step with the oracle on the local planes (ghosts included) and the
    lattice's hash noise cut to the slab; the interior planes are the result."""
    from oracle import oracle as O
    tab, tmin, dinv, npts = vs
    noise = O.noise_field(slab.shape, step, O.K_PASS2, seed, ns, 0)
    noise = np.ascontiguousarray(noise[slab.local_planes()])
    a, b = phi.numpy().copy(), pi.numpy().copy()
    O.rk2_step_table(a, b, dt, dx, eta, mu, noise, np.empty_like(a), np.empty_like(b), inv_a2,
                     tab, tmin, dinv, npts)
    phi_out.copy_(torch.from_numpy(a))
    pi_out.copy_(torch.from_numpy(b))


def _step_case(rank, world, shape, nsteps):
    from oracle import oracle as O
    rng = np.random.default_rng(9)
    phi_g, pi_g = rng.normal(0.6, 0.5, shape), rng.normal(0.0, 0.3, shape)
    tab, tmin, dinv = O.build_table(lambda x: O.toy_vprime(x, 1.0), 0.0, 3.0, 512)
    a, b = phi_g.copy(), pi_g.copy()
    for n in range(nsteps):
        noise = O.noise_field(shape, n, O.K_PASS2, 3, 0.2, 0)
        O.rk2_step_table(a, b, 0.05, 1.0, 1.0, 1.0, noise, np.empty(shape), np.empty(shape), 1.0,
                         tab, tmin, dinv, 512)
    sl = Slab(shape, rank=rank, world=world)
    phi = sl.scatter(torch.from_numpy(phi_g))
    pi = sl.scatter(torch.from_numpy(pi_g))
    po, vo = torch.empty_like(phi), torch.empty_like(pi)
    for n in range(nsteps):
        sl.step(phi, pi, po, vo, 0.05, 1.0, 1.0, 1.0, 1.0, (tab, tmin, dinv, 512), noise_scale=0.2,
                noise_step=n, seed=3, stepper=_oracle_stepper)
        phi, po = po, phi
        pi, vo = vo, pi
    assert np.array_equal(sl.gather(phi).numpy(), a)
    assert np.array_equal(sl.gather(pi).numpy(), b)


@pytest.mark.parametrize("world,shape", [(1, (6, 5, 4)), (2, (8, 5, 4)), (3, (7, 4, 6))])
def test_decomposed_step_equals_lattice_step(world, shape):
    """Exchange + per-slab steps over 3 steps reproduce the single-lattice oracle
    trajectory exactly."""
    if world == 1:
        _step_case(0, 1, shape, 3)
    else:
        _run(world, _step_case, shape, 3)


def _combine_case(rank, world):
    sl = Slab((4 * world, 2, 4), rank=rank, world=world)
    out = torch.arange(10, dtype=torch.float64) * (rank + 1)
    out[7] = -rank - 1.0   # min
    out[8] = 10.0 * rank   # max
    r = sl.combine(out)
    tot = sum(range(1, world + 1))
    want = torch.arange(10, dtype=torch.float64) * tot
    want[7] = -float(world)
    want[8] = 10.0 * (world - 1)
    assert torch.equal(r, want)


def test_observables_combine():
    """Slab observables combine as sums of means/counts, min and max."""
    _run(2, _combine_case)
