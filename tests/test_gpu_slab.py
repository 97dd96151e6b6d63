"""The slab stepper and slab observables on one GPU: W slabs of one lattice,
their ghost planes filled from the other slabs (the exchange emulated by
copies in one process), stepped with tipt_rk2_step_table_slab and compared
with the single-lattice step -- bit for bit -- and with the lattice's
observables."""
import numpy as np
import pytest
import torch

from thermal_inflation_phase_transition_b200 import _lib as L
from thermal_inflation_phase_transition_b200 import observables as OB
from thermal_inflation_phase_transition_b200 import real_field as RF
from thermal_inflation_phase_transition_b200._common import table_source
from thermal_inflation_phase_transition_b200.slab import Slab

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda")


def _state(shape, storage, seed):
    g = torch.Generator(device=DEV)
    g.manual_seed(seed)
    phi = 0.6 + 0.5 * torch.randn(shape, dtype=torch.float64, device=DEV, generator=g)
    pi = 0.3 * torch.randn(shape, dtype=torch.float64, device=DEV, generator=g)
    if storage == "f32c":
        return RF.to_f32c(phi), RF.to_f32c(pi)
    return phi, pi


def _vs():
    from oracle import oracle as O
    tab, tmin, dinv = O.build_table(lambda x: O.toy_vprime(x, 1.0), 0.0, 3.0, 1024)
    t = torch.from_numpy(tab).to(DEV)
    return table_source(t, tmin, dinv, 1024), t


def _cat(slabs, locs):
    parts = [s.interior(x) for s, x in zip(slabs, locs)]
    return torch.cat(parts, dim=1 if locs[0].dim() == 4 else 0).contiguous()


@pytest.mark.parametrize("storage", ["f32c", "f64"])
@pytest.mark.parametrize("shape,world", [((64, 16, 64), 2), ((37, 8, 32), 3), ((9, 6, 10), 2),
                                         ((12, 4, 8), 4)])
@pytest.mark.parametrize("policy", [0, 1])
def test_slab_steps_equal_lattice_steps(storage, shape, world, policy):
    vs, _t = _vs()
    phi, pi = _state(shape, storage, 3)
    L.set_kernel_policy(policy)
    try:
        a, b = phi.clone(), pi.clone()
        ao, bo = torch.empty_like(a), torch.empty_like(b)
        for n in range(3):
            RF.rk2_step_table_into(a, b, ao, bo, 0.05, 1.0, 1.0, 1.0, 1.0, vs, noise_scale=0.3,
                                   noise_step=n, seed=4)
            a, ao = ao, a
            b, bo = bo, b
        slabs = [Slab(shape, rank=r, world=world) for r in range(world)]
        cur_phi, cur_pi = phi, pi
        for n in range(3):
            lp = [s.scatter(cur_phi) for s in slabs]   # ghosts from the neighbouring slabs
            lv = [s.scatter(cur_pi) for s in slabs]
            op = [torch.full_like(x, float("nan")) for x in lp]
            ov = [torch.full_like(x, float("nan")) for x in lv]
            for s, x, y, xo, yo in zip(slabs, lp, lv, op, ov):
                s.step_local(x, y, xo, yo, 0.05, 1.0, 1.0, 1.0, 1.0, vs, noise_scale=0.3,
                             noise_step=n, seed=4)
            cur_phi, cur_pi = _cat(slabs, op), _cat(slabs, ov)
        torch.cuda.synchronize()
        assert torch.equal(cur_phi, a) and torch.equal(cur_pi, b)
        assert L.device_status() == 0
    finally:
        L.set_kernel_policy(0)


@pytest.mark.parametrize("storage", ["f32c", "f64"])
@pytest.mark.parametrize("shape,world", [((64, 16, 64), 2), ((37, 8, 32), 3), ((9, 6, 10), 2)])
def test_slab_observables_combine_to_lattice(storage, shape, world):
    phi, pi = _state(shape, storage, 5)
    kw = dict(dx=0.8, inv_a2=0.9, lam=0.1, mphi=0.2, mu=1.1, thr=0.7)
    want = OB.observables(phi, pi, **kw).cpu().numpy()
    slabs = [Slab(shape, rank=r, world=world) for r in range(world)]
    outs = [s.observables_local(s.scatter(phi), s.scatter(pi), **kw).cpu().numpy()
            for s in slabs]
    got = np.sum(outs, axis=0)
    got[7] = min(o[7] for o in outs)
    got[8] = max(o[8] for o in outs)
    np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-14)
    assert got[9] == 0


def test_slab_rejects_bad_ranges():
    phi, pi = _state((8, 4, 8), "f64", 1)
    vs, _t = _vs()
    with pytest.raises(L.TiptError):
        L.call("tipt_rk2_step_table_slab", L.TIPT_F64, phi.data_ptr(), pi.data_ptr(),
               phi.data_ptr(), pi.data_ptr(), 6, 4, 8, 3, 8,
               RF.step_params(0.05, 1, 1, 1, 1), vs, None)


@pytest.mark.parametrize("storage", ["f64", "f32c"])
def test_slab_far_planes_use_64bit_site_keys(storage):
    """A slab whose lattice-wide site indices pass 2^32 runs the kernels' 64-bit
    noise-key path: the step equals the oracle step with the noise keyed by the
    lattice-wide index, and the marching and generic kernels agree bit for bit."""
    from oracle import oracle as O
    n1, n2, nxl = 16, 32, 4
    i_lo = (1 << 32) // (n1 * n2) + 5
    nxg = i_lo + nxl + 10
    ns, step, seed = 0.3, 7, 2
    rng = np.random.default_rng(31)
    shape = (nxl + 2, n1, n2)
    phi0, pi0 = rng.normal(0.6, 0.5, shape), rng.normal(0.0, 0.3, shape)
    keys = np.array([O.noise_key(((i_lo - 1 + q) * n1 + j) * n2 + k, step, O.K_PASS2, seed)
                     for q in range(nxl + 2) for j in range(n1) for k in range(n2)],
                    dtype=np.uint64)
    noise = (ns * O.hash_pair(keys)[2]).reshape(shape)
    tab, tmin, dinv = O.build_table(lambda x: O.toy_vprime(x, 1.0), 0.0, 3.0, 1024)
    a, b = phi0.copy(), pi0.copy()
    O.rk2_step_table(a, b, 0.05, 1.0, 1.0, 1.0, noise, np.empty(shape), np.empty(shape), 1.0,
                     tab, tmin, dinv, 1024)
    vs, _t = _vs()
    outs = []
    for policy in (0, 1):
        L.set_kernel_policy(policy)
        try:
            phi = torch.from_numpy(phi0).to(DEV)
            pi = torch.from_numpy(pi0).to(DEV)
            if storage == "f32c":
                phi, pi = RF.to_f32c(phi), RF.to_f32c(pi)
            po, vo = torch.zeros_like(phi), torch.zeros_like(pi)
            sp = RF.step_params(0.05, 1.0, 1.0, 1.0, 1.0, ns, step, seed)
            L.call("tipt_rk2_step_table_slab", L.TIPT_F32C if storage == "f32c" else L.TIPT_F64,
                   phi.data_ptr(), pi.data_ptr(), po.data_ptr(), vo.data_ptr(), nxl, n1, n2,
                   i_lo, nxg, sp, vs, None)
            torch.cuda.synchronize()
        finally:
            L.set_kernel_policy(0)
        outs.append((po, vo))
    assert torch.equal(outs[0][0], outs[1][0]) and torch.equal(outs[0][1], outs[1][1])
    po, vo = outs[0]
    if storage == "f32c":
        po, vo = RF.from_f32c(po), RF.from_f32c(vo)
    got_phi, got_pi = po.cpu().numpy()[1:-1], vo.cpu().numpy()[1:-1]
    tol = 1e-12 if storage == "f64" else 2e-6
    np.testing.assert_allclose(got_phi, a[1:-1], rtol=0, atol=tol * np.abs(a).max())
    np.testing.assert_allclose(got_pi, b[1:-1], rtol=0, atol=tol * np.abs(b).max())
    assert L.device_status() == 0


@pytest.mark.parametrize("storage", ["f32c", "f64"])
@pytest.mark.parametrize("shape", [(16, 8, 64), (3, 4, 32), (2, 4, 16)])
def test_overlapped_slab_step_equals_plain(storage, shape):
    """One rank: the exchange on the side stream with the interior planes stepped
    meanwhile and the edge planes after it gives the plain step's bits, which are
    the single-lattice step's."""
    vs, _t = _vs()
    phi, pi = _state(shape, storage, 6)
    a, b = phi.clone(), pi.clone()
    ao, bo = torch.empty_like(a), torch.empty_like(b)
    for n in range(3):
        RF.rk2_step_table_into(a, b, ao, bo, 0.05, 1.0, 1.0, 1.0, 1.0, vs, noise_scale=0.3,
                               noise_step=n, seed=4)
        a, ao = ao, a
        b, bo = bo, b
    sl = Slab(shape, rank=0, world=1)
    res = []
    for overlap in (False, True):
        x, y = sl.scatter(phi), sl.scatter(pi)
        xo, yo = torch.empty_like(x), torch.empty_like(y)
        for n in range(3):
            sl.step(x, y, xo, yo, 0.05, 1.0, 1.0, 1.0, 1.0, vs, noise_scale=0.3, noise_step=n,
                    seed=4, overlap=overlap)
            x, xo = xo, x
            y, yo = yo, y
        torch.cuda.synchronize()
        res.append((sl.interior(x).contiguous(), sl.interior(y).contiguous()))
    assert torch.equal(res[0][0], res[1][0]) and torch.equal(res[0][1], res[1][1])
    assert torch.equal(res[1][0], a) and torch.equal(res[1][1], b)
    assert L.device_status() == 0
