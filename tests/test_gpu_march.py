"""The TMA marching stage kernel against the generic stage kernel (bitwise: both
run the same per-site arithmetic) and against the CPU oracle."""
import math

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from oracle import oracle as O  # noqa: E402
from thermal_inflation_phase_transition_b200 import _lib as L  # noqa: E402
from thermal_inflation_phase_transition_b200 import real_field as RF  # noqa: E402
from thermal_inflation_phase_transition_b200._common import poly_source, table_source  # noqa: E402

DEV = "cuda"


@pytest.fixture(autouse=True)
def _reset_policy():
    yield
    L.set_kernel_policy(0)
    L.set_march_tiles(0, 0, 0)
    L.set_march_kseg(0)
    L.set_march_fixed(True)


def _state(shape, storage, seed):
    g = torch.Generator(device=DEV)
    g.manual_seed(seed)
    phi = 0.6 + 0.7 * torch.randn(shape, dtype=torch.float64, device=DEV, generator=g)
    pi = 0.4 * torch.randn(shape, dtype=torch.float64, device=DEV, generator=g)
    if storage == "f32c":
        return RF.to_f32c(phi), RF.to_f32c(pi)
    if storage == "f32":
        return phi.float(), pi.float()
    return phi, pi


def _run(policy, shape, storage, steps=3, tiles=(0, 0), table2d=False):
    L.set_kernel_policy(policy)
    L.set_march_tiles(*tiles)
    phi, pi = _state(shape, storage, 11)
    if table2d:
        t2, tmin, dinv, Tmin, Tdinv = O.build_table_2d(O.toy_vprime, 0.0, 3.0, 4096, 0.97, 1.06,
                                                        64)
        tab = torch.from_numpy(t2).to(DEV)
    else:
        t1, tmin, dinv = O.build_table(lambda x: O.toy_vprime(x, 1.01), 0.0, 3.0, 4096)
        tab = torch.from_numpy(t1).to(DEV)
    a = [phi, pi]
    b = [torch.empty_like(phi), torch.empty_like(pi)]
    for n in range(steps):
        T = 1.04 - 0.001 * n
        vs = table_source(tab, tmin, dinv, 4096, T, Tmin, Tdinv) if table2d else \
            table_source(tab, tmin, dinv, 4096)
        RF.rk2_step_table_into(a[0], a[1], b[0], b[1], 0.05, 1.0, 0.9, 1.0, 1.0, vs,
                               noise_scale=math.sqrt(2 * T * 0.05), noise_step=n, seed=7)
        a, b = b, a
    torch.cuda.synchronize()
    return a


SHAPES = [(16, 8, 64), (7, 8, 48), (70, 8, 16), (32, 32, 32), (9, 4, 512), (24, 32, 1),
          (1, 16, 128), (128, 1, 1), (5, 12, 96),
          # shared-memory rows that are not a multiple of 128 bytes (padded pitch)
          (32, 24, 1), (8, 16, 40), (3, 8, 288)]


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("storage", ["f32c", "f64", "f32"])
def test_march_equals_generic(shape, storage):
    ref = _run(1, shape, storage)
    got = _run(2, shape, storage)
    assert torch.equal(ref[0], got[0]) and torch.equal(ref[1], got[1])
    assert L.device_status() == 0


# rows of 512 sites in 4-row tiles and of 256 sites in 8-row tiles: the automatic
# geometry takes the kernels compiled for them
FIXED_SHAPES = [(8, 16, 512), (9, 4, 512), (6, 16, 256), (40, 8, 256)]


@pytest.mark.parametrize("shape", FIXED_SHAPES)
@pytest.mark.parametrize("table2d", [False, True])
def test_fixed_geometry_equals_runtime_geometry(shape, table2d):
    L.set_march_fixed(False)
    ref = _run(2, shape, "f32c", table2d=table2d)
    L.set_march_fixed(True)
    got = _run(2, shape, "f32c", table2d=table2d)
    assert torch.equal(ref[0], got[0]) and torch.equal(ref[1], got[1])
    assert L.device_status() == 0


@pytest.mark.parametrize("shape", FIXED_SHAPES[:3])
def test_fixed_geometry_range_variant(shape):
    """The range-folding form of the fixed-geometry kernels: the same field as the
    run-time-geometry kernel and the same range words."""
    t1, tmin, dinv = O.build_table(lambda x: O.toy_vprime(x, 1.01), 0.0, 3.0, 4096)
    vs = table_source(torch.from_numpy(t1).to(DEV), tmin, dinv, 4096)
    out = []
    for fixed in (False, True):
        L.set_march_fixed(fixed)
        L.set_kernel_policy(2)
        phi, pi = _state(shape, "f32c", 21)
        po, qo = torch.empty_like(phi), torch.empty_like(pi)
        rng = RF.PhiRange()
        RF.rk2_step_table_into(phi, pi, po, qo, 0.05, 1.0, 0.9, 1.0, 1.0, vs, noise_scale=0.3,
                               noise_step=4, seed=2, phi_range=rng)
        torch.cuda.synchronize()
        out.append((po, qo, rng.last.clone()))
    assert all(torch.equal(a, b) for a, b in zip(out[0], out[1]))
    assert L.device_status() == 0


@pytest.mark.parametrize("tiles", [(2, 1), (2, 3), (4, 5, 3), (8, 64), (16, 7, 5), (16, 40, 4)])
def test_march_tilings_agree(tiles):
    shape = (37, 16, 64)
    ref = _run(1, shape, "f32c", steps=2)
    got = _run(2, shape, "f32c", steps=2, tiles=tiles)
    assert torch.equal(ref[0], got[0]) and torch.equal(ref[1], got[1])


@pytest.mark.parametrize("shape", [(20, 12, 96), (8, 16, 512), (6, 16, 256)])
def test_march_2d_table(shape):
    """The generic kernel (the FP32 row staged as values) against the marching
    kernel (the specialised forms stage (value, slope) pairs; 512- and 256-site
    rows take the fixed-geometry kernels)."""
    ref = _run(1, shape, "f32c", table2d=True)
    got = _run(2, shape, "f32c", table2d=True)
    assert torch.equal(ref[0], got[0]) and torch.equal(ref[1], got[1])


def test_march_f64_vs_oracle():
    shape = (18, 8, 32)
    rng = np.random.default_rng(4)
    phi0, pi0 = rng.normal(0.6, 0.7, shape), rng.normal(0, 0.4, shape)
    tab, tmin, dinv = O.build_table(lambda x: O.toy_vprime(x, 1.0), 0.0, 3.0, 4096)
    a, b = phi0.copy(), pi0.copy()
    for n in range(4):
        O.rk2_step_table(a, b, 0.05, 1.0, 1.0, 1.0, None, np.empty(shape), np.empty(shape), 1.0,
                         tab, tmin, dinv, 4096, noise_scale=0.31, noise_step=n, noise_seed=2)
    L.set_kernel_policy(2)
    phi, pi = torch.from_numpy(phi0).to(DEV), torch.from_numpy(pi0).to(DEV)
    pt, vt = torch.empty_like(phi), torch.empty_like(pi)
    for n in range(4):
        RF.rk2_step_table(phi, pi, 0.05, 1.0, 1.0, 1.0, None, pt, vt, 1.0,
                          torch.from_numpy(tab).to(DEV), tmin, dinv, 4096, noise_scale=0.31,
                          noise_step=n, seed=2)
    torch.cuda.synchronize()
    np.testing.assert_allclose(phi.cpu().numpy(), a, atol=1e-13)
    np.testing.assert_allclose(pi.cpu().numpy(), b, atol=1e-13)


def test_fp32_box_muller_accuracy():
    """F32C kicks: FP32 Box-Muller of the exact hash bits vs the FP64 z."""
    shape = (64, 64, 64)
    zero = torch.zeros((2,) + shape, dtype=torch.float32, device=DEV)
    phi, pi = zero.clone(), zero.clone()
    po, vo = torch.empty_like(phi), torch.empty_like(pi)
    # V' = 0, dt = 0: pi' = kick = ns * z exactly
    RF.rk2_step_table_into(phi, pi, po, vo, 0.0, 1.0, 0.0, 1.0, 1.0, poly_source(0, 0, 0),
                           noise_scale=1.0, noise_step=17, seed=3)
    torch.cuda.synchronize()
    z32 = RF.from_f32c(vo).cpu().numpy()
    z64 = O.noise_field(shape, 17, O.K_PASS2, 3, 1.0, 0)
    err = np.abs(z32 - z64)
    assert err.max() < 2e-6 * max(1.0, np.abs(z64).max())
    rel = err / np.maximum(np.abs(z64), 1e-3)
    assert np.median(rel) < 3e-7


# ------------------------------------------------------------ complex field --
from thermal_inflation_phase_transition_b200 import complex_field as CF  # noqa: E402


def _cstate(shape, seed):
    g = torch.Generator(device=DEV)
    g.manual_seed(seed)
    f = [0.5 + 0.6 * torch.randn(shape, dtype=torch.float64, device=DEV, generator=g)
         for _ in range(2)]
    f += [0.3 * torch.randn(shape, dtype=torch.float64, device=DEV, generator=g) for _ in range(2)]
    return [RF.to_f32c(a) for a in f]


def _crun(policy, shape, steps=3, tiles=(0, 0, 0), poly=False, eps4=1e-3, kseg=0):
    L.set_kernel_policy(policy)
    L.set_march_tiles(*tiles)
    L.set_march_kseg(kseg)
    a = _cstate(shape, 5)
    b = [torch.empty_like(x) for x in a]
    if poly:
        vs = poly_source(-0.02, -0.15, 0.1)
    else:
        t1, tmin, dinv = O.build_table(lambda x: O.toy_vprime(x, 1.01), 0.0, 4.0, 4096)
        tab = torch.from_numpy(t1).to(DEV)
        vs = table_source(tab, tmin, dinv, 4096)
    for n in range(steps):
        CF.rk2_step_table_into(a, b, 0.05, 1.0, 0.9, 1.0, 1.0, vs, eps4=eps4, noise_scale=0.3,
                               noise_step=n, seed=2)
        a, b = b, a
    torch.cuda.synchronize()
    return a


@pytest.mark.parametrize("shape", [(16, 16, 64), (8, 12, 128), (5, 16, 16), (3, 8, 256),
                                   (20, 4, 96)])
def test_complex_march_equals_generic(shape):
    a = _crun(1, shape)
    b = _crun(2, shape)
    for x, y in zip(a, b):
        assert torch.equal(x, y)


@pytest.mark.parametrize("tiles", [(1, 2, 3), (2, 3, 4), (4, 64, 5), (2, 1, 3)])
def test_complex_march_tilings_agree(tiles):
    shape = (9, 16, 64)
    ref = _crun(1, shape, poly=True, eps4=0.0)
    got = _crun(2, shape, tiles=tiles, poly=True, eps4=0.0)
    for x, y in zip(ref, got):
        assert torch.equal(x, y)


@pytest.mark.parametrize("shape,kseg", [((3, 8, 256), 0), ((4, 8, 512), 256), ((5, 4, 512), 256)])
def test_complex_fixed_geometry_equals_runtime_geometry(shape, kseg):
    """256-site segments in 4-row tiles (unsplit rows of 256, split rows of 512): the
    kernel compiled for that geometry against the run-time-geometry kernel."""
    L.set_march_fixed(False)
    ref = _crun(2, shape, kseg=kseg)
    L.set_march_fixed(True)
    got = _crun(2, shape, kseg=kseg)
    for x, y in zip(ref, got):
        assert torch.equal(x, y)
    assert L.device_status() == 0


def test_complex_march_refuses_zn_when_forced():
    L.set_kernel_policy(2)
    a = _cstate((8, 8, 32), 1)
    b = [torch.empty_like(x) for x in a]
    vs = poly_source(-0.02, -0.15, 0.1)
    with pytest.raises(L.TiptError):
        CF.rk2_step_table_into(a, b, 0.05, 1.0, 0.9, 1.0, 1.0, vs, zn=(4.0, 0.01, 1.0))


def test_complex_march_vs_oracle():
    """Marching F32C complex steps against the FP64 CPU oracle (eps Re Phi^4 on)."""
    shape = (12, 16, 64)
    rng = np.random.default_rng(21)
    f = [rng.normal(0.5, 0.6, shape) for _ in range(2)] + [rng.normal(0, 0.3, shape) for _ in range(2)]
    tab, tmin, dinv = O.build_table(lambda x: O.toy_vprime(x, 1.0), 0.0, 4.0, 4096)
    ref = [a.copy() for a in f]
    for n in range(4):
        O.rk2_step_table_complex(*ref, 0.05, 1.0, 1.0, 1.0, None, None,
                                 *[np.empty(shape) for _ in range(4)], 1.0, tab, tmin, dinv, 4096,
                                 eps4=1e-3, noise_scale=0.3, noise_step=n, noise_seed=2)
    L.set_kernel_policy(2)
    st = [RF.to_f32c(torch.from_numpy(a).to(DEV)) for a in f]
    tmp = [torch.empty_like(a) for a in st]
    for n in range(4):
        CF.rk2_step_table(*st, 0.05, 1.0, 1.0, 1.0, None, None, *tmp, 1.0,
                          torch.from_numpy(tab).to(DEV), tmin, dinv, 4096, eps4=1e-3,
                          noise_scale=0.3, noise_step=n, seed=2)
    torch.cuda.synchronize()
    for a, r in zip(st, ref):
        got = RF.from_f32c(a).cpu().numpy()
        assert np.abs(got - r).max() <= 5e-6 * np.abs(r).max()


@pytest.mark.parametrize("shape,kseg,tiles", [((4, 8, 512), 0, (0, 0, 0)),
                                              ((4, 8, 512), 128, (2, 2, 4)),
                                              ((5, 16, 256), 128, (4, 3, 3)),
                                              ((3, 6, 256), 128, (2, 1, 5)),
                                              ((6, 8, 384), 128, (0, 0, 0))])
def test_complex_march_row_segments_equal_generic(shape, kseg, tiles):
    """Rows split into segments whose end neighbours come from the halo boxes."""
    a = _crun(1, shape)
    b = _crun(2, shape, tiles=tiles, kseg=kseg)
    for x, y in zip(a, b):
        assert torch.equal(x, y)


def test_bounded_wait_expires_and_reports():
    """A plane that never arrives: block 0's producer withholds ring position 1, the
    first plane its consumers compute (no copy is issued for it or after it, so none
    is left in flight; every block's work needs at least positions 0-2).  Its consumers'
    bounded waits run out, the launch returns, the device status reads
    TIPT_ERR_TIMEOUT (6), and the context stays usable: the next steps on it equal
    the generic kernel's bit for bit and leave the status clear."""
    assert L.device_status(clear=True) == 0
    shape = (32, 32, 64)
    L.set_kernel_policy(2)
    phi, pi = _state(shape, "f32c", 11)
    t1, tmin, dinv = O.build_table(lambda x: O.toy_vprime(x, 1.01), 0.0, 3.0, 4096)
    vs = table_source(torch.from_numpy(t1).to(DEV), tmin, dinv, 4096)
    po, qo = torch.empty_like(phi), torch.empty_like(pi)
    L.test_withhold_plane(1)
    RF.rk2_step_table_into(phi, pi, po, qo, 0.05, 1.0, 0.9, 1.0, 1.0, vs, noise_scale=0.3,
                           noise_step=0, seed=7)
    torch.cuda.synchronize()
    assert L.device_status(clear=True) == 6  # TIPT_ERR_TIMEOUT
    # armed for one launch only: the next launches run normally
    ref = _run(1, shape, "f32c")
    got = _run(2, shape, "f32c")
    assert torch.equal(ref[0], got[0]) and torch.equal(ref[1], got[1])
    assert L.device_status() == 0
