"""The bench configuration at its full size (512^3, compensated FP32, 2-D V'(phi, T)
table, hash noise seed 1, cooling schedule), checked through size-independent
properties: the marching kernel that the bench times (compiled for 512-site rows,
staged table and hash noise) equals the generic one-site-per-thread kernel bit for
bit, the range it folds encloses the field it writes, and one step matches the CPU
oracle (FP64) to the compensated-FP32 tolerance.  About 9 GB on the device."""
import math

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from oracle import oracle as O  # noqa: E402
from thermal_inflation_phase_transition_b200 import _lib as L  # noqa: E402
from thermal_inflation_phase_transition_b200 import real_field as RF  # noqa: E402
from thermal_inflation_phase_transition_b200._common import table_source  # noqa: E402

DEV = "cuda"
N = 512
DT, DX, ETA = 0.05, 1.0, 1.0


@pytest.fixture(scope="module")
def setup():
    t2, tmin, dinv, Tmin, Tdinv = O.build_table_2d(O.toy_vprime, 0.0, 3.0, 4096, 0.97, 1.06, 256)
    g = torch.Generator(device=DEV)
    g.manual_seed(1234)
    phi64 = 0.3 + 0.2 * torch.randn((N, N, N), dtype=torch.float64, device=DEV, generator=g)
    pi64 = 0.1 * torch.randn((N, N, N), dtype=torch.float64, device=DEV, generator=g)
    yield dict(t2=t2, tab=torch.from_numpy(t2).to(DEV), tmin=tmin, dinv=dinv, Tmin=Tmin,
               Tdinv=Tdinv, phi64=phi64, pi64=pi64)
    L.set_kernel_policy(0)


def _steps(s, policy, steps, rng_words=None):
    L.set_kernel_policy(policy)
    a = [RF.to_f32c(s["phi64"]), RF.to_f32c(s["pi64"])]
    b = [torch.empty_like(a[0]), torch.empty_like(a[1])]
    for n in range(steps):
        T = 1.05 - 0.07 * n / 10000.0
        vs = table_source(s["tab"], s["tmin"], s["dinv"], 4096, T, s["Tmin"], s["Tdinv"])
        RF.rk2_step_table_into(a[0], a[1], b[0], b[1], DT, DX, ETA, 1.0, 1.0, vs,
                               noise_scale=math.sqrt(2 * ETA * T * DT), noise_step=n, seed=1,
                               phi_range=rng_words)
        a, b = b, a
    torch.cuda.synchronize()
    L.set_kernel_policy(0)
    return a


def test_fullsize_marching_equals_generic(setup):
    ref = _steps(setup, 1, 2)
    got = _steps(setup, 2, 2)
    assert torch.equal(ref[0], got[0]) and torch.equal(ref[1], got[1])
    assert L.device_status() == 0


def test_fullsize_range_encloses_field(setup):
    rng = RF.PhiRange()
    phi, _ = _steps(setup, 2, 2, rng_words=rng)
    lo, hi, bad = RF.PhiRange.decode(rng.last.cpu().numpy())
    v = phi[0].double() + phi[1].double()
    vmin, vmax = float(v.min()), float(v.max())
    assert not bad
    assert lo <= vmin and hi >= vmax
    # outward rounding to FP32 moves a bound by at most one FP32 ulp
    assert vmin - lo <= 2.0 ** -22 * max(1.0, abs(vmin))
    assert hi - vmax <= 2.0 ** -22 * max(1.0, abs(vmax))


def test_fullsize_step_vs_oracle(setup):
    """One step of the bench configuration against the FP64 CPU oracle (all of the
    512^3 lattice; the oracle runs on the host's cores)."""
    T = 1.05
    phi0 = setup["phi64"].cpu().numpy()
    pi0 = setup["pi64"].cpu().numpy()
    row = O.table_blend_row(setup["t2"], setup["Tmin"], setup["Tdinv"], T)
    a, b = phi0.copy(), pi0.copy()
    O.rk2_step_table(a, b, DT, DX, ETA, 1.0, None, np.empty_like(a), np.empty_like(b), 1.0, row,
                     setup["tmin"], setup["dinv"], 4096, noise_scale=math.sqrt(2 * ETA * T * DT),
                     noise_step=0, noise_seed=1)
    got_phi, got_pi = _steps(setup, 2, 1)
    gp = (got_phi[0].double() + got_phi[1].double()).cpu().numpy()
    gq = (got_pi[0].double() + got_pi[1].double()).cpu().numpy()
    assert np.abs(gp - a).max() <= 2e-6 * np.abs(a).max()
    assert np.abs(gq - b).max() <= 2e-6 * max(np.abs(b).max(), 1.0)


def test_fullsize_complex_marching_equals_generic(setup):
    """The complex-field configuration at full size (512^3, V'(|Phi|) table + eps Re Phi^4,
    hash noise): the marching kernel the complex bench times (256-site segments in
    4-row tiles, compiled for that geometry) equals the generic kernel bit for bit."""
    from thermal_inflation_phase_transition_b200 import complex_field as CF
    t1, tmin, dinv = O.build_table(lambda x: O.toy_vprime_rho(x, 0.98), 0.0, 3.0, 4096)
    vs = table_source(torch.from_numpy(t1).to(DEV), tmin, dinv, 4096)
    g = torch.Generator(device=DEV)
    g.manual_seed(77)
    init = [RF.to_f32c(0.4 * torch.randn((N, N, N), dtype=torch.float64, device=DEV, generator=g))
            for _ in range(4)]
    res = []
    for policy in (1, 2):
        L.set_kernel_policy(policy)
        if policy == 2:  # the complex bench's tiles: 4 rows, 128 planes, 4 stages, 256-site segments
            L.set_march_tiles(4, 128, 4)
            L.set_march_kseg(256)
        a = [x.clone() for x in init]
        b = [torch.empty_like(x) for x in init]
        CF.rk2_step_table_into(a, b, DT, DX, ETA, 1.0, 1.0, vs, eps4=1e-3,
                               noise_scale=math.sqrt(2 * ETA * 0.98 * DT), noise_step=3, seed=2)
        torch.cuda.synchronize()
        res.append(b)
        del a
    L.set_kernel_policy(0)
    L.set_march_tiles(0, 0, 0)
    L.set_march_kseg(0)
    for x, y in zip(*res):
        assert torch.equal(x, y)
    assert L.device_status() == 0
