"""The step kernel's fused range output (the reference loop's per-step phi.min() /
phi.max(), R:3655-3660): the range of the field written, rounded outward to FP32
(so a value one FP64 ulp outside a table bound is never folded back inside it),
bitwise the same fields as the plain step, alternating buffers, and the
non-finite flag."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from thermal_inflation_phase_transition_b200 import real_field as RF  # noqa: E402
from thermal_inflation_phase_transition_b200._common import table_source  # noqa: E402

# (shape, storage): marching kernel (F32C, nz % 4 == 0), generic kernels otherwise
CASES = [((16, 12, 32), "f32c"), ((9, 7, 5), "f32c"), ((16, 12, 32), "f64"),
         ((9, 7, 5), "f32"), ((32, 24, 1), "f64")]


def _state(shape, storage, seed):
    g = torch.Generator(device="cuda").manual_seed(seed)
    phi = 0.8 + 0.5 * torch.randn(shape, dtype=torch.float64, device="cuda", generator=g)
    pi = 0.3 * torch.randn(shape, dtype=torch.float64, device="cuda", generator=g)
    if storage == "f32c":
        return RF.to_f32c(phi), RF.to_f32c(pi)
    if storage == "f32":
        return phi.float(), pi.float()
    return phi, pi


def _exact(t):
    """The values written in FP64: hi + lo of a compensated field (exact here)."""
    if t.dim() == 4:
        return t[0].double() + t[1].double()
    return t.double()


def rd32(x):
    """Largest FP32 value <= x (x a float64 scalar)."""
    f = np.float32(x)
    return float(np.nextafter(f, np.float32(-np.inf))) if float(f) > x else float(f)


def ru32(x):
    """Smallest FP32 value >= x."""
    f = np.float32(x)
    return float(np.nextafter(f, np.float32(np.inf))) if float(f) < x else float(f)


@pytest.mark.parametrize("shape,storage", CASES)
def test_range_matches_written_field(shape, storage):
    x = torch.linspace(-1.0, 4.0, 4096, dtype=torch.float64, device="cuda")
    vs = table_source(x * x * x - x, -1.0, 4095 / 5.0, 4096)
    phi, pi = _state(shape, storage, 3)
    a = [phi.clone(), pi.clone(), torch.empty_like(phi), torch.empty_like(pi)]
    b = [phi.clone(), pi.clone(), torch.empty_like(phi), torch.empty_like(pi)]
    rng = RF.PhiRange()
    for n in range(5):
        RF.rk2_step_table_into(a[0], a[1], a[2], a[3], 0.05, 1.0, 1.0, 1.0, 1.0, vs,
                               noise_scale=0.4, noise_step=n, seed=1, phi_range=rng)
        RF.rk2_step_table_into(b[0], b[1], b[2], b[3], 0.05, 1.0, 1.0, 1.0, 1.0, vs,
                               noise_scale=0.4, noise_step=n, seed=1)
        torch.cuda.synchronize()
        assert torch.equal(a[2], b[2]) and torch.equal(a[3], b[3])
        lo, hi, bad = RF.PhiRange.decode(rng.last.cpu().numpy())
        v = _exact(a[2])
        assert lo == rd32(float(v.min())) and hi == ru32(float(v.max())) and not bad, n
        a = [a[2], a[3], a[0], a[1]]
        b = [b[2], b[3], b[0], b[1]]


def test_range_flags_non_finite():
    vs = table_source(torch.zeros(64, dtype=torch.float64, device="cuda"), 0.0, 1.0, 64)
    phi, pi = _state((16, 12, 32), "f32c", 5)
    phi[0, 3, 4, 8] = float("nan")            # planted in the input data
    rng = RF.PhiRange()
    po, qo = torch.empty_like(phi), torch.empty_like(pi)
    RF.rk2_step_table_into(phi, pi, po, qo, 0.05, 1.0, 1.0, 1.0, 1.0, vs, phi_range=rng)
    torch.cuda.synchronize()
    assert RF.PhiRange.decode(rng.last.cpu().numpy())[2]
    # the next launch starts from reset words: a finite state reports no flag
    phi2, pi2 = _state((16, 12, 32), "f32c", 6)
    RF.rk2_step_table_into(phi2, pi2, po, qo, 0.05, 1.0, 1.0, 1.0, 1.0, vs, phi_range=rng)
    RF.rk2_step_table_into(phi2, pi2, po, qo, 0.05, 1.0, 1.0, 1.0, 1.0, vs, phi_range=rng)
    torch.cuda.synchronize()
    assert not RF.PhiRange.decode(rng.last.cpu().numpy())[2]


def test_reference_signature_with_range():
    """rk2_step_table (R:1875 signature) with phi_range= keeps its in-place semantics."""
    shape = (16, 12, 32)
    x = np.linspace(0.0, 3.0, 512)
    tab = torch.from_numpy(2 * x - x ** 2).cuda()
    phi, pi = _state(shape, "f64", 9)
    rng = RF.PhiRange()
    RF.rk2_step_table(phi, pi, 0.05, 1.0, 1.0, 1.0, None, torch.empty_like(phi),
                      torch.empty_like(pi), 1.0, tab, 0.0, 511 / 3.0, 512, noise_scale=0.2,
                      noise_step=0, phi_range=rng)
    torch.cuda.synchronize()
    lo, hi, _ = RF.PhiRange.decode(rng.last.cpu().numpy())
    assert lo == rd32(float(phi.min())) and hi == ru32(float(phi.max()))


def test_range_rounds_outward_at_a_table_bound():
    """A phi one FP64 ulp above the table's upper bound t_hi (an FP32 value) reads
    as above it, and one ulp below the lower bound as below it: the rebuild test
    of the run loop (lo < t_lo or hi > t_hi) sees both, as the reference's
    full-precision phi.min()/phi.max() would (nearest rounding to FP32 would map
    both back onto the bound)."""
    shape = (16, 12, 32)
    t_lo, t_hi = 0.25, 3.0
    vs = table_source(torch.zeros(64, dtype=torch.float64, device="cuda"), 0.0, 1.0, 64)
    phi = torch.full(shape, 1.0, dtype=torch.float64, device="cuda")
    phi[1, 2, 3] = np.nextafter(t_hi, np.inf)
    phi[4, 5, 6] = np.nextafter(t_lo, -np.inf)
    pi = torch.zeros_like(phi)
    rng = RF.PhiRange()
    po, qo = torch.empty_like(phi), torch.empty_like(pi)
    # dt = 0 and no noise: the step writes phi unchanged
    RF.rk2_step_table_into(phi, pi, po, qo, 0.0, 1.0, 1.0, 1.0, 1.0, vs, phi_range=rng)
    torch.cuda.synchronize()
    assert torch.equal(po, phi)
    lo, hi, bad = RF.PhiRange.decode(rng.last.cpu().numpy())
    assert hi > t_hi and lo < t_lo and not bad
    assert hi == ru32(float(phi.max())) and lo == rd32(float(phi.min()))
    # compensated storage: hi + lo just outside the bounds
    pc = RF.to_f32c(phi)
    assert float((pc[0].double() + pc[1].double()).max()) > t_hi
    qc = torch.zeros_like(pc)
    RF.rk2_step_table_into(pc, qc, torch.empty_like(pc), torch.empty_like(qc), 0.0, 1.0, 1.0,
                           1.0, 1.0, vs, phi_range=rng)
    torch.cuda.synchronize()
    lo, hi, bad = RF.PhiRange.decode(rng.last.cpu().numpy())
    assert hi > t_hi and lo < t_lo and not bad


def test_table_source_keeps_its_table_alive():
    """A V' source built from a temporary table tensor keeps the tensor: later
    allocations of the same size (filled with NaN) do not reach the table the
    launches read."""
    shape = (32, 32, 64)
    x = torch.linspace(-1.0, 4.0, 4096, dtype=torch.float64, device="cuda")
    kept = x * x * x - x
    vs_kept = table_source(kept, -1.0, 4095 / 5.0, 4096)
    vs_temp = table_source(x * x * x - x, -1.0, 4095 / 5.0, 4096)
    junk = [torch.full((4096,), float("nan"), dtype=torch.float64, device="cuda")
            for _ in range(64)]
    phi, pi = _state(shape, "f32c", 3)
    outs = []
    for vs in (vs_kept, vs_temp):
        po = torch.full_like(phi, 12345.0)
        qo = torch.full_like(pi, 12345.0)
        RF.rk2_step_table_into(phi, pi, po, qo, 0.05, 1.0, 1.0, 1.0, 1.0, vs)
        outs.append((po, qo))
    torch.cuda.synchronize()
    assert torch.isfinite(outs[1][0]).all()
    assert torch.equal(outs[0][0], outs[1][0]) and torch.equal(outs[0][1], outs[1][1])
    del junk


# complex field: the range of |Phi| (C:4263-4288)
CPLX_CASES = [((8, 8, 256), "f32c"), ((9, 7, 5), "f32c"), ((9, 7, 5), "f64"), ((9, 7, 5), "f32")]


def _cstate(shape, storage, seed):
    g = torch.Generator(device="cuda").manual_seed(seed)
    st = [0.6 * torch.randn(shape, dtype=torch.float64, device="cuda", generator=g)
          for _ in range(4)]
    if storage == "f32c":
        return [RF.to_f32c(a) for a in st]
    if storage == "f32":
        return [a.float() for a in st]
    return st


def _rho_check(a, b, lo, hi):
    """float32 storage: the FP32 |Phi| of the reference's float32 arrays, exactly.
    FP64: the FP64 |Phi| rounded outward.  Compensated: FP32 bounds that enclose
    the exact |Phi| and lie within 4 FP32 ulp of it."""
    if a.dim() == 4:
        ae, be = a[0].double() + a[1].double(), b[0].double() + b[1].double()
        r = torch.sqrt(ae * ae + be * be)
        rmin, rmax = float(r.min()), float(r.max())
        return lo <= rmin and hi >= rmax and rmin - lo <= 4 * 2.0 ** -24 * rmin \
            and hi - rmax <= 4 * 2.0 ** -24 * rmax
    if a.dtype == torch.float32:
        r = torch.sqrt(a * a + b * b)
        return lo == float(r.min()) and hi == float(r.max())
    r = torch.sqrt(a * a + b * b)
    return lo == rd32(float(r.min())) and hi == ru32(float(r.max()))


@pytest.mark.parametrize("shape,storage", CPLX_CASES)
def test_complex_rho_range(shape, storage):
    from thermal_inflation_phase_transition_b200 import complex_field as CF
    x = torch.linspace(0.0, 4.0, 4096, dtype=torch.float64, device="cuda")
    vs = table_source(x * x * x - x, 0.0, 4095 / 4.0, 4096)
    a = _cstate(shape, storage, 2)
    b = [t.clone() for t in a]
    oa = [torch.empty_like(t) for t in a]
    ob = [torch.empty_like(t) for t in a]
    rng = RF.PhiRange()
    for n in range(3):
        CF.rk2_step_table_into(a, oa, 0.05, 1.0, 1.0, 1.0, 1.0, vs, noise_scale=0.3,
                               noise_step=n, seed=2, rho_range=rng)
        CF.rk2_step_table_into(b, ob, 0.05, 1.0, 1.0, 1.0, 1.0, vs, noise_scale=0.3,
                               noise_step=n, seed=2)
        torch.cuda.synchronize()
        assert all(torch.equal(u, v) for u, v in zip(oa, ob))
        lo, hi, bad = RF.PhiRange.decode(rng.last.cpu().numpy())
        assert _rho_check(oa[0], oa[1], lo, hi) and not bad, n
        a, oa = oa, a
        b, ob = ob, b
