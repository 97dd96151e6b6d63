"""Surrogate network kernels against the CPU oracle: forward, gradient (BF16
operands, FP32 accumulation), Adam, determinism, and a training run."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from oracle import mlp as M  # noqa: E402
from thermal_inflation_phase_transition_b200 import _lib as L  # noqa: E402
from thermal_inflation_phase_transition_b200 import surrogate as S  # noqa: E402

# 1: mma.sync kernels, 2: tcgen05 kernels (tensor-memory accumulators)
POLICIES = [1, 2]


@pytest.fixture
def policy(request):
    L.call("tipt_mlp_set_policy", request.param)
    yield request.param
    L.call("tipt_mlp_set_policy", 0)


def _batch(rows, seed=0):
    rng = np.random.default_rng(seed)
    x = rng.normal(size=(rows, 6)).astype(np.float32)
    t = np.zeros((rows, M.TGT_COLS), np.float32)
    t[:, 0] = rng.integers(0, 2, rows)
    t[:, 1] = rng.uniform(0.1, 2.0, rows)
    t[:, 2] = rng.uniform(0.5, 1.0, rows)
    t[:, 3] = rng.uniform(0.0, 1.0, rows)
    t[:, 4:] = rng.uniform(0.0, 1.0, (rows, 16))
    return x, t


def _params(seed):
    p = M.init_params(seed)
    rng = np.random.default_rng(seed + 100)
    lay, _ = M.layout()
    # non-trivial biases and a larger output layer than the initialiser's
    for (w, b, fi, fo) in lay:
        p[b:b + fo] = rng.normal(0, 0.2, fo)
    w3, b3, _, _ = lay[3]
    p[w3:b3] *= 5.0
    p[b3 + 17:b3 + 32] = 0.0
    return p


@pytest.mark.parametrize("policy", POLICIES, indirect=True)
@pytest.mark.parametrize("rows", [1, 128, 300])
def test_forward_matches_oracle(rows, policy):
    p = _params(1)
    x, _ = _batch(rows)
    net = S.SurrogateNet(p)
    y = net.forward(x).cpu().numpy()
    ref, _ = M.forward(p, x)
    scale = np.abs(ref).max()
    assert np.abs(y - ref).max() <= 2e-3 * scale, (np.abs(y - ref).max(), scale)


@pytest.mark.parametrize("policy", POLICIES, indirect=True)
@pytest.mark.parametrize("rows", [96, 300])
def test_gradient_matches_oracle(rows, policy):
    p = _params(2)
    x, t = _batch(rows, 5)
    net = S.SurrogateNet(p)
    lr_dev = torch.zeros(rows, dtype=torch.float32, device="cuda")
    g = net.grad(x, t, loss_rows=lr_dev).cpu().numpy().astype(np.float64)
    loss, lrow, gr = M.loss_and_grad(p, x, t)
    np.testing.assert_allclose(lr_dev.cpu().numpy(), lrow, rtol=5e-3, atol=5e-4)
    lay, _ = M.layout()
    for li, (w, b, fi, fo) in enumerate(lay):
        for sl in (slice(w, b), slice(b, b + fo)):
            err = np.linalg.norm(g[sl] - gr[sl]) / max(np.linalg.norm(gr[sl]), 1e-30)
            assert err < 1e-2, (li, sl, err)
    # padding stays untouched by the gradient
    assert g[lay[3][0] + 17] == 0.0 and not g[6 * 128:16 * 128].any()


@pytest.mark.parametrize("policy", POLICIES, indirect=True)
def test_gradient_deterministic_and_norm_argument(policy):
    p = _params(3)
    x, t = _batch(500, 7)
    net = S.SurrogateNet(p)
    a = net.grad(x, t).clone()
    b = net.grad(x, t).clone()
    assert torch.equal(a, b)
    c = net.grad(x, t, norm=1000.0).clone()
    torch.testing.assert_close(c, a * 0.5, rtol=1e-6, atol=1e-12)


def test_adam_matches_oracle():
    p = _params(4)
    x, t = _batch(200, 9)
    net = S.SurrogateNet(p)
    pp, m, v = p.astype(np.float64), np.zeros(p.size), np.zeros(p.size)
    for step in range(1, 4):
        g = net.grad(x, t).clone()
        net.adam(g, 1e-3, weight_decay=1e-4)
        # the oracle takes the GPU's gradient so the comparison isolates Adam
        pp, m, v = M.adam(pp, g.cpu().numpy(), m, v, step, 1e-3, wd=1e-4)
    np.testing.assert_allclose(net.params.cpu().numpy(), pp, rtol=1e-5, atol=1e-7)
    assert int(net.counter.item()) == 3


def test_fit_reduces_loss_on_smooth_rates():
    """Rows drawn from a known smooth log-rate and fraction curve: training through the
    graph-captured loop reaches a loss close to the generating model's."""
    rng = np.random.default_rng(11)
    n = 6000
    x = rng.uniform(-1, 1, (n, 6)).astype(np.float32)
    x[:, 5] = rng.choice([-0.5, 0.5], n)
    true_l = 0.8 * x[:, 0] - 0.5 * x[:, 1] + 0.3 * x[:, 2] * x[:, 3] - 1.0
    ex = rng.uniform(0.2, 3.0, n)
    t_ev = rng.exponential(1.0 / np.exp(true_l))
    ev = (t_ev < ex).astype(np.float32)
    tk = (np.arange(1, 17) / 16.0)[None, :]
    frac = 1.0 / (1.0 + np.exp(-(4.0 * x[:, :1] + 6.0 * (tk - 0.5))))
    tgt = np.zeros((n, M.TGT_COLS), np.float32)
    tgt[:, 0] = ev
    tgt[:, 1] = np.minimum(t_ev, ex)
    tgt[:, 2] = 1.0
    tgt[:, 3] = 1.0
    tgt[:, 4:] = frac
    # loss of the generating model itself: the floor a perfect fit reaches
    y_true = np.concatenate([true_l[:, None], np.log(frac / (1.0 - frac))], axis=1)
    floor = float(M.row_loss_and_dy(y_true, tgt, n)[0].mean())
    net = S.SurrogateNet(seed=0)
    l0 = net.loss(x, tgt)
    hist = net.fit(x, tgt, iters=600, lr=3e-3, lr_final=3e-4, batch=1024, graph_iters=50)
    l1 = net.loss(x, tgt)
    assert len(hist) == 12 and l0 - floor > 0.3
    assert l1 - floor < 0.1 * (l0 - floor), (l0, l1, floor)
    pred = net.forward(x).cpu().numpy()
    assert np.corrcoef(pred[:, 0], true_l)[0, 1] > 0.85  # one noisy event per row
    assert np.abs(1.0 / (1.0 + np.exp(-pred[:, 1:])) - frac).mean() < 0.05


def test_tcgen05_and_mma_sync_agree():
    """Both kernel paths on the same batch: equal up to FP32 accumulation order."""
    p = _params(6)
    x, t = _batch(700, 13)
    net = S.SurrogateNet(p)
    out = {}
    for pol in POLICIES:
        L.call("tipt_mlp_set_policy", pol)
        out[pol] = (net.forward(x).clone(), net.grad(x, t).clone())
    L.call("tipt_mlp_set_policy", 0)
    (y1, g1), (y2, g2) = out[1], out[2]
    assert (y1 - y2).abs().max() <= 1e-3 * y1.abs().max()
    assert float((g1 - g2).norm() / g1.norm()) < 1e-3
    assert L.device_status(clear=True) == 0
