"""Surrogate network pieces that need no GPU: the CPU oracle's analytic gradient
against finite differences, its BF16 rounding, and the parameter layout and
initialisation shared by the oracle and the library."""
import numpy as np

from oracle import mlp as M
from thermal_inflation_phase_transition_b200 import _lib as L
from thermal_inflation_phase_transition_b200 import surrogate as S


def _batch(rows, seed=0):
    rng = np.random.default_rng(seed)
    x = rng.normal(size=(rows, 6))
    t = np.zeros((rows, M.TGT_COLS))
    t[:, 0] = rng.integers(0, 2, rows)
    t[:, 1] = rng.uniform(0.1, 2.0, rows)
    t[:, 2] = rng.uniform(0.5, 1.0, rows)
    t[:, 3] = rng.uniform(0.0, 1.0, rows)
    t[:, 4:] = rng.uniform(0.0, 1.0, (rows, 16))
    return x, t


def test_layout_matches_library():
    lay, total = M.layout()
    assert total == int(L.lib().tipt_mlp_param_count()) == 39328
    assert S.layout() == (lay, total)


def test_init_params_identical_and_padding_zero():
    p = S.init_params(3)
    assert np.array_equal(p, M.init_params(3))
    (W0, _), _, _, (W3, b3) = M.unpack(p)
    assert not W0[6:].any() and not W3[:, 17:].any() and not b3[17:].any()


def test_oracle_gradient_matches_finite_differences():
    p = M.init_params(1).astype(np.float64)
    x, t = _batch(37)
    _, _, g = M.loss_and_grad(p, x, t, bf16_ops=False)
    lay, _ = M.layout()
    idx = [0, 5, lay[0][1] + 3, lay[1][0] + 100, lay[2][0] + 5000, lay[3][0] + 5 * 32 + 3,
           lay[3][1], lay[3][1] + 16, lay[2][1] + 77]
    fd = M.grad_fd(p, x, t, idx)
    np.testing.assert_allclose(g[idx], fd, rtol=2e-5, atol=1e-9)
    # padding receives exactly zero gradient
    assert g[lay[3][0] + 17] == 0.0 and g[lay[3][1] + 20] == 0.0 and not g[6 * 128:16 * 128].any()


def test_bf16_rounding_is_nearest_even():
    vals = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -9, -2.5, 3.0e38],
                    np.float32)
    r = M.bf16(vals)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2 ** -6 and r[3] == 1.0
    assert r[4] == -2.5


def test_features_centre_of_box_is_zero():
    f = S.features(0.995, 0.05, 0.1, 0.125, np.exp(12.0), 2.5)
    assert np.allclose(f, 0.0, atol=1e-6)
    f = S.features([0.97, 1.02], 0.03, 0.05, 0.05, [16384, 262144], [2, 3])
    assert f.shape == (2, 6) and np.allclose(f[:, 0], [-1, 1]) and np.allclose(f[:, 5], [-0.5, 0.5])


def test_adam_oracle_first_step_is_sign_step():
    p = np.array([1.0, -2.0, 0.5])
    g = np.array([0.3, -0.1, 0.0])
    q, m, v = M.adam(p, g, np.zeros(3), np.zeros(3), 1, lr=0.01)
    np.testing.assert_allclose(q, p - 0.01 * np.sign(g) * (g != 0), atol=1e-7)
