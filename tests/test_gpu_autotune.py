"""Autotuner of the marching kernel's tile shape: every candidate it times runs,
the JSON cache persists the winner, and a tuned shape changes no result bit."""
import json

import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from thermal_inflation_phase_transition_b200 import _lib as L  # noqa: E402
from thermal_inflation_phase_transition_b200 import autotune as AT  # noqa: E402
from thermal_inflation_phase_transition_b200 import real_field as RF  # noqa: E402
from thermal_inflation_phase_transition_b200._common import table_source  # noqa: E402


def _run(shape, steps=6):
    torch.manual_seed(3)
    phi = RF.to_f32c(0.01 * torch.randn(shape, dtype=torch.float64, device="cuda"))
    pi = torch.zeros_like(phi)
    po, qo = torch.empty_like(phi), torch.empty_like(pi)
    tab = torch.linspace(-0.1, 0.1, 4096, dtype=torch.float64, device="cuda")
    vs = table_source(tab, 0.0, 4095 / 3.0, 4096)
    for n in range(steps):
        RF.rk2_step_table_into(phi, pi, po, qo, 0.05, 1.0, 1.0, 1.0, 1.0, vs, noise_scale=0.3,
                               noise_step=n, seed=1)
        phi, po = po, phi
        pi, qo = qo, pi
    torch.cuda.synchronize()
    return phi.clone(), pi.clone()


def test_tune_persists_and_apply_is_bitwise_neutral(tmp_path, monkeypatch):
    monkeypatch.setenv("TIPT_AUTOTUNE_CACHE", str(tmp_path / "tune.json"))
    shape = (64, 64, 64)
    ref = _run(shape)
    res = AT.tune(shape, "f32c", steps=3, warmup=1)
    assert res["tried"] >= 3 and res["ms"] > 0 and len(res["best"]) == 3
    cache = json.load(open(tmp_path / "tune.json"))
    key = AT.cache_key(shape, "f32c", 4096)
    assert cache[key]["best"] == res["best"]
    installed = AT.apply(shape, "f32c")
    try:
        got = _run(shape)
    finally:
        L.set_march_tiles(0, 0, 0)
    assert installed is None or list(installed) == res["best"]
    assert torch.equal(got[0], ref[0]) and torch.equal(got[1], ref[1])


def test_candidates_cover_default_shapes():
    c = AT.candidates((512, 512, 512))
    assert {tj for tj, _, _ in c} == {1, 2, 4}
    assert all(st in (3, 4, 5) for _, _, st in c)
    assert AT.candidates((128, 128, 1))  # 2-D lattices march along x


def test_tune_complex_field(tmp_path, monkeypatch):
    """The complex-field marching kernel is tuned under its own cache key."""
    monkeypatch.setenv("TIPT_AUTOTUNE_CACHE", str(tmp_path / "tune.json"))
    shape = (8, 16, 64)
    res = AT.tune(shape, "f32c", steps=2, warmup=1, field="complex")
    assert res["tried"] >= 3
    cache = json.load(open(tmp_path / "tune.json"))
    assert AT.cache_key(shape, "f32c", 4096, field="complex") in cache
    assert AT.cache_key(shape, "f32c", 4096) not in cache
    cands = AT.candidates(shape, "complex")
    assert all(len(c) == 4 and 64 % c[3] == 0 for c in cands)
    assert {c[3] for c in AT.candidates((8, 16, 512), "complex")} == {128, 256, 512}
