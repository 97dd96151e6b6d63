"""The allocation-free half-step pair (tipt_rk2_fused_table_noalloc).

Callers that cannot allocate device memory -- code running inside another
library's CUDA-graph capture, hosts without a device allocator, real-time loops
-- get this entry point, which keeps the intermediate state in a device array
inside the library instead of caller scratch.  Checked here through the C ABI
against tipt_rk2_fused_table with caller scratch, on two calls in a row.
"""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from oracle import oracle as O  # noqa: E402
from thermal_inflation_phase_transition_b200 import _lib as L  # noqa: E402
from thermal_inflation_phase_transition_b200 import real_field as RF  # noqa: E402
from thermal_inflation_phase_transition_b200._common import (ptr, step_params,  # noqa: E402
                                                             stream_handle, table_source)

DEV = "cuda"


def _state(shape, storage, seed):
    rng = np.random.default_rng(seed)
    phi = torch.from_numpy(rng.normal(0.6, 0.6, shape)).to(DEV)
    pi = torch.from_numpy(rng.normal(0.0, 0.3, shape)).to(DEV)
    if storage == L.TIPT_F32C:
        return RF.to_f32c(phi), RF.to_f32c(pi)
    return phi, pi


@pytest.mark.parametrize("storage", [L.TIPT_F64, L.TIPT_F32C])
@pytest.mark.parametrize("shape", [(24, 20, 16), (40, 36, 1)])
def test_noalloc_matches_scratch_entry(storage, shape):
    lib = L.lib()
    ta, tmin, dinv = O.build_table(lambda x: O.toy_vprime(x, 1.03), 0.0, 3.0, 4096)
    tb, _, _ = O.build_table(lambda x: O.toy_vprime(x, 1.029), 0.0, 3.0, 4096)
    tab_a, tab_b = torch.from_numpy(ta).to(DEV), torch.from_numpy(tb).to(DEV)
    va = table_source(tab_a, tmin, dinv, 4096)
    vb = table_source(tab_b, tmin, dinv, 4096)
    nx, ny, nz = shape
    ref = list(_state(shape, storage, 1))
    got = [t.clone() for t in ref]
    mid = [torch.empty_like(ref[0]), torch.empty_like(ref[1])]
    for n in range(2):  # two calls in a row
        sp = step_params(0.05, 1.0, 0.8, 1.0, 1.0, 0.31, n, 5)
        rc = lib.tipt_rk2_fused_table(storage, ptr(ref[0]), ptr(ref[1]), ptr(ref[0]),
                                      ptr(ref[1]), ptr(mid[0]), ptr(mid[1]), nx, ny, nz, sp, va,
                                      vb, None, stream_handle())
        assert rc == 0, lib.tipt_last_error()
        rc = lib.tipt_rk2_fused_table_noalloc(storage, ptr(got[0]), ptr(got[1]), ptr(got[0]),
                                              ptr(got[1]), nx, ny, nz, sp, va, vb, None,
                                              stream_handle())
        assert rc == 0, lib.tipt_last_error()
    torch.cuda.synchronize()
    # the same kernels run on the same inputs: bitwise equal
    for a, b in zip(ref, got):
        assert torch.equal(a, b)
    assert not torch.equal(ref[0], _state(shape, storage, 1)[0])  # the state advanced


def test_noalloc_rejects_oversized_lattice():
    lib = L.lib()
    # 128^3 FP64 needs 32 MiB of intermediate state: refused before any launch
    sp = step_params(0.05, 1.0, 1.0, 1.0, 1.0, 0.0, 0, 0)
    v = L.VSource(L.VP_POLY, 0, None, 0.0, 0.0, 0, 0, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0)
    buf = torch.empty(8, dtype=torch.float64, device=DEV)
    rc = lib.tipt_rk2_fused_table_noalloc(L.TIPT_F64, ptr(buf), ptr(buf), ptr(buf), ptr(buf), 128,
                                          128, 128, sp, v, v, None, stream_handle())
    assert rc == 5  # TIPT_ERR_UNSUPPORTED
    assert b"allocation-free" in lib.tipt_last_error()
