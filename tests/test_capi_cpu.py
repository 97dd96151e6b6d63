"""C-ABI checks that need no GPU: the library loads, exports every symbol that
include/tipt.h declares, and rejects bad arguments before touching a device."""
import ctypes as C
import os
import re

import pytest

from thermal_inflation_phase_transition_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _header_symbols():
    src = open(os.path.join(ROOT, "include", "tipt.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(tipt_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_header_symbols():
    lib = L.lib()
    syms = _header_symbols()
    assert len(syms) >= 10
    for s in syms:
        assert hasattr(lib, s), f"libtipt.so does not export {s}"


def test_python_binding_covers_header():
    assert set(_header_symbols()) <= set(L.exported_symbols())


def test_status_strings():
    lib = L.lib()
    assert lib.tipt_status_string(0) == b"ok"
    assert b"argument" in lib.tipt_status_string(1)
    assert lib.tipt_version().startswith(b"tipt")


def _sp():
    return L.StepParams(0.05, 1.0, 1.0, 1.0, 1.0, 0.0, 0, 0)


def _vs():
    return L.VSource(L.VP_POLY, 0, None, 0.0, 0.0, 0, 0, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0)


def test_rejects_null_state():
    lib = L.lib()
    rc = lib.tipt_rk2_step_table(L.TIPT_F64, None, None, None, None, 4, 4, 4, _sp(), _vs(), None,
                                 None)
    assert rc == 1
    assert b"NULL" in lib.tipt_last_error()


def test_rejects_bad_storage_and_dims():
    lib = L.lib()
    buf = (C.c_double * 64)()
    p = C.cast(buf, C.c_void_p)
    assert lib.tipt_rk2_step_table(7, p, p, p, p, 4, 4, 4, _sp(), _vs(), None, None) == 2
    assert lib.tipt_rk2_step_table(L.TIPT_F64, p, p, p, p, 0, 4, 4, _sp(), _vs(), None, None) == 1


def test_rejects_aliasing_output():
    """The fused stage reads neighbours: writing over its input is refused."""
    lib = L.lib()
    a = (C.c_double * 64)()
    b = (C.c_double * 64)()
    c = (C.c_double * 64)()
    pa, pb, pc = (C.cast(x, C.c_void_p) for x in (a, b, c))
    rc = lib.tipt_rk2_step_table(L.TIPT_F64, pa, pb, pa, pc, 4, 4, 4, _sp(), _vs(), None, None)
    assert rc == 1
    assert b"overlap" in lib.tipt_last_error()


def test_rejects_misaligned():
    lib = L.lib()
    a = (C.c_double * 80)()
    base = C.cast(a, C.c_void_p).value
    mis = C.c_void_p(base + 4)
    ok = C.c_void_p(base + 8 * 70)
    rc = lib.tipt_rk2_step_table(L.TIPT_F64, mis, ok, ok, ok, 1, 1, 1, _sp(), _vs(), None, None)
    assert rc == 3


def test_rejects_bad_table():
    lib = L.lib()
    a = (C.c_double * 8)()
    bufs = [(C.c_double * 8)() for _ in range(4)]
    ps = [C.cast(x, C.c_void_p) for x in bufs]
    vs = L.VSource(L.VP_TABLE, 1, C.cast(a, C.c_void_p).value, 0.0, 1.0, 0, 0, 0.0, 0.0, 0.0,
                   0.0, 0.0, 0.0)
    rc = lib.tipt_rk2_step_table(L.TIPT_F64, *ps, 2, 2, 2, _sp(), vs, None, None)
    assert rc == 1 and b"npts" in lib.tipt_last_error()


def test_observables_workspace_size_is_positive():
    assert L.lib().tipt_observables_workspace_size(512, 512, 512) > 0
    assert L.lib().tipt_observables_workspace_size(0, 1, 1) == 0


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    monkeypatch.setattr(L, "_lib", None)
    monkeypatch.setattr(L, "LIB_PATH", str(tmp_path / "libtipt.so"))
    with pytest.raises(RuntimeError, match="no CPU"):
        L.lib()


def test_gamma_mle_censoring():
    from thermal_inflation_phase_transition_b200.ensemble import gamma_mle
    # 3 events at steps 9, 19, 99 and one censored at 100 steps, volume 8, dt 0.5
    g, rel, n = gamma_mle([9, 19, 99, -1], 100, 8.0, 0.5)
    assert n == 3
    assert abs(g - 3 / (8.0 * 0.5 * (10 + 20 + 100 + 100))) < 1e-15
    assert abs(rel - 1 / 3 ** 0.5) < 1e-15


def test_slab_entries_reject_bad_ranges():
    """The slab step and slab observables check the plane range before any launch."""
    lib = L.lib()
    buf = (C.c_double * 4096)()
    p = C.cast(buf, C.c_void_p)
    # nz = 1 (2-D lattices are one GPU's work)
    assert lib.tipt_rk2_step_table_slab(L.TIPT_F64, p, p, p, p, 4, 4, 1, 0, 8, _sp(), _vs(),
                                        None) == 1
    # planes [6, 10) outside an 8-plane lattice
    assert lib.tipt_rk2_step_table_slab(L.TIPT_F64, p, p, p, p, 4, 4, 4, 6, 8, _sp(), _vs(),
                                        None) == 1
    assert b"outside" in lib.tipt_last_error()
    # site count below the slab's
    out = (C.c_double * 10)()
    assert lib.tipt_observables_slab(L.TIPT_F64, p, None, 4, 4, 4, 10, 1.0, 1.0, 0.0, 0.0, 1.0,
                                     1.0, C.cast(out, C.c_void_p), p, 8 * 4096, None) == 1
    # workspace too small
    assert lib.tipt_observables_slab(L.TIPT_F64, p, None, 4, 4, 4, 512, 1.0, 1.0, 0.0, 0.0, 1.0,
                                     1.0, C.cast(out, C.c_void_p), p, 8, None) == 1
    assert b"workspace" in lib.tipt_last_error()
