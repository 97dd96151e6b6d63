"""ctypes binding of libtipt.so (the C ABI declared in include/tipt.h).

There is no fallback: if the library is missing or a call fails, a Python
exception is raised.
"""
from __future__ import annotations

import ctypes as C
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libtipt.so")

TIPT_F64, TIPT_F32, TIPT_F32C = 0, 1, 2
VP_TABLE, VP_TABLE2D, VP_POLY, VP_THERMAL = 0, 1, 2, 3
K_PASS2 = 73856093
K_PASS4 = 19349669


class TiptError(RuntimeError):
    def __init__(self, status: int, where: str, detail: str):
        super().__init__(f"{where}: status {status} ({detail})")
        self.status = status


class VSource(C.Structure):
    _fields_ = [("kind", C.c_int32), ("npts", C.c_int32), ("table", C.c_void_p),
                ("tmin", C.c_double), ("dinv", C.c_double), ("nT", C.c_int32),
                ("pad_", C.c_int32), ("T_min", C.c_double), ("T_dinv", C.c_double),
                ("T", C.c_double), ("c1", C.c_double), ("c2", C.c_double), ("c3", C.c_double),
                ("thermal", C.c_void_p)]


class StepParams(C.Structure):
    _fields_ = [("dt", C.c_double), ("dx", C.c_double), ("eta_eff", C.c_double),
                ("mu", C.c_double), ("inv_a2", C.c_double), ("noise_scale", C.c_double),
                ("noise_step", C.c_uint64), ("noise_seed", C.c_uint64)]


class Thermal(C.Structure):
    _fields_ = [("lam", C.c_double), ("mphi", C.c_double), ("boson_mass_sq", C.c_double),
                ("boson_coupling", C.c_double), ("boson_gauge_coupling", C.c_double),
                ("fermion_coupling", C.c_double), ("fermion_gauge_coupling", C.c_double),
                ("coeff_b", C.c_double), ("coeff_f", C.c_double), ("x_min", C.c_double),
                ("h", C.c_double), ("nseg", C.c_int32), ("form", C.c_int32),
                ("spline", C.c_void_p)]


class Replica(C.Structure):
    _fields_ = [("n0", C.c_int32), ("n1", C.c_int32), ("n2", C.c_int32), ("m1", C.c_uint32),
                ("m2", C.c_uint32), ("pad_", C.c_int32), ("offset", C.c_int64),
                ("c1", C.c_double), ("c2", C.c_double), ("c3", C.c_double),
                ("noise_scale", C.c_double), ("seed", C.c_uint64)]


class Chunk(C.Structure):
    _fields_ = [("replica", C.c_int32), ("count", C.c_int32), ("begin", C.c_int64)]


class ComplexTerms(C.Structure):
    _fields_ = [("zn_n", C.c_double), ("zn_dv", C.c_double), ("zn_active", C.c_double),
                ("eps4", C.c_double)]


_p, _i64, _u64, _d, _i = C.c_void_p, C.c_int64, C.c_uint64, C.c_double, C.c_int

# name -> argtypes (restype int unless listed in _RESTYPE)
_SIGS = {
    "tipt_version": [],
    "tipt_status_string": [_i],
    "tipt_last_error": [],
    "tipt_hash_rng_pair": [_p, _i64, _p, _p, _p, _p],
    "tipt_generate_noise_field": [_i, _p, _i64, _i64, _i64, _d, _u64, _u64, _u64, _i, _p],
    "tipt_rk2_step_table": [_i, _p, _p, _p, _p, _i64, _i64, _i64, C.POINTER(StepParams),
                            C.POINTER(VSource), _p, _p],
    "tipt_rk2_step_table_range": [_i, _p, _p, _p, _p, _i64, _i64, _i64, C.POINTER(StepParams),
                                  C.POINTER(VSource), _p, _p, _p, _p],
    "tipt_rk2_fused_table": [_i, _p, _p, _p, _p, _p, _p, _i64, _i64, _i64,
                             C.POINTER(StepParams), C.POINTER(VSource), C.POINTER(VSource), _p,
                             _p],
    "tipt_rk2_step_table_sched": [_i, _p, _p, _p, _p, _i64, _i64, _i64, C.POINTER(StepParams),
                                  C.POINTER(VSource), _p, _i64, _p, _i64, _p],
    "tipt_rk2_step_table_sched4": [_i, _p, _p, _p, _p, _i64, _i64, _i64, C.POINTER(StepParams),
                                  C.POINTER(VSource), _p, _i64, _p, _i64, _p],
    "tipt_rk2_step_table_slab": [_i, _p, _p, _p, _p, _i64, _i64, _i64, _i64, _i64,
                                 C.POINTER(StepParams), C.POINTER(VSource), _p],
    "tipt_rk2_step_table_slab_planes": [_i, _p, _p, _p, _p, _i64, _i64, _i64, _i64, _i64, _i64,
                                        _i64, C.POINTER(StepParams), C.POINTER(VSource), _p],
    "tipt_counter_add": [_p, _i64, _p],
    "tipt_ensemble_step": [_i, _p, _p, _p, _p, _i64, _p, _p, C.c_int32, _p,
                           C.POINTER(StepParams), _p, _i64, _p],
    "tipt_ensemble_observe": [_i, _p, _i64, _p, C.c_int32, _p, _p, _d, _d, _d, _u64, _p, _i64,
                              _p, _p, _p],
    "tipt_rk2_fused_table_noalloc": [_i, _p, _p, _p, _p, _i64, _i64, _i64,
                                     C.POINTER(StepParams), C.POINTER(VSource),
                                     C.POINTER(VSource), _p, _p],
    "tipt_complex_rk2_step_table": [_i, _p, _p, _p, _p, _p, _p, _p, _p, _i64, _i64, _i64,
                                    C.POINTER(StepParams), C.POINTER(VSource),
                                    C.POINTER(ComplexTerms), _p, _p, _p],
    "tipt_complex_rk2_step_table_range": [_i, _p, _p, _p, _p, _p, _p, _p, _p, _i64, _i64, _i64,
                                    C.POINTER(StepParams), C.POINTER(VSource),
                                    C.POINTER(ComplexTerms), _p, _p, _p, _p, _p],
    "tipt_complex_rk2_fused_table": [_i, _p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _i64,
                                     _i64, _i64, C.POINTER(StepParams), C.POINTER(VSource),
                                     C.POINTER(VSource), C.POINTER(ComplexTerms), _p, _p, _p],
    "tipt_compute_winding_number": [_i, _p, _p, _i64, _i64, _i64, _p, _p, _p, _i64, _p, _p],
    "tipt_observables_workspace_size": [_i64, _i64, _i64],
    "tipt_observables": [_i, _p, _p, _i64, _i64, _i64, _d, _d, _d, _d, _d, _d, _p, _p, _i64,
                         _p],
    "tipt_observables_slab": [_i, _p, _p, _i64, _i64, _i64, _i64, _d, _d, _d, _d, _d, _d, _p,
                              _p, _i64, _p],
    "tipt_overdamped_step_table": [_i, _p, _p, _i64, _i64, _i64, C.POINTER(StepParams),
                                   C.POINTER(VSource), _p],
    "tipt_baoab_step_table": [_i, _p, _p, _p, _p, _i64, _i64, _i64, C.POINTER(StepParams),
                              C.POINTER(VSource), _p],
    "tipt_complex_overdamped_step_table": [_i, _p, _p, _p, _p, _i64, _i64, _i64,
                                           C.POINTER(StepParams), C.POINTER(VSource),
                                           C.POINTER(ComplexTerms), _p],
    "tipt_complex_baoab_step_table": [_i, _p, _p, _p, _p, _p, _p, _p, _p, _i64, _i64, _i64,
                                      C.POINTER(StepParams), C.POINTER(VSource),
                                      C.POINTER(ComplexTerms), _p],
    "tipt_thermal_dj": [_i, _p, C.c_int32, _p, _p, _d, _p, _p],
    "tipt_thermal_vprime_field": [_i, _p, _d, C.POINTER(Thermal), _p, _i64, _i64, _i64, _p],
    "tipt_thermal_vprime_table": [_d, _d, C.c_int32, _p, C.c_int32, C.POINTER(Thermal), _p, _p],
    "tipt_thermal_vprime_field_complex": [_i, _p, _p, _d, C.POINTER(Thermal),
                                          C.POINTER(ComplexTerms), _p, _p, _i64, _i64, _i64, _p],
    "tipt_laplacian_periodic": [_i, _p, _p, _i64, _i64, _i64, _d, _p],
    "tipt_cubic_eval_uniform": [_p, _i64, _d, _d, C.c_int32, _p, _p, _p, _p, _p, _p],
    "tipt_label_workspace_size": [_i64, _i64, _i64],
    "tipt_label_components": [_i, _p, _d, _i64, _i64, _i64, _i, _p, _p, _p, _i64, _p],
    "tipt_label_stats": [_i, _p, _p, _i64, _i64, _i64, C.c_int32, _p, _p, _p, _p, _p, _p],
    "tipt_mlp_param_count": [],
    "tipt_mlp_set_policy": [_i],
    "tipt_mlp_workspace_size": [_i64],
    "tipt_mlp_forward": [_p, _p, _i64, _p, _p],
    "tipt_mlp_grad": [_p, _p, _p, _i64, C.c_float, _p, _p, _p, _i64, _p],
    "tipt_mlp_adam": [_p, _p, _p, _p, _p, _i64, C.c_float, _p, _i64, C.c_float, C.c_float,
                      C.c_float, C.c_float, _p],
    "tipt_set_kernel_policy": [_i],
    "tipt_set_march_tiles": [_i, _i, _i],
    "tipt_set_march_kseg": [_i],
    "tipt_set_march_fixed": [_i],
    "tipt_device_status": [C.POINTER(C.c_int), _i],
    "tipt_test_withhold_plane": [_i],
    "tipt_ensemble_march_supported": [C.c_int32, C.c_int32, C.c_int32],
    "tipt_ensemble_step_march": [_p, _p, _p, _p, _i64, _p, _p, C.c_int32, _p, C.c_int32,
                                 C.c_int32, C.c_int32, _p, C.POINTER(StepParams), _p, _i64, _p],
    "tipt_ensemble_compact": [_p, C.c_int32, _p, _p, _p, _p],
}
_RESTYPE = {"tipt_version": C.c_char_p, "tipt_status_string": C.c_char_p,
            "tipt_last_error": C.c_char_p, "tipt_observables_workspace_size": C.c_int64,
            "tipt_mlp_param_count": C.c_int64, "tipt_mlp_workspace_size": C.c_int64,
            "tipt_label_workspace_size": C.c_int64}

_lib = None


def exported_symbols() -> list[str]:
    return list(_SIGS)


def lib():
    """Load libtipt.so (once).  Raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with "
                "`python -m thermal_inflation_phase_transition_b200.build` (there is no CPU "
                "fallback)")
        L = C.CDLL(LIB_PATH)
        for name, args in _SIGS.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = _RESTYPE.get(name, C.c_int)
        _lib = L
    return _lib


def check(status: int, where: str) -> None:
    if status != 0:
        L = lib()
        raise TiptError(status, where, f"{L.tipt_status_string(status).decode()}: "
                                       f"{L.tipt_last_error().decode()}")


def call(name: str, *args) -> None:
    check(getattr(lib(), name)(*args), name)


def set_kernel_policy(policy: int) -> None:
    """0 automatic, 1 generic stage kernel, 2 marching stage kernel (tests/tuning)."""
    call("tipt_set_kernel_policy", int(policy))


def set_march_tiles(rows: int = 0, planes: int = 0, stages: int = 0) -> None:
    """Marching-kernel tile shape (0 = automatic); performance only."""
    call("tipt_set_march_tiles", int(rows), int(planes), int(stages))


def set_march_fixed(enable: bool) -> None:
    """Compensated-FP32 marching kernels compiled for fixed geometries (real, complex,
    integrator and ensemble-class stages) on or off; performance only (tests/tuning)."""
    call("tipt_set_march_fixed", int(bool(enable)))


def set_march_kseg(kseg: int) -> None:
    """Row segment of the complex marching kernel (0 = automatic; tests/tuning)."""
    call("tipt_set_march_kseg", int(kseg))


def test_withhold_plane(position: int) -> None:
    """Test of the bounded device waits: the next compensated-FP32 marching stage
    launch withholds ring position `position` in its block 0 (< 0 disarms)."""
    call("tipt_test_withhold_plane", int(position))


def device_status(clear: bool = False) -> int:
    """Device status word of bounded device waits (0 = ok).  Synchronises."""
    v = C.c_int(0)
    call("tipt_device_status", C.byref(v), int(bool(clear)))
    return v.value
