"""B200-native lattice Langevin stepper for thermal-inflation phase transitions.

Drop-in for the numba hot path of simulation/latticeSimeRescale_numba.py
(``real_field``) and simulation/latticeSimComplex_numba.py (``complex_field``):
same kernel names and positional signatures, CUDA tensors instead of numpy
arrays, hand-written sm_100a kernels behind the C ABI of include/tipt.h.
"""
from . import _lib
from ._lib import TiptError

__all__ = ["TiptError", "real_field", "complex_field", "observables"]


def library_path() -> str:
    return _lib.LIB_PATH


def version() -> str:
    return _lib.lib().tipt_version().decode()
