"""Load the reference's own numba kernels without running its scripts.

The reference simulation scripts (``simulation/latticeSimeRescale_numba.py`` and
``simulation/latticeSimComplex_numba.py``) parse argv, import matplotlib and
cosmoTransitions and start a run at import time, so they cannot be imported.
This module parses them with ``ast``, keeps only the requested top-level
function definitions (and simple constant assignments they read), and
``exec``s those definitions, unmodified apart from ``cache=True`` being turned
off (numba cannot cache functions compiled from a string), in a namespace that
supplies the module globals they close over (``_POT_COEFFS``, ``_ZN_PARAMS``,
the dJ spline arrays).

Fixture generation only: this runs where the reference checkout is present and
is never imported by the product, the GPU tests, ``smoke()`` or ``bench.py``.
"""
from __future__ import annotations

import ast
import math
import os

import numba as nb
import numpy as np

# The reference checkout's root directory: set TIPT_REFERENCE_ROOT before running
# a fixture generator (there is no default location).
REF_ROOT = os.environ.get("TIPT_REFERENCE_ROOT", "")
if not REF_ROOT or not os.path.isdir(os.path.join(REF_ROOT, "simulation")):
    raise RuntimeError("set TIPT_REFERENCE_ROOT to the reference checkout (the directory that "
                       "holds simulation/latticeSimeRescale_numba.py)")
REAL_SCRIPT = os.path.join(REF_ROOT, "simulation", "latticeSimeRescale_numba.py")
COMPLEX_SCRIPT = os.path.join(REF_ROOT, "simulation", "latticeSimComplex_numba.py")


class _NoCache(ast.NodeTransformer):
    def visit_keyword(self, node):
        if node.arg == "cache":
            return ast.keyword(arg="cache", value=ast.Constant(False))
        return node


def _load(path: str, names: list[str], consts: list[str], globs: dict) -> dict:
    with open(path, "r") as f:
        tree = ast.parse(f.read(), filename=path)
    keep = []
    for node in tree.body:
        if isinstance(node, ast.FunctionDef) and node.name in names:
            keep.append(_NoCache().visit(node))
        elif isinstance(node, ast.Assign) and len(node.targets) == 1:
            t = node.targets[0]
            if isinstance(t, ast.Name) and t.id in consts and isinstance(node.value, ast.Constant):
                keep.append(node)
    missing = set(names) - {n.name for n in keep if isinstance(n, ast.FunctionDef)}
    if missing:
        raise RuntimeError(f"functions not found in {path}: {sorted(missing)}")
    mod = ast.Module(body=keep, type_ignores=[])
    ast.fix_missing_locations(mod)
    ns = {"np": np, "nb": nb, "math": math}
    ns.update(globs)
    exec(compile(mod, path, "exec"), ns)
    return ns


def default_spline_globals(nseg: int = 255, ymax: float = 100.0) -> dict:
    """Finite stand-in dJ spline coefficients (the real ones need cosmoTransitions).

    The kernels accept any coefficient arrays; the values only have to be the
    same on both sides of a parity comparison.
    """
    rng = np.random.default_rng(1234)
    h = ymax / nseg
    return {
        "c0_b": rng.normal(0, 1e-4, nseg), "c1_b": rng.normal(0, 1e-3, nseg),
        "c2_b": rng.normal(0, 1e-2, nseg), "c3_b": rng.normal(0, 1e-1, nseg),
        "c0_f": rng.normal(0, 1e-4, nseg), "c1_f": rng.normal(0, 1e-3, nseg),
        "c2_f": rng.normal(0, 1e-2, nseg), "c3_f": rng.normal(0, 1e-1, nseg),
        "x_min": 0.0, "h_y": h, "inv_hy": 1.0 / h,
        "xhi_clamp": h * nseg - 1e-12, "nseg": nseg,
    }


def load_real(pot_coeffs=(1.0, 1.0), splines: dict | None = None) -> dict:
    """Kernels of the real-field script (R = latticeSimeRescale_numba.py)."""
    g = {"_POT_COEFFS": np.array(pot_coeffs, dtype=np.float64)}
    g.update(splines or default_spline_globals())
    return _load(
        REAL_SCRIPT,
        ["_hash_rng_pair", "rk2_step_table", "rk2_fused_table", "rk2_fused_single_pass",
         "rk2_step_inline", "_vprime_inline", "compute_energy_densities", "laplacian_periodic",
         "baoab_step_table", "overdamped_euler_step_table", "cubic_eval_uniform",
         "Vprime_field", "rk2_step", "rk2_step_fused"],
        ["RK2_INLINE_TILE_J", "RK2_INLINE_TILE_K", "RK2_NF_TILE_J", "RK2_NF_TILE_K",
         "BAOAB_TILE_J", "BAOAB_TILE_K", "OVERDAMPED_TILE_J", "OVERDAMPED_TILE_K"],
        g,
    )


def load_complex(zn_params=(0.0, 0.0, 0.0), pot_coeffs=(2.0, -1.0), splines: dict | None = None) -> dict:
    """Kernels of the complex-field script (C = latticeSimComplex_numba.py).

    ``_ZN_PARAMS`` is frozen into the compiled kernels at first compile, so a
    different Z_N setting needs a fresh ``load_complex`` call.
    """
    g = {
        "_POT_COEFFS": np.array(pot_coeffs, dtype=np.float64),
        "_ZN_PARAMS": np.array(zn_params, dtype=np.float64),
    }
    g.update(splines or default_spline_globals())
    return _load(
        COMPLEX_SCRIPT,
        ["_hash_rng_pair", "rk2_step_table", "rk2_fused_table", "compute_winding_number",
         "rk2_fused_single_pass", "_vprime_inline", "_vprime_complex_inline",
         "baoab_step_table", "overdamped_euler_step_table", "rk2_step_inline",
         "rk2_step", "rk2_step_fused", "Vprime_field", "laplacian_periodic",
         "cubic_eval_uniform"],
        ["RK2_INLINE_TILE_J", "RK2_INLINE_TILE_K", "RK2_NF_TILE_J", "RK2_NF_TILE_K",
         "BAOAB_TILE_J", "BAOAB_TILE_K",
         "OVERDAMPED_TILE_J", "OVERDAMPED_TILE_K"],
        g,
    )
