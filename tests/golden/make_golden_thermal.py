"""Golden fixtures of the thermal V' path (tests/golden/thermal.npz), generated
from the REFERENCE's own code:

    TIPT_REFERENCE_ROOT=<reference checkout> python tests/golden/make_golden_thermal.py

* dJ_B(u), dJ_F(u) on the reference's grid (u = m/T in [0, 100], 256 points):
  the quadratures ``FlatonPotential._dJb_exact`` / ``_dJf_exact`` of
  potential/flatonPotential.py (the same integrals as cosmoTransitions'
  finiteT.dJb_exact / dJf_exact that the simulation calls; cosmoTransitions is
  not vendored, and flatonPotential imports it at module level, so the two
  methods are AST-extracted and bound to numpy);
* the lattice-counterterm soft parts (R:461-490 ``_dJ_soft_boson`` /
  ``_dJ_soft_fermion``, nested in the script's ``if cli_args.counterterm``,
  AST-extracted) at one cutoff;
* the not-a-knot cubic spline coefficients the script builds (R:437-447,
  scipy.interpolate.CubicSpline);
* ``Vprime_field`` (R:1435, the numba kernel, AST-extracted) on a random field
  and ``Vprime_scalar`` / ``build_vprime_table`` (R:805-849) on a phi grid, with
  the script's default couplings (R:642-643, R:744-748).
"""
from __future__ import annotations

import ast
import math
import os
import sys
import types

import numpy as np
from scipy.integrate import quad
from scipy.interpolate import CubicSpline

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import ref_extract  # noqa: E402

REF = os.path.dirname(os.path.dirname(ref_extract.REAL_SCRIPT))
POT = os.path.join(REF, "potential", "flatonPotential.py")


def _methods(path, cls, names):
    tree = ast.parse(open(path).read())
    out = {}
    for node in tree.body:
        if isinstance(node, ast.ClassDef) and node.name == cls:
            for f in node.body:
                if isinstance(f, ast.FunctionDef) and f.name in names:
                    mod = ast.Module(body=[f], type_ignores=[])
                    ns = {"scipy": __import__("scipy"), "np": np, "math": math}
                    __import__("scipy.integrate")
                    exec(compile(ast.fix_missing_locations(mod), path, "exec"), ns)
                    out[f.name] = ns[f.name]
    return out


def _nested(path, names):
    """Functions defined inside top-level `if` blocks of a script."""
    tree = ast.parse(open(path).read())
    out = {}
    for node in tree.body:
        if isinstance(node, ast.If):
            for f in node.body:
                if isinstance(f, ast.FunctionDef) and f.name in names:
                    mod = ast.Module(body=[f], type_ignores=[])
                    ns = {"math": math, "_ct_quad": quad}
                    exec(compile(ast.fix_missing_locations(mod), path, "exec"), ns)
                    out[f.name] = ns[f.name]
    return out


def main():
    fp = _methods(POT, "FlatonPotential", ["_dJb_exact", "_dJf_exact"])
    self = types.SimpleNamespace(exp=np.exp, sqrt=np.sqrt, log=np.log)
    u = np.linspace(0.0, 100.0, 256, dtype=np.float64)
    djb = np.array([fp["_dJb_exact"](self, x) for x in u])
    djf = np.array([fp["_dJf_exact"](self, x) for x in u])
    soft = _nested(ref_extract.REAL_SCRIPT, ["_dJ_soft_boson", "_dJ_soft_fermion"])
    x_cut = 2.5
    sb = np.array([soft["_dJ_soft_boson"](float(y), x_cut) for y in u])
    sf = np.array([soft["_dJ_soft_fermion"](float(y), x_cut) for y in u])
    cb = CubicSpline(u, djb, bc_type="not-a-knot").c
    cf = CubicSpline(u, djf, bc_type="not-a-knot").c
    spl = {"c0_b": cb[0].copy(), "c1_b": cb[1].copy(), "c2_b": cb[2].copy(), "c3_b": cb[3].copy(),
           "c0_f": cf[0].copy(), "c1_f": cf[1].copy(), "c2_f": cf[2].copy(), "c3_f": cf[3].copy(),
           "x_min": 0.0, "h_y": float(u[1] - u[0]), "inv_hy": 1.0 / float(u[1] - u[0]),
           "xhi_clamp": float(u[1] - u[0]) * 255 - 1e-12, "nseg": 255}
    R = ref_extract.load_real(pot_coeffs=(1.0, 1.0), splines=spl)
    couplings = dict(lam=1e-24, mphi=1000.0, bosonMassSquared=1.0e6, bosonCoupling=1.09,
                     bosonGaugeCoupling=1.05, fermionCoupling=1.09, fermionGaugeCoupling=1.05)
    rng = np.random.default_rng(11)
    phi = rng.normal(0.0, 4000.0, (12, 10, 8))
    T = 3000.0
    out = np.empty_like(phi)
    R["Vprime_field"](out, phi, T, couplings["lam"], couplings["mphi"],
                      couplings["bosonMassSquared"], couplings["bosonCoupling"],
                      couplings["bosonGaugeCoupling"], couplings["fermionCoupling"],
                      couplings["fermionGaugeCoupling"])
    g = dict(spl)
    g.update(couplings)
    g["_POT_COEFFS"] = np.array([1.0, 1.0])
    S = ref_extract._load(ref_extract.REAL_SCRIPT, ["Vprime_scalar", "build_vprime_table"], [], g)
    tab, tmin, dinv = S["build_vprime_table"](T, -20000.0, 20000.0, 4096)
    np.savez_compressed(os.path.join(HERE, "thermal.npz"), u=u, djb=djb, djf=djf, x_cut=x_cut,
                        soft_b=sb, soft_f=sf, cb=cb, cf=cf, phi=phi, T=T, vprime_field=out,
                        table=tab, tmin=tmin, dinv=dinv,
                        **{k: np.float64(v) for k, v in couplings.items()})
    print("wrote thermal.npz", djb[:3], djf[:3], sb[:3])


if __name__ == "__main__":
    main()
