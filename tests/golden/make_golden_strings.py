"""Generate tests/golden/strings.npz: string networks evolved by the REFERENCE's own
complex-field kernels, with the reference's winding numbers of the evolved field.

    TIPT_REFERENCE_ROOT=<reference checkout> python tests/golden/make_golden_strings.py

A complex field Phi = phi1 + i phi2 starts near zero with random phases and is
quenched below T0 (U(1) toy potential V(|Phi|) = D(T^2-T0^2)|Phi|^2 - E T |Phi|^3
+ lam/4 |Phi|^4, tabulated in |Phi|): the phases order domain by domain and a
network of global strings is left where the domains meet.  The evolution is the
reference's complex ``rk2_step_table`` (C:2067-2215, AST-extracted by
ref_extract.py) on float32 arrays -- the reference's default precision
(USE_FLOAT32, C:346) -- with its hash noise (C:2958-2974 seeding, one cos/sin
pair per site) filled into the noise arrays.  The winding numbers are the
reference's ``compute_winding_number`` (C:2683-2744) on FP64 casts of the
float32 fields, as its snapshot writer calls it (C:4627-4629), and the string
count is its ``np.sum(np.abs(winding) > 0.5)`` (C:4661).  The per-orientation
plaquette windings come from the reference's vectorised restatement
``tools/winding.py`` (imported from the checkout).

Fixture generation only: the GPU box never needs the reference.
"""
from __future__ import annotations

import importlib.util
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import make_golden as MG  # noqa: E402  (hash noise fill, tables, save)
import ref_extract  # noqa: E402

D, E, LAM, T0 = 0.1, 0.05, 0.1, 1.0


def _winding_tool():
    path = os.path.join(ref_extract.REF_ROOT, "tools", "winding.py")
    spec = importlib.util.spec_from_file_location("ref_tools_winding", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def evolve(Ck, shape, T, n_steps, seed):
    """Quench: |Phi| ~ 0.05, uniform random phases, pi = 0; n_steps of the
    reference's complex midpoint step at temperature T on float32 arrays."""
    dt, dx, eta, mu, inv_a2 = 0.05, 1.0, 1.0, 1.0, 1.0
    ns = math.sqrt(2.0 * eta * T * dt / dx ** 3)
    x = np.linspace(0.0, 4.0, 4096)
    tab = (2.0 * D * (T * T - T0 * T0) * x - 3.0 * E * T * x * x + LAM * x ** 3).astype(np.float64)
    tmin, dinv, npts = 0.0, 4095 / 4.0, 4096
    rng = np.random.default_rng(seed)
    th = rng.uniform(-np.pi, np.pi, shape)
    rho = 0.05 * np.abs(rng.normal(1.0, 0.3, shape))
    f32 = np.float32
    p1, p2 = (rho * np.cos(th)).astype(f32), (rho * np.sin(th)).astype(f32)
    v1, v2 = np.zeros(shape, f32), np.zeros(shape, f32)
    tmp = [np.empty(shape, f32) for _ in range(4)]
    for n in range(n_steps):
        n1 = MG.noise(shape, n, MG.K_PASS2, ns, 0, f32)
        n2 = MG.noise(shape, n, MG.K_PASS2, ns, 1, f32)
        Ck["rk2_step_table"](p1, p2, v1, v2, dt, dx, eta, mu, n1, n2, *tmp, inv_a2, tab, tmin,
                             dinv, npts)
    return p1, p2


def main():
    Ck = ref_extract.load_complex()
    tool = _winding_tool()
    out = {}
    # (tag, shape, T, steps, seed): a cubic network and a non-cubic lattice with a
    # hotter, noisier one (more phase differences near +-pi)
    cases = [("a", (48, 48, 48), 0.6, 600, 71), ("b", (40, 32, 24), 0.8, 300, 72)]
    for tag, shape, T, steps, seed in cases:
        p1, p2 = evolve(Ck, shape, T, steps, seed)
        w = np.empty(shape, np.float32)
        Ck["compute_winding_number"](p1.astype(np.float64), p2.astype(np.float64), w)
        a1, a2 = p1.astype(np.float64), p2.astype(np.float64)
        th = np.arctan2(a2, a1)
        r = lambda a, ax: np.roll(a, -1, axis=ax)  # noqa: E731
        w3 = np.stack([
            tool._plaquette_winding_arr(th, r(th, 0), r(r(th, 0), 1), r(th, 1)),
            tool._plaquette_winding_arr(th, r(th, 0), r(r(th, 0), 2), r(th, 2)),
            tool._plaquette_winding_arr(th, r(th, 1), r(r(th, 1), 2), r(th, 2))])
        w3i = np.round(w3).astype(np.int8)
        out[f"{tag}_phi1"], out[f"{tag}_phi2"] = p1, p2
        out[f"{tag}_w"] = np.round(w).astype(np.int8)
        out[f"{tag}_w3"] = w3i
        out[f"{tag}_n_strings"] = np.int64(np.sum(np.abs(w) > 0.5))  # C:4661
        out[f"{tag}_n_pierced"] = np.array([(w3i[o] != 0).sum() for o in range(3)], np.int64)
        out[f"{tag}_string_voxel_fraction"] = tool.string_voxel_fraction(w)
        out[f"{tag}_T"], out[f"{tag}_steps"] = T, steps
        # the two restatements of the reference agree on the per-site sum
        assert np.array_equal(np.round(w), np.round(w3.sum(axis=0)))
        d = np.abs(np.arctan2(np.sin(r(th, 0) - th), np.cos(r(th, 0) - th)))
        print(f"{tag}: {shape} T={T} steps={steps}: strings {out[f'{tag}_n_strings']}, "
              f"pierced {out[f'{tag}_n_pierced'].tolist()}, "
              f"|dtheta| > 3.1 on {int((d > 3.1).sum())} links")
    MG.save("strings.npz", **out)


if __name__ == "__main__":
    main()
