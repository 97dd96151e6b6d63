"""Golden fixtures of the reference's alternative integrators (BAOAB and
overdamped Euler-Maruyama, R:1973-2193, C:2222-2528), generated by running the
REFERENCE's own numba kernels (AST-extracted by ref_extract.py):

    TIPT_REFERENCE_ROOT=<reference checkout> python tests/golden/make_golden_integrators.py

The reference kernels update the field in place inside a parallel loop, so a
site can see neighbours already advanced in the same sweep, and they draw their
noise from numpy's Mersenne Twister.  Both make a multi-threaded run
unreproducible.  The fixtures therefore run the kernels on one thread (a
deterministic sweep: i planes in order, 16 x 16 (j, k) tiles within a plane) with
zero noise amplitude, which pins the force, table and update arithmetic; the
oracle restates that serial sweep (``sweep="serial"``) and its simultaneous
(Jacobi) form, which the CUDA kernels implement.
"""
from __future__ import annotations

import os
import sys

import numba as nb
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import ref_extract  # noqa: E402
from make_golden import table  # noqa: E402


def main():
    nb.set_num_threads(1)
    out = {}
    rng = np.random.default_rng(77)
    tab, tmin, dinv, npts = table(1.01, 0.0, 4.0, 4096)
    out.update(table=tab, tmin=tmin, dinv=dinv, npts=npts, dt=0.05, dx=0.9, mu=1.1,
               inv_a2=0.95, gamma=0.8, eta=1.3)
    R = ref_extract.load_real()
    shape = (5, 20, 18)  # j and k extents above the 16 x 16 tile
    phi0 = rng.normal(0.4, 0.6, shape)
    pi0 = rng.normal(0.0, 0.3, shape)
    phi, pi = phi0.copy(), pi0.copy()
    for n in range(2):
        R["baoab_step_table"](phi, pi, 0.05, 0.9, 0.8, 1.1, 0.95, tab, tmin, dinv, npts, 0.0, n)
    out.update(real_phi0=phi0, real_pi0=pi0, real_baoab_phi=phi, real_baoab_pi=pi)
    phi = phi0.copy()
    for n in range(2):
        R["overdamped_euler_step_table"](phi, 0.05, 0.9, 1.3, 1.1, 0.95, tab, tmin, dinv, npts,
                                         0.0, n)
    out.update(real_od_phi=phi)
    C = ref_extract.load_complex()
    cshape = (4, 18, 17)
    f0 = [rng.normal(0.3, 0.7, cshape) for _ in range(2)] + \
         [rng.normal(0.0, 0.3, cshape) for _ in range(2)]
    f = [a.copy() for a in f0]
    for n in range(2):
        C["baoab_step_table"](*f, 0.05, 0.9, 0.8, 1.1, 0.95, tab, tmin, dinv, npts, 0.0, n)
    out.update(cplx_f0=np.stack(f0), cplx_baoab=np.stack(f))
    g = [a.copy() for a in f0[:2]]
    for n in range(2):
        C["overdamped_euler_step_table"](*g, 0.05, 0.9, 1.3, 1.1, 0.95, tab, tmin, dinv, npts,
                                         0.0, n)
    out.update(cplx_od=np.stack(g))
    np.savez_compressed(os.path.join(HERE, "integrators.npz"), **out)
    print("wrote integrators.npz", sorted(out))


if __name__ == "__main__":
    main()
