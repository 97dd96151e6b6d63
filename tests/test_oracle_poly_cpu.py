"""The oracle's polynomial V' midpoint step (the batched replicas' potential,
V'(x) = c1 x + c2 x^2 + c3 x^3) pinned to its table step, which the reference's
own rk2_step_table fixtures pin (R:1875-1966): with a fine table of the same
potential the two differ only by the table's interpolation error, and a wrong
sign or a dropped term is far outside that."""
import numpy as np

from oracle import oracle as O

D, LAM, T0 = 0.1, 0.1, 1.0


def _coeffs(T, E):
    return 2.0 * D * (T * T - T0 * T0), -3.0 * E * T, LAM


def _run(step, shape=(12, 10, 8), nsteps=5):
    rng = np.random.default_rng(7)
    phi = rng.normal(0.8, 0.5, shape)
    pi = rng.normal(0.0, 0.3, shape)
    for n in range(nsteps):
        step(phi, pi, n)
    return phi, pi


def test_poly_midpoint_matches_fine_table():
    T, E = 0.99, 0.055
    c1, c2, c3 = _coeffs(T, E)
    lo, hi, npts = -3.0, 4.0, 1 << 16
    tab, tmin, dinv = O.build_table(lambda x: O.toy_vprime(x, T, D, E, LAM, T0), lo, hi, npts)

    def table_step(phi, pi, n):
        O.rk2_step_table(phi, pi, 0.05, 1.0, 1.0, 1.0, None, np.empty_like(phi),
                         np.empty_like(pi), 1.0, tab, tmin, dinv, npts, noise_scale=0.31,
                         noise_step=n, noise_seed=4)

    def poly_step(coeffs):
        def f(phi, pi, n):
            O.rk2_step_poly(phi, pi, 0.05, 1.0, 1.0, 1.0, 1.0, *coeffs, noise_scale=0.31,
                            noise_step=n, noise_seed=4)
        return f

    a = _run(table_step)
    b = _run(poly_step((c1, c2, c3)))
    err = max(np.abs(a[0] - b[0]).max(), np.abs(a[1] - b[1]).max())
    assert err < 1e-7, err
    # the comparison sees each coefficient: a flipped sign of c2 or a dropped c1 fails
    for bad in ((c1, -c2, c3), (0.0, c2, c3), (c1, c2, -c3)):
        w = _run(poly_step(bad))
        assert max(np.abs(a[0] - w[0]).max(), np.abs(a[1] - w[1]).max()) > 1e-4, bad


def test_poly_midpoint_2d_lattice():
    """nz = 1: the 7-point stencil degenerates to the 5-point one (kp = km = k)."""
    T, E = 1.005, 0.045
    c = _coeffs(T, E)
    tab, tmin, dinv = O.build_table(lambda x: O.toy_vprime(x, T, D, E, LAM, T0), -3.0, 4.0,
                                    1 << 16)
    a = _run(lambda p, q, n: O.rk2_step_table(p, q, 0.05, 1.0, 1.0, 1.0, None, np.empty_like(p),
                                              np.empty_like(q), 1.0, tab, tmin, dinv, 1 << 16,
                                              noise_scale=0.3, noise_step=n, noise_seed=9),
             shape=(16, 12, 1))
    b = _run(lambda p, q, n: O.rk2_step_poly(p, q, 0.05, 1.0, 1.0, 1.0, 1.0, *c, noise_scale=0.3,
                                             noise_step=n, noise_seed=9), shape=(16, 12, 1))
    assert max(np.abs(a[0] - b[0]).max(), np.abs(a[1] - b[1]).max()) < 1e-7
