"""The alternative integrators' oracle (BAOAB, overdamped Euler-Maruyama) against
the reference's own kernels run on one thread with zero noise
(tests/golden/integrators.npz, made by tests/golden/make_golden_integrators.py)."""
import numpy as np
import pytest

from oracle import integrators as I


@pytest.fixture(scope="module")
def g(golden):
    return golden("integrators.npz")


def _par(g):
    f = lambda k: float(g[k])  # noqa: E731
    return g["table"], f("tmin"), f("dinv"), int(g["npts"]), f("dt"), f("dx"), f("mu"), f("inv_a2")


def test_real_baoab_serial_matches_reference(g):
    tab, tmin, dinv, npts, dt, dx, mu, ia2 = _par(g)
    phi, pi = g["real_phi0"], g["real_pi0"]
    for n in range(2):
        phi, pi = I.baoab_step_table(phi, pi, dt, dx, float(g["gamma"]), mu, ia2, tab, tmin, dinv,
                                     npts, 0.0, n, sweep="serial")
    np.testing.assert_allclose(phi, g["real_baoab_phi"], rtol=0, atol=1e-13)
    np.testing.assert_allclose(pi, g["real_baoab_pi"], rtol=0, atol=1e-13)


def test_real_overdamped_serial_matches_reference(g):
    tab, tmin, dinv, npts, dt, dx, mu, ia2 = _par(g)
    phi = g["real_phi0"]
    for n in range(2):
        phi = I.overdamped_step_table(phi, dt, dx, float(g["eta"]), mu, ia2, tab, tmin, dinv,
                                      npts, 0.0, n, sweep="serial")
    np.testing.assert_allclose(phi, g["real_od_phi"], rtol=0, atol=1e-13)


def test_complex_baoab_serial_matches_reference(g):
    tab, tmin, dinv, npts, dt, dx, mu, ia2 = _par(g)
    f = list(g["cplx_f0"])
    for n in range(2):
        f = list(I.complex_baoab_step_table(*f, dt, dx, float(g["gamma"]), mu, ia2, tab, tmin,
                                            dinv, npts, 0.0, n, sweep="serial"))
    for a, b in zip(f, g["cplx_baoab"]):
        np.testing.assert_allclose(a, b, rtol=0, atol=1e-13)


def test_complex_overdamped_serial_matches_reference(g):
    tab, tmin, dinv, npts, dt, dx, mu, ia2 = _par(g)
    f = list(g["cplx_f0"][:2])
    for n in range(2):
        f = list(I.complex_overdamped_step_table(*f, dt, dx, float(g["eta"]), mu, ia2, tab, tmin,
                                                 dinv, npts, 0.0, n, sweep="serial"))
    for a, b in zip(f, g["cplx_od"]):
        np.testing.assert_allclose(a, b, rtol=0, atol=1e-13)


def test_serial_and_simultaneous_sweeps_differ(g):
    """The reference's in-place sweep (neighbours visited earlier are already advanced)
    and the simultaneous update differ by a fraction of the step's own increment."""
    tab, tmin, dinv, npts, dt, dx, mu, ia2 = _par(g)
    phi0 = g["real_phi0"]
    a = I.overdamped_step_table(phi0, dt, dx, 1.3, mu, ia2, tab, tmin, dinv, npts, 0.0, 0)
    b = I.overdamped_step_table(phi0, dt, dx, 1.3, mu, ia2, tab, tmin, dinv, npts, 0.0, 0,
                                sweep="serial")
    d = np.abs(a - b).max()
    assert 0 < d < 0.2 * np.abs(a - phi0).max()
