"""Generate the golden fixtures in tests/golden/ by running the REFERENCE's own
numba kernels (AST-extracted by ref_extract.py from the reference checkout).

Run in a container that has the reference checkout and numba:
    TIPT_REFERENCE_ROOT=<reference checkout> python tests/golden/make_golden.py
The fixtures are small .npz files; the GPU box never needs the reference.

Every fixture stores its inputs, the reference's outputs and the parameters,
so the tests can replay the case through the oracle and the CUDA library.
Noise that the reference takes as an array is filled with the reference's own
hash (R:2322-2336) and Box-Muller expression (R:2519-2521) keyed by the
reference seeding (R:2511-2520), so the same fields drive every implementation.
"""
from __future__ import annotations

import math
import os
import sys

import numba as nb
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import ref_extract  # noqa: E402

K_PASS2 = 73856093
K_PASS4 = 19349669
TWO_PI_LIT = 6.283185307179586

R = ref_extract.load_real()
_hash = R["_hash_rng_pair"]


@nb.njit(fastmath=True, cache=False)
def _bm_cos(u1, u2):
    # the expression of R:2519-2521
    return math.sqrt(-2.0 * math.log(u1)) * math.cos(6.283185307179586 * u2)


@nb.njit(fastmath=True, cache=False)
def _bm_sin(u1, u2):
    # the expression of C:2968-2970
    return math.sqrt(-2.0 * math.log(u1)) * math.sin(6.283185307179586 * u2)


def _make_noise_fill(hash_fn):
    @nb.njit(parallel=True, cache=False)
    def fill(out, step, mul, scale, component):
        nx, ny, nz = out.shape
        nyz = nb.int64(ny) * nb.int64(nz)
        for i in nb.prange(nx):
            for j in range(ny):
                for k in range(nz):
                    site = nb.int64(i) * nyz + nb.int64(j) * nb.int64(nz) + nb.int64(k)
                    seed = nb.uint64(site * nb.int64(mul)) ^ nb.uint64(step)
                    u1, u2 = hash_fn(seed)
                    if component == 0:
                        out[i, j, k] = scale * _bm_cos(u1, u2)
                    else:
                        out[i, j, k] = scale * _bm_sin(u1, u2)
    return fill


_fill = _make_noise_fill(_hash)


def noise(shape, step, mul=K_PASS2, scale=1.0, component=0, dtype=np.float64):
    out = np.empty(shape, np.float64)
    _fill(out, np.uint64(step), mul, scale, component)
    return out.astype(dtype)


def toy_vprime(phi, T, D=0.1, E=0.05, lam=0.1, T0=1.0):
    return 2.0 * D * (T * T - T0 * T0) * phi - 3.0 * E * T * phi * phi + lam * phi ** 3


def table(T, lo=0.0, hi=3.0, n=4096):
    x = np.linspace(lo, hi, n, dtype=np.float64)
    return toy_vprime(x, T).astype(np.float64), float(lo), 1.0 / ((hi - lo) / (n - 1)), n


def save(name, **kw):
    path = os.path.join(HERE, name)
    np.savez_compressed(path, **kw)
    print(f"wrote {name}: {os.path.getsize(path) / 1024:.1f} KiB")


# ---------------------------------------------------------------- 1. hash
def gen_hash():
    rng = np.random.default_rng(11)
    seeds = [0, 1, 2, 3, 5, 1 << 32, (1 << 64) - 1, 1 << 63]
    # keys of real lattice sites/steps at the two pass multipliers
    for site in [0, 1, 2, 255, 65535, 16777215, 134217727]:
        for step in [0, 1, 2, 1999, 9999, 19999, 49999]:
            for mul in (K_PASS2, K_PASS4):
                seeds.append(((site * mul) & (2 ** 64 - 1)) ^ step)
    seeds += [int(x) for x in rng.integers(0, 2 ** 63, 4000, dtype=np.int64)]
    seeds = np.array(seeds, dtype=np.uint64)
    u1 = np.empty(seeds.size)
    u2 = np.empty(seeds.size)
    zc = np.empty(seeds.size)
    zs = np.empty(seeds.size)
    for n, s in enumerate(seeds):
        a, b = _hash(np.uint64(s))
        u1[n], u2[n] = a, b
        zc[n], zs[n] = _bm_cos(a, b), _bm_sin(a, b)
    # reference's own inline path: rk2_fused_single_pass with dt = 0, pi = 0,
    # noise_scale = 2 and zero couplings leaves pi = z(K_PASS2) + z(K_PASS4).
    sh = (6, 5, 4)
    phi = np.zeros(sh)
    pi = np.zeros(sh)
    step = 7
    R["rk2_fused_single_pass"](phi, pi, 0.0, 1.0, 0.0, 1.0, 1.0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0,
                               0.0, 0.0, 2.0, np.uint64(step), np.empty(sh), np.empty(sh), 1.0)
    save("hash_pairs.npz", seeds=seeds, u1=u1, u2=u2, z_cos=zc, z_sin=zs,
         inline_shape=np.array(sh), inline_step=step, inline_pi=pi)


# ------------------------------------------------------- 2. real midpoint
CASES = {"2d": (32, 24, 1), "3d": (12, 10, 8), "odd": (17, 9, 5)}


def _ic(shape, rng, dtype):
    # phi spans negative values (table extrapolation, R:1923-1930), the
    # barrier and the broken phase; pi is thermal-sized
    phi = rng.normal(0.6, 0.7, shape).astype(dtype)
    pi = rng.normal(0.0, 0.4, shape).astype(dtype)
    return phi, pi


def gen_rk2_step_table():
    out = {}
    dt, dx, eta, mu, inv_a2, T = 0.05, 1.0, 1.0, 1.0, 1.0, 1.02
    ns = math.sqrt(2.0 * eta * T * dt / dx ** 3)
    tab, tmin, dinv, npts = table(T)
    for tag, shape in CASES.items():
        for dtype, dn in ((np.float64, "f64"), (np.float32, "f32")):
            rng = np.random.default_rng(100 + len(tag))
            phi, pi = _ic(shape, rng, dtype)
            out[f"{tag}_{dn}_phi0"], out[f"{tag}_{dn}_pi0"] = phi.copy(), pi.copy()
            traj = []
            for n in range(10):
                nf = noise(shape, n, K_PASS2, ns, dtype=dtype)
                R["rk2_step_table"](phi, pi, dt, dx, eta, mu, nf, np.empty_like(phi),
                                    np.empty_like(pi), inv_a2, tab, tmin, dinv, npts)
                if n in (0, 9):
                    traj.append((phi.copy(), pi.copy()))
            out[f"{tag}_{dn}_phi1"], out[f"{tag}_{dn}_pi1"] = traj[0]
            out[f"{tag}_{dn}_phi10"], out[f"{tag}_{dn}_pi10"] = traj[1]
    save("rk2_step_table.npz", dt=dt, dx=dx, eta=eta, mu=mu, inv_a2=inv_a2, T=T, ns=ns,
         table=tab, tmin=tmin, dinv=dinv, npts=npts, **out)


# ------------------------------------------------------- 3. half-step pair
def gen_rk2_fused_table():
    out = {}
    dt, dx, eta, mu, inv_a2, T, Tm = 0.05, 1.0, 0.7, 1.0, 1.0, 1.03, 1.029
    ns = math.sqrt(2.0 * eta * T * dt / dx ** 3)
    ta, tmin_a, dinv_a, na = table(T)
    tb, tmin_b, dinv_b, nb_ = table(Tm, lo=-0.5, hi=3.5, n=2048)
    for tag, shape in CASES.items():
        for dtype, dn in ((np.float64, "f64"), (np.float32, "f32")):
            rng = np.random.default_rng(200 + len(tag))
            phi, pi = _ic(shape, rng, dtype)
            out[f"{tag}_{dn}_phi0"], out[f"{tag}_{dn}_pi0"] = phi.copy(), pi.copy()
            for n in range(5):
                nf = noise(shape, n, K_PASS2, ns, dtype=dtype)
                R["rk2_fused_table"](phi, pi, dt, dx, eta, mu, nf, np.empty_like(phi),
                                     np.empty_like(pi), inv_a2, ta, tmin_a, dinv_a, na, tb,
                                     tmin_b, dinv_b, nb_)
            out[f"{tag}_{dn}_phi5"], out[f"{tag}_{dn}_pi5"] = phi, pi
    save("rk2_fused_table.npz", dt=dt, dx=dx, eta=eta, mu=mu, inv_a2=inv_a2, T=T, T_mid=Tm,
         ns=ns, table_T=ta, tmin_T=tmin_a, dinv_T=dinv_a, npts_T=na, table_Tm=tb,
         tmin_Tm=tmin_b, dinv_Tm=dinv_b, npts_Tm=nb_, **out)


# ------------------------------------- 4. inline hash-noise 4-pass kernel
def gen_fused_single_pass():
    """rk2_fused_single_pass (R:2339-2647) with zero thermal couplings, so its
    inline V' reduces to lam phi^3 - mphi^2 phi (R:2228) and the case pins the
    4-pass structure with inline hash noise at both multipliers."""
    out = {}
    dt, dx, eta, mu, inv_a2 = 0.05, 1.0, 1.0, 1.0, 1.0
    T, Tm, lam, mphi, ns = 1.0, 1.0, 0.1, 0.3, 0.3
    for tag, shape in CASES.items():
        rng = np.random.default_rng(300 + len(tag))
        phi, pi = _ic(shape, rng, np.float64)
        out[f"{tag}_phi0"], out[f"{tag}_pi0"] = phi.copy(), pi.copy()
        for n in range(5):
            R["rk2_fused_single_pass"](phi, pi, dt, dx, eta, T, Tm, mu, lam, mphi, 0.0, 0.0, 0.0,
                                       0.0, 0.0, ns, np.uint64(n), np.empty_like(phi),
                                       np.empty_like(pi), inv_a2)
        out[f"{tag}_phi5"], out[f"{tag}_pi5"] = phi, pi
    save("rk2_fused_single_pass.npz", dt=dt, dx=dx, eta=eta, mu=mu, inv_a2=inv_a2, T=T,
         T_mid=Tm, lam=lam, mphi=mphi, ns=ns, **out)


# ------------------------------------------------------------- 5. complex
def gen_complex():
    out = {}
    dt, dx, eta, mu, inv_a2, T = 0.05, 1.0, 1.0, 1.0, 1.0, 1.0
    ns = math.sqrt(2.0 * eta * T * dt / dx ** 3)
    rt, rmin, rdinv, rn = table(T, lo=0.0, hi=4.0, n=4096)
    for zn_tag, zn in (("u1", (0.0, 0.0, 0.0)), ("z4", (4.0, 1e-2, 1.0))):
        Ck = ref_extract.load_complex(zn_params=zn)
        for tag, shape in CASES.items():
            rng = np.random.default_rng(400 + len(tag))
            rho = np.abs(rng.normal(0.8, 0.6, shape))
            th = rng.uniform(-np.pi, np.pi, shape)
            p1, p2 = rho * np.cos(th), rho * np.sin(th)
            v1, v2 = rng.normal(0, 0.3, shape), rng.normal(0, 0.3, shape)
            key = f"{zn_tag}_{tag}"
            out[f"{key}_phi1_0"], out[f"{key}_phi2_0"] = p1.copy(), p2.copy()
            out[f"{key}_pi1_0"], out[f"{key}_pi2_0"] = v1.copy(), v2.copy()
            for n in range(5):
                n1 = noise(shape, n, K_PASS2, ns, 0)
                n2 = noise(shape, n, K_PASS2, ns, 1)
                tmp = [np.empty(shape) for _ in range(4)]
                Ck["rk2_step_table"](p1, p2, v1, v2, dt, dx, eta, mu, n1, n2, *tmp, inv_a2, rt,
                                     rmin, rdinv, rn)
            out[f"{key}_phi1_5"], out[f"{key}_phi2_5"] = p1, p2
            out[f"{key}_pi1_5"], out[f"{key}_pi2_5"] = v1, v2
    save("rk2_complex.npz", dt=dt, dx=dx, eta=eta, mu=mu, inv_a2=inv_a2, T=T, ns=ns, table=rt,
         tmin=rmin, dinv=rdinv, npts=rn, zn_z4=np.array((4.0, 1e-2, 1.0)), **out)


# ------------------------------------------------------------- 6. winding
def _vortex_field(shape, rng, n_lines=3):
    nx, ny, nz = shape
    x, y, z = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    th = np.zeros(shape)
    for _ in range(n_lines):
        axis = rng.integers(0, 3)
        c = rng.uniform(0, max(shape), 3) + 0.37
        s = rng.choice([-1.0, 1.0])
        if axis == 0:
            th += s * np.arctan2(z - c[2] * nz / max(shape), y - c[1] * ny / max(shape))
        elif axis == 1:
            th += s * np.arctan2(z - c[2] * nz / max(shape), x - c[0] * nx / max(shape))
        else:
            th += s * np.arctan2(y - c[1] * ny / max(shape), x - c[0] * nx / max(shape))
    th += rng.normal(0, 0.9, shape)  # roughen: random windings appear too
    rho = np.abs(rng.normal(1.0, 0.3, shape))
    return (rho * np.cos(th)).astype(np.float32), (rho * np.sin(th)).astype(np.float32)


def gen_winding():
    Ck = ref_extract.load_complex()
    out = {}
    for tag, shape in {"a": (16, 12, 10), "b": (9, 7, 5), "c": (24, 20, 1)}.items():
        rng = np.random.default_rng(500 + ord(tag))
        p1, p2 = _vortex_field(shape, rng)
        w = np.empty(shape, np.float32)
        # the reference casts the float32 fields to FP64 first (C:4627-4629)
        Ck["compute_winding_number"](p1.astype(np.float64), p2.astype(np.float64), w)
        out[f"{tag}_phi1"], out[f"{tag}_phi2"], out[f"{tag}_w"] = p1, p2, w
        out[f"{tag}_n_strings"] = np.int64(np.sum(np.abs(w) > 0.5))  # C:4661
    save("winding.npz", **out)


# ---------------------------------------------------------- 7. energies
def gen_energies():
    out = {}
    for tag, shape in CASES.items():
        rng = np.random.default_rng(600 + len(tag))
        phi, pi = _ic(shape, rng, np.float64)
        ek, eg, ep = R["compute_energy_densities"](phi, pi, 0.7, 0.9, 0.1, 0.3, 1.3)
        out[f"{tag}_phi"], out[f"{tag}_pi"] = phi, pi
        out[f"{tag}_E"] = np.array([ek, eg, ep])
    save("energies.npz", dx=0.7, inv_a2=0.9, lam=0.1, mphi=0.3, mu=1.3, **out)


# ------------------------------------------- 8. 2-D 256^2 FP64 trajectory
def gen_trajectory_2d():
    """2-D 256x256 periodic lattice, FP64, dx=1, dt=0.05, gamma=1, toy potential
    D=0.1 E=0.05 lam=0.1 T0=1 at T=1.02, 4096-point table on [0,3], midpoint
    RK2 (the reference's rk2_step_table) with hash noise seed 0 at the pass-2
    multiplier, phi ~ N(0, 0.01^2), pi = 0, 2000 steps."""
    shape = (256, 256, 1)
    dt, dx, eta, mu, inv_a2, T = 0.05, 1.0, 1.0, 1.0, 1.0, 1.02
    ns = math.sqrt(2.0 * eta * T * dt / dx ** 2)
    tab, tmin, dinv, npts = table(T)
    rng = np.random.default_rng(2024)
    phi = rng.normal(0.0, 0.01, shape)
    pi = np.zeros(shape)
    phi0 = phi.copy()
    n_steps = 2000
    phi2 = np.empty(n_steps)
    frac = np.empty(n_steps)
    tmp1, tmp2 = np.empty(shape), np.empty(shape)
    noise0 = None
    for n in range(n_steps):
        nf = noise(shape, n, K_PASS2, ns)
        if n == 0:
            noise0 = nf.copy()
        R["rk2_step_table"](phi, pi, dt, dx, eta, mu, nf, tmp1, tmp2, inv_a2, tab, tmin, dinv, npts)
        phi2[n] = np.mean(phi * phi)
        frac[n] = np.mean(phi > 1.0)
        if n == 99:
            phi100, pi100 = phi.copy(), pi.copy()
    save("trajectory_2d_256.npz", dt=dt, dx=dx, eta=eta, mu=mu, inv_a2=inv_a2, T=T, ns=ns,
         table=tab, tmin=tmin, dinv=dinv, npts=npts, phi0=phi0, noise0=noise0, phi100=phi100,
         pi100=pi100, phi2_mean=phi2, frac_above_1=frac, phi_final=phi, pi_final=pi)


if __name__ == "__main__":
    gen_hash()
    gen_rk2_step_table()
    gen_rk2_fused_table()
    gen_fused_single_pass()
    gen_complex()
    gen_winding()
    gen_energies()
    gen_trajectory_2d()
