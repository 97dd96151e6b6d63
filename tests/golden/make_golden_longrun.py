"""Generate tests/golden/longrun.npz: long-run statistics of the REFERENCE's own
kernels, for the ensemble-level parity tests (mean nucleation time, string
density), where trajectories of different implementations cannot be compared
step by step.

    TIPT_REFERENCE_ROOT=<reference checkout> python tests/golden/make_golden_longrun.py

Real field (nucleation): 64 replicas of a 32^3 periodic lattice, toy potential
V = D(T^2-T0^2)phi^2 - E T phi^3 + lam/4 phi^4 (D = 0.1, E = 0.05, lam = 0.1,
T0 = 1) at T = 1.07 (above T0: the symmetric phase is metastable and the
first passage is spread over thousands of steps), V' tabulated on 4096 points
of [-3, 4] -- the range the noisy field explores, phi < 0 included, so the
table represents the same potential as the polynomial V' of the batched
engine the test compares with (a table starting at 0 would extrapolate
linearly below it, a different potential for phi < 0) -- dt = 0.05, dx = 1,
gamma = 1, phi ~ N(0, 0.01^2), pi = 0.  Each
replica is stepped by the reference's ``rk2_step_table`` (R:1875-1966) on
float32 arrays (its default precision, USE_FLOAT32, R:348) until the converted
fraction mean(phi > 1) exceeds 1/2 at a check every 10 steps (at most 10^4
steps); the first-passage step is the last step of that check interval.

Complex field (strings): 16 replicas of a 32^3 lattice quenched from
|Phi| ~ 0.05 with random phases at T = 0.6 (U(1) toy potential tabulated in
|Phi|), the reference's complex ``rk2_step_table`` (C:2067-2215) on float32
arrays for 1000 steps; every 100 steps the reference's
``compute_winding_number`` (C:2683-2744, on FP64 casts as C:4627-4629) and the
string voxel fraction mean(|w| > 0.5) (tools/winding.py:67-70, C:4661).

Noise: the reference kernels take noise arrays; they are filled with the
reference's hash (R:2322-2336) and Box-Muller expression (R:2519-2521, the
complex field's cos/sin pair C:2965-2970) at the reference key
uint64(site*73856093) ^ step (R:2511-2520), plus replica_seed *
0x9E3779B97F4A7C15 (mod 2^64) -- the seed extension of this library, zero for
the reference's own single run -- so that replicas are independent.

Fixture generation only: the GPU box never needs the reference.
"""
from __future__ import annotations

import math
import os
import sys

import numba as nb
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import make_golden as MG  # noqa: E402
import ref_extract  # noqa: E402

D, E, LAM, T0 = 0.1, 0.05, 0.1, 1.0
DT = 0.05
SEED_STRIDE = 0x9E3779B97F4A7C15

REAL = dict(shape=(32, 32, 32), T=1.07, replicas=64, max_steps=10000, check_every=10,
            thr=1.0, stop_frac=0.5, seed0=1)
CPLX = dict(shape=(32, 32, 32), T=0.6, replicas=16, steps=1000, every=100, seed0=101)


def _make_seeded_fill(hash_fn):
    @nb.njit(parallel=True, cache=False)
    def fill(out1, out2, step, mul, seed, scale):
        nx, ny, nz = out1.shape
        nyz = nb.int64(ny) * nb.int64(nz)
        add = nb.uint64(seed) * nb.uint64(SEED_STRIDE)
        for i in nb.prange(nx):
            for j in range(ny):
                for k in range(nz):
                    site = nb.int64(i) * nyz + nb.int64(j) * nb.int64(nz) + nb.int64(k)
                    key = (nb.uint64(site * nb.int64(mul)) ^ nb.uint64(step)) + add
                    u1, u2 = hash_fn(key)
                    r = math.sqrt(-2.0 * math.log(u1))
                    out1[i, j, k] = scale * (r * math.cos(6.283185307179586 * u2))
                    out2[i, j, k] = scale * (r * math.sin(6.283185307179586 * u2))
    return fill


def toy(x, T):
    return 2.0 * D * (T * T - T0 * T0) * x - 3.0 * E * T * x * x + LAM * x ** 3


def real_runs(R, fill):
    c = REAL
    shape, T = c["shape"], c["T"]
    x = np.linspace(-3.0, 4.0, 4096)
    tab, tmin, dinv, npts = toy(x, T).astype(np.float64), -3.0, 4095 / 7.0, 4096
    ns = math.sqrt(2.0 * T * DT)
    f32 = np.float32
    n1, n2 = np.empty(shape), np.empty(shape)
    first = np.full(c["replicas"], -1, np.int64)
    curves = np.full((c["replicas"], c["max_steps"] // c["check_every"]), np.nan)
    for r in range(c["replicas"]):
        seed = c["seed0"] + r
        rng = np.random.default_rng(1000 + seed)
        phi = rng.normal(0.0, 0.01, shape).astype(f32)
        pi = np.zeros(shape, f32)
        tmp = [np.empty(shape, f32), np.empty(shape, f32)]
        for n in range(c["max_steps"]):
            fill(n1, n2, np.uint64(n), MG.K_PASS2, np.uint64(seed), ns)
            R["rk2_step_table"](phi, pi, DT, 1.0, 1.0, 1.0, n1.astype(f32), *tmp, 1.0, tab, tmin,
                                dinv, npts)
            if (n + 1) % c["check_every"] == 0:
                fr = float(np.mean(phi > c["thr"]))
                curves[r, (n + 1) // c["check_every"] - 1] = fr
                if fr > c["stop_frac"]:
                    first[r] = n
                    break
        print(f"real replica {r}: first passage {first[r]}", flush=True)
    return first, curves


def complex_runs(Ck, fill, winding_tool):
    c = CPLX
    shape, T = c["shape"], c["T"]
    x = np.linspace(0.0, 4.0, 4096)
    tab, tmin, dinv, npts = toy(x, T).astype(np.float64), 0.0, 4095 / 4.0, 4096
    ns = math.sqrt(2.0 * T * DT)
    f32 = np.float32
    n1, n2 = np.empty(shape), np.empty(shape)
    fr = np.zeros((c["replicas"], c["steps"] // c["every"]))
    for r in range(c["replicas"]):
        seed = c["seed0"] + r
        rng = np.random.default_rng(2000 + seed)
        th = rng.uniform(-np.pi, np.pi, shape)
        rho = 0.05 * np.abs(rng.normal(1.0, 0.3, shape))
        p1, p2 = (rho * np.cos(th)).astype(f32), (rho * np.sin(th)).astype(f32)
        v1, v2 = np.zeros(shape, f32), np.zeros(shape, f32)
        tmp = [np.empty(shape, f32) for _ in range(4)]
        w = np.empty(shape, np.float32)
        for n in range(c["steps"]):
            fill(n1, n2, np.uint64(n), MG.K_PASS2, np.uint64(seed), ns)
            Ck["rk2_step_table"](p1, p2, v1, v2, DT, 1.0, 1.0, 1.0, n1.astype(f32),
                                 n2.astype(f32), *tmp, 1.0, tab, tmin, dinv, npts)
            if (n + 1) % c["every"] == 0:
                Ck["compute_winding_number"](p1.astype(np.float64), p2.astype(np.float64), w)
                fr[r, (n + 1) // c["every"] - 1] = winding_tool.string_voxel_fraction(w)
        print(f"complex replica {r}: string fraction {fr[r].round(4).tolist()}", flush=True)
    return fr


def main():
    import importlib.util
    R = ref_extract.load_real()
    Ck = ref_extract.load_complex()
    fill = _make_seeded_fill(R["_hash_rng_pair"])
    spec = importlib.util.spec_from_file_location(
        "ref_tools_winding", os.path.join(ref_extract.REF_ROOT, "tools", "winding.py"))
    wt = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(wt)
    first, curves = real_runs(R, fill)
    sfrac = complex_runs(Ck, fill, wt)
    out = {"real_first_passage": first, "real_frac_curves": curves,
           "complex_string_fraction": sfrac}
    for k, v in REAL.items():
        out[f"real_{k}"] = np.array(v)
    for k, v in CPLX.items():
        out[f"complex_{k}"] = np.array(v)
    MG.save("longrun.npz", **out)


if __name__ == "__main__":
    main()
