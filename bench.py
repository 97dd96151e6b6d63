#!/usr/bin/env python3
"""Benchmark of the lattice Langevin stepper (site-updates/s, HBM roofline).

Workload (one "step" = one midpoint RK2 dt-step of the whole lattice): real
scalar field on a 512^3 periodic lattice, FP32-compensated (hi/lo) storage,
7-point Laplacian, 2-D V'(phi, T) table (4096 phi x 256 T points, bilinear)
of V = D(T^2-T0^2)phi^2 - E T phi^3 + lam/4 phi^4 (D=0.1, E=0.05, lam=0.1,
T0=1), T cooling linearly 1.05 -> 0.98 over 1e4 steps, dt=0.05, dx=1, gamma=1,
counter-based hash noise with seed 1, phi ~ N(0, 0.01^2), pi = 0.
Synthetic inputs (the reference has no dataset).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl tipt|reference]

N > 1 (torchrun, one rank per GPU): by default one (N*512) x 512 x 512 lattice
split into x-slabs of 512 planes per rank (weak scaling), with the ghost planes
of phi and pi exchanged point to point over NCCL every step, overlapped with
the interior planes (slab.Slab); the W ranks reproduce the single-lattice step
bit for bit.  `--decomp replicas` runs independent 512^3 replicas instead (seed
1 + rank, no collective on the data path).  The elapsed time is the max over
ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "site-updates/s"
D, E, LAM, T0 = 0.1, 0.05, 0.1, 1.0
DT, DX, ETA = 0.05, 1.0, 1.0
T_START, T_END, N_COOL = 1.05, 0.98, 10000
NPHI, NT, PHI_LO, PHI_HI, TT_LO, TT_HI = 4096, 256, 0.0, 3.0, 0.97, 1.06
BYTES_PER_SITE = {"f32c": 32, "f64": 32, "f32": 16}


def temperature(n):
    """Linear cooling T(t) = T_start - rate*t (the temperature(t) form of R:2828-2829)."""
    rate = (T_START - T_END) / (N_COOL * DT)
    return max(T_START - rate * (n * DT), 0.0)


def noise_scale(T):
    """ns = sqrt(2 eta T dt / dx^3) (R:3714-3718 with a = mu = dx_phys = 1)."""
    return math.sqrt(2.0 * ETA * T * DT / DX ** 3)


def toy_vprime(phi, T):
    return 2.0 * D * (T * T - T0 * T0) * phi - 3.0 * E * T * phi * phi + LAM * phi ** 3


def build_table_2d():
    x = np.linspace(PHI_LO, PHI_HI, NPHI, dtype=np.float64)
    Ts = np.linspace(TT_LO, TT_HI, NT, dtype=np.float64)
    t2 = np.stack([toy_vprime(x, T) for T in Ts]).astype(np.float64)
    return (np.ascontiguousarray(t2), PHI_LO, 1.0 / ((PHI_HI - PHI_LO) / (NPHI - 1)), TT_LO,
            1.0 / ((TT_HI - TT_LO) / (NT - 1)))


# ---------------------------------------------------------------- clocks ---
class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE,
                stderr=subprocess.DEVNULL, text=True)
            self.thr = threading.Thread(target=self._read, daemon=True)
            self.thr.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                mx = float(f[1])
            except ValueError:
                continue
            for nm, v in zip(names, f[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------ distributed ---
def dist_setup(args):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        # NCCL's communicator set-up log (ranks, devices, transports) on stderr
        os.environ.setdefault("NCCL_DEBUG", "INFO")
        os.environ.setdefault("NCCL_DEBUG_SUBSYS", "INIT")
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    return world, rank, local


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# -------------------------------------------------------------- CPU arms ---
def cpu_oracle_rate(n_side, budget_s=12.0, max_steps=20, shape=None, warmup=1,
                    dtype=np.float64):
    """Site-updates/s of the CPU restatement (oracle/, OpenMP, all host threads) on
    the same step: midpoint RK2, blended 2-D table row, inline hash noise.  float64
    arrays: the FP64 step; float32 arrays: the reference's float32 mode (its default,
    USE_FLOAT32 = True, R:348: float32 state and neighbour sums, FP64 arithmetic)."""
    from oracle import oracle as O
    O.build()
    shape = shape or (n_side, n_side, n_side)
    t2, tmin, dinv, Tmin, Tdinv = build_table_2d()
    rng = np.random.default_rng(1)
    phi = rng.normal(0.0, 0.01, shape).astype(dtype)
    pi = np.zeros(shape, dtype)
    tmp = [np.empty(shape, dtype), np.empty(shape, dtype)]

    def one(n):
        T = temperature(n)
        row = O.table_blend_row(t2, Tmin, Tdinv, T)
        O.rk2_step_table(phi, pi, DT, DX, ETA, 1.0, None, *tmp, 1.0, row, tmin, dinv, NPHI,
                         noise_scale=noise_scale(T), noise_step=n, noise_seed=1)

    for w in range(max(1, warmup)):
        one(w)
    w0 = max(1, warmup)
    t0 = time.perf_counter()
    n = 0
    while n < max_steps and (time.perf_counter() - t0) < budget_s:
        one(w0 + n)
        n += 1
    el = time.perf_counter() - t0
    return n * phi.size / el, n, O.num_threads(), shape


def run_reference(args, world, rank):
    """--impl reference: the reference's CPU algorithm for this path (the oracle
    port: the reference is numba/Python inside scripts that cannot be imported and
    cannot travel), all host threads, on this arm's workload; each step is one
    full-lattice step.  The value is the reference's default precision, float32
    arrays (USE_FLOAT32 = True, R:348; the oracle's float32 mode is pinned to the
    reference kernel on float32 arrays); the FP64 mode is timed beside it."""
    if rank != 0:
        return
    n = args.size
    shape = (n, n, n)
    warm = max(3, args.warmup)
    rate, steps, threads, shp = cpu_oracle_rate(n, budget_s=30.0, max_steps=max(args.steps, 1),
                                                shape=shape, warmup=warm, dtype=np.float32)
    rate64, steps64, _, _ = cpu_oracle_rate(n, budget_s=30.0, max_steps=max(args.steps, 1),
                                            shape=shape, warmup=1)
    line = {
        "metric": METRIC, "value": rate, "unit": "site-updates/s", "impl": "reference",
        "n_gpus": args.gpus, "steps": steps, "warmup": warm,
        "ms_per_step": 1000.0 * n ** 3 / rate, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": workload_name(n, "f32"), "lattice": [n, n, n],
                   "reference_mode": "float32 arrays (the reference's default, R:348)"},
        "cpu_baseline": {"value": rate, "unit": "site-updates/s", "cores": threads,
                         "kind": "port",
                         "sample": f"{steps} full {n}^3 steps on float32 arrays (after {warm} "
                                   "warm-up steps) of the CPU restatement of the reference's "
                                   "float32 mode, OpenMP over all host threads",
                         "fp64_value": rate64, "fp64_steps": steps64},
        "e2e": {"value": rate, "unit": "site-updates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def workload_name(n, storage):
    st = {"f32c": "FP32-compensated (hi/lo) storage", "f64": "FP64 storage",
          "f32": "FP32 storage"}[storage]
    return (f"real scalar field {n}^3 periodic, {st}, fused midpoint RK2 (7-point Laplacian), "
            "2-D V'(phi,T) table 4096x256 bilinear, T cooling 1.05->0.98, hash noise seed 1")


def read_traffic(storage, n):
    """DRAM bytes per launch from the committed ncu summary, if one exists."""
    path = os.path.join(ROOT, "profiles", f"rk2_stage_{storage}_{n}.txt")
    if not os.path.exists(path):
        return None
    for ln in open(path):
        if ln.startswith("dram_bytes_per_launch:"):
            try:
                return float(ln.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


# ------------------------------------------------------------------- main ---
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["tipt", "reference"], default="tipt")
    ap.add_argument("--size", type=int, default=512)
    ap.add_argument("--storage", choices=["f32c", "f64", "f32"], default="f32c")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--e2e-result", choices=["range", "observables"], default="range",
                    help="per-step result the e2e leg reads back: the new phi's range folded by "
                         "the step kernel (the reference loop's phi.min()/max()), or the 10 "
                         "observables of a separate reduction")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", choices=["lattice", "complex", "ensemble", "surrogate", "extras",
                                           "precision"],
                    default="lattice",
                    help="lattice: the 512^3 site-update headline; ensemble: Gamma estimates "
                         "per GPU-hour of the batched replica engine vs one-at-a-time launches")
    ap.add_argument("--decomp", choices=["replicas", "slab"], default=None,
                    help="N > 1: one (N n) x n x n lattice in x-slabs of n planes per rank "
                         "with a halo exchange of the ghost planes every step (slab.Slab; "
                         "the default), or independent n^3 replicas per rank; N = 1: the "
                         "single-lattice step (default) or one slab with local ghost copies")
    ap.add_argument("--prec-steps", type=int, default=10000,
                    help="steps of the precision workload (FP32C beside FP64)")
    ap.add_argument("--ens-steps", type=int, default=2000)
    ap.add_argument("--ens-scale", type=int, default=1,
                    help="divide the replica counts of the ensemble workload (profiling runs)")
    ap.add_argument("--ens-plain", type=int, default=6,
                    help="replicas per size class timed one at a time")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.decomp is None:
        args.decomp = "slab" if int(os.environ.get("WORLD_SIZE", "1")) > 1 else "replicas"
    if args.workload == "ensemble" and args.impl == "tipt":
        run_ensemble_bench(args)
        return
    if args.workload == "surrogate" and args.impl == "tipt":
        run_surrogate_bench(args)
        return
    if args.workload == "complex" and args.impl == "tipt":
        run_complex_bench(args)
        return
    if args.workload == "extras" and args.impl == "tipt":
        run_extras_bench(args)
        return
    if args.workload == "precision" and args.impl == "tipt":
        run_precision_bench(args)
        return

    if args.impl == "reference":
        world = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        run_reference(args, world, rank)
        return

    import torch
    from thermal_inflation_phase_transition_b200 import real_field as RF
    from thermal_inflation_phase_transition_b200._common import table_source
    from thermal_inflation_phase_transition_b200.observables import observables

    world, rank, local = dist_setup(args)
    dev = torch.device("cuda", torch.cuda.current_device())
    n = args.size
    shape = (n, n, n)
    N = n ** 3
    seed = 1 + rank

    t2, tmin, dinv, Tmin, Tdinv = build_table_2d()
    t2d = torch.from_numpy(t2).to(dev)

    def vsrc(step):
        return table_source(t2d, tmin, dinv, NPHI, temperature(step), Tmin, Tdinv)

    g = torch.Generator(device=dev)
    g.manual_seed(1234 + rank)
    phi64 = torch.randn(shape, dtype=torch.float64, device=dev, generator=g) * 0.01

    def make_state():
        if args.storage == "f32c":
            a = RF.to_f32c(phi64)
            b = torch.zeros((2,) + shape, dtype=torch.float32, device=dev)
        elif args.storage == "f64":
            a = phi64.clone()
            b = torch.zeros(shape, dtype=torch.float64, device=dev)
        else:
            a = phi64.float()
            b = torch.zeros(shape, dtype=torch.float32, device=dev)
        return [a, b], [torch.empty_like(a), torch.empty_like(b)]

    cur, nxt = make_state()
    slab = None
    if args.decomp == "slab":
        from thermal_inflation_phase_transition_b200.slab import Slab
        slab = Slab((world * n, n, n), rank=rank, world=world)
        loc = [slab.empty(args.storage, dev) for _ in range(4)]
        for a, b in zip(loc[:2], cur):
            slab.interior(a).copy_(b)
        cur, nxt = loc[:2], loc[2:]
        seed = 1  # one lattice: the noise is keyed by the lattice-wide site index
    stream = torch.cuda.current_stream()
    # per-step V' sources prepared outside the timed region (they only pack scalars)
    total = args.warmup + args.steps
    vsources = [vsrc(s) for s in range(total)]

    def step(s):
        nonlocal cur, nxt
        T = temperature(s)
        if slab is not None:  # ghost-plane exchange, then the slab's planes
            slab.step(cur[0], cur[1], nxt[0], nxt[1], DT, DX, ETA, 1.0, 1.0, vsources[s],
                      noise_scale=noise_scale(T), noise_step=s, seed=seed)
        else:
            RF.rk2_step_table_into(cur[0], cur[1], nxt[0], nxt[1], DT, DX, ETA, 1.0, 1.0,
                                   vsources[s], noise_scale=noise_scale(T), noise_step=s,
                                   seed=seed)
        cur, nxt = nxt, cur

    for s in range(args.warmup):
        step(s)
    torch.cuda.synchronize()
    barrier(world)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        time.sleep(0.3)
        torch.cuda.synchronize()
        barrier(world)
        ev0.record(stream)
        for s in range(args.warmup, total):
            step(s)
        ev1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
    ms = ev0.elapsed_time(ev1)
    ms = max_over_ranks(ms, world)
    per_step_ms = ms / args.steps
    value = world * N * args.steps / (ms / 1000.0)
    bps = BYTES_PER_SITE[args.storage]
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        peak = json.load(open(peaks_path))["hbm_gbs"]
        peak_src = "measured"
    else:
        peak, peak_src = 6650.0, "fallback"
    achieved = bps * N / (per_step_ms / 1000.0) / 1e9
    traffic = read_traffic(args.storage, n)
    # sanity: the state really advanced and stayed finite
    if slab is not None:
        slab.exchange(cur[0], cur[1])  # the last outputs' ghost planes
    o = observables(cur[0], cur[1]).cpu().numpy()
    finite_ok = bool(o[9] == 0)

    e2e = None
    if not args.no_e2e and slab is None:
        e2e = run_e2e(args, shape, seed, RF, observables, torch, dev, world)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, steps_c, threads, shp = cpu_oracle_rate(n, budget_s=12.0, max_steps=20,
                                                      shape=(n, n, max(n // 4, 1)))
        cpu = {"value": rate, "unit": "site-updates/s", "cores": threads, "kind": "port",
               "sample": f"{steps_c} FP64 steps (after 1 warm-up) of the CPU restatement on a "
                         f"{shp[0]}x{shp[1]}x{shp[2]} periodic sub-lattice, OpenMP, same "
                         "step arithmetic (blended 2-D table, inline hash noise)"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "site-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_step_ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": args.storage, "data": "synthetic",
            "config": {"workload": workload_name(n, args.storage), "lattice": [n, n, n],
                       "storage": args.storage, "state_bytes": bps // 2 * N,
                       "l2": "inputs larger than L2 (state %.1f GB vs 126 MB L2)"
                             % (bps * N / 1e9),
                       "parallelism": (f"x-slabs x{world} of a {world * n}x{n}x{n} lattice, "
                                       "ghost-plane exchange every step"
                                       if slab is not None else
                                       f"replicas x{world}" if world > 1 else "single GPU"),
                       "finite_after_run": finite_ok},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "peak_source": peak_src,
                         "algorithmic_bytes_per_site": bps,
                         "kernel": "rk2 fused midpoint stage"},
            "gpu_launches": args.steps,
            "clocks": clk.summary(),
            "e2e": e2e,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_e2e(args, shape, seed, RF, observables, torch, dev, world):
    """End to end through the public API from pinned HOST buffers: upload the state,
    K steps of real_field.rk2_step_table (in-place semantics) each followed by a
    device->host read of the step's result, download the state.  The result is the
    new phi's range (min, max, non-finite flag) that the step kernel folds as it
    writes (the reference loop reads phi.min() and phi.max() every step), or with
    --e2e-result observables the 10 observables of a separate reduction."""
    n = args.size
    N = n ** 3
    rng = np.random.default_rng(99)
    if args.storage == "f32c":
        host_shape = (2,) + shape
        hdt = torch.float32
    else:
        host_shape = shape
        hdt = torch.float64 if args.storage == "f64" else torch.float32
    h_phi = torch.empty(host_shape, dtype=hdt).pin_memory()
    h_pi = torch.zeros(host_shape, dtype=hdt).pin_memory()
    h_phi.copy_(torch.from_numpy(rng.normal(0, 0.01, host_shape).astype(
        np.float32 if hdt == torch.float32 else np.float64)))
    if args.storage == "f32c":
        h_phi[1].zero_()
    use_range = args.e2e_result == "range"
    h_obs = torch.empty((2, 10), dtype=torch.float64).pin_memory()
    h_rng = torch.empty((2, 4), dtype=torch.int32).pin_memory()
    prange = RF.PhiRange(dev) if use_range else None
    d_phi = torch.empty(host_shape, dtype=hdt, device=dev)
    d_pi = torch.empty_like(d_phi)
    d_pt, d_vt = torch.empty_like(d_phi), torch.empty_like(d_pi)
    d_obs = torch.empty(10, dtype=torch.float64, device=dev)
    ws = torch.empty(1 << 16, dtype=torch.float64, device=dev)
    K = args.steps
    stream = torch.cuda.current_stream()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t2, tmin, dinv, Tmin, Tdinv = build_table_2d()
    table = torch.from_numpy(t2).to(dev)

    ready = [torch.cuda.Event(), torch.cuda.Event()]
    seen = []

    def one(s):
        # enqueue step s and its observables, then read step s-1's observables (the
        # host loop trails the device by one step, so the device never idles)
        T = temperature(s)
        RF.rk2_step_table(d_phi, d_pi, DT, DX, ETA, 1.0, None, d_pt, d_vt, 1.0, table, tmin, dinv,
                          NPHI, noise_scale=noise_scale(T), noise_step=s, seed=seed,
                          vp_T=T, vp_T_min=Tmin, vp_T_dinv=Tdinv, phi_range=prange)
        if use_range:
            h_rng[s % 2].copy_(prange.last, non_blocking=True)
        else:
            observables(d_phi, d_pi, out=d_obs, workspace=ws)
            h_obs[s % 2].copy_(d_obs, non_blocking=True)
        ready[s % 2].record(stream)
        if s > 0:
            read(s - 1)

    def read(s):
        ready[s % 2].synchronize()
        if use_range:
            lo, hi, bad = RF.PhiRange.decode(h_rng[s % 2].numpy())
            assert not bad, f"non-finite phi after step {s}"
            seen.append(hi - lo)  # width of phi's range after step s
        else:
            seen.append(float(h_obs[s % 2, 4]))  # <phi^2> of step s

    # warm-up (untimed)
    d_phi.copy_(h_phi)
    d_pi.copy_(h_pi)
    for s in range(3):
        one(s)
    read(2)
    torch.cuda.synchronize()
    barrier(world)
    t0 = time.perf_counter()
    ev0.record(stream)
    d_phi.copy_(h_phi, non_blocking=True)
    d_pi.copy_(h_pi, non_blocking=True)
    seen.clear()
    for s in range(K):
        one(s)
    read(K - 1)
    h_phi.copy_(d_phi, non_blocking=True)
    h_pi.copy_(d_pi, non_blocking=True)
    ev1.record(stream)
    torch.cuda.synchronize()
    assert len(seen) == K
    wall = time.perf_counter() - t0
    ms = max_over_ranks(ev0.elapsed_time(ev1), world)
    state_bytes = 2 * h_phi.numel() * h_phi.element_size()
    per_step = 16 if use_range else 80
    what = ("the new phi's min, max and non-finite flag, folded by the step kernel itself"
            if use_range else "the 10 observables of a separate reduction")
    return {"value": world * N * K / (ms / 1000.0), "unit": "site-updates/s",
            "h2d_bytes_per_step": state_bytes / K, "d2h_bytes_per_step": state_bytes / K + per_step,
            "wall_s": wall, "steps": K, "result": args.e2e_result,
            "note": "state uploaded once and downloaded once per run (amortised per step); "
                    f"every step's result ({what}) is read back to the host (the host reads "
                    "step s-1's values after enqueuing step s)"}


def run_ensemble_bench(args):
    """Batched ensemble of 1792 replicas (1024 x 128^2, 512 x 64^3, 256 x 96^3,
    T ~ U[0.98, 1.01], E ~ U[0.04, 0.06]) for up to --ens-steps steps: first-passage events of the batched
    engine per GPU-hour, and of the same replicas launched one at a time (timed on
    --ens-plain replicas per size class and scaled by the class counts; both arms produce
    bitwise identical trajectories, hence identical events).  The one-at-a-time arm is
    reported with and without its per-replica setup (state upload, graph capture).  An estimate of Gamma at
    +-10 % Poisson error needs 100 events."""
    import torch
    from thermal_inflation_phase_transition_b200 import ensemble as EN
    torch.cuda.set_device(0)
    sc = max(1, args.ens_scale)
    specs = EN.mixed_lattice_specs(n128=1024 // sc, n64=512 // sc, n96=256 // sc)
    ens = EN.Ensemble(specs, check_every=10)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    fs = ens.run(args.ens_steps, poll_every=10, record_curves=False)
    t_batched = time.perf_counter() - t0
    events = int((fs >= 0).sum())
    site_steps = 0
    for r, sp in enumerate(specs):
        n = int(np.prod(sp.shape))
        site_steps += n * ((fs[r] + 1) if fs[r] >= 0 else args.ens_steps)
    # one at a time: time a few replicas of each size class with the same engine settings
    classes = {}
    for r, sp in enumerate(specs):
        classes.setdefault(sp.shape, []).append(r)
    t_plain = 0.0
    t_plain_run = 0.0
    plain_checked = 0
    by_class = {}
    for shape, idx in classes.items():
        pick = idx[:args.ens_plain]
        tm = {}
        pf = EN.plain_first_passage([specs[r] for r in pick], args.ens_steps, check_every=10,
                                    timing=tm)
        plain_checked += int((pf == fs[pick]).sum())
        t_plain += (tm["setup_s"] + tm["run_s"]) / len(pick) * len(idx)
        t_plain_run += tm["run_s"] / len(pick) * len(idx)
        by_class["x".join(map(str, shape))] = {
            "replicas": len(idx), "timed": len(pick),
            "setup_s_per_replica": tm["setup_s"] / len(pick),
            "run_s_per_replica": tm["run_s"] / len(pick),
            "mean_first_passage_step": float(np.mean([f if f >= 0 else args.ens_steps
                                                      for f in pf]))}
    est_b = events / 100.0 / (t_batched / 3600.0)
    est_p = events / 100.0 / (t_plain / 3600.0)
    line = {
        "metric": "Gamma estimates per GPU-hour (+-10% Poisson, 100 events each)",
        "value": est_b, "unit": "estimates/GPU-hour", "n_gpus": 1, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32c", "data": "synthetic",
        "config": {"workload": "batched ensemble: 1024 x 128^2 (2-D), 512 x 64^3, 256 x 96^3 "
                               "replicas, T~U[0.98,1.01], E~U[0.04,0.06], stop at converted "
                               "fraction (phi > 1) > 0.5", "max_steps": args.ens_steps,
                   "replicas": len(specs), "events": events, "site_updates": site_steps},
        "batched_s": t_batched, "batched_site_updates_per_s": site_steps / t_batched,
        "plain_s_extrapolated": t_plain, "plain_estimates_per_gpu_hour": est_p,
        "speedup_vs_plain": t_plain / t_batched,
        "plain_stepping_only_s_extrapolated": t_plain_run,
        "plain_by_class": by_class,
        "speedup_vs_plain_stepping_only": t_plain_run / t_batched,
        "plain_events_checked_equal": f"{plain_checked}/{sum(min(len(v), args.ens_plain) for v in classes.values())}",
    }
    print(json.dumps(line, default=lambda o: o.item() if hasattr(o, "item") else str(o)),
          flush=True)


def run_precision_bench(args):
    """The cooling run in compensated FP32 beside FP64: n^3 (--size; 256 for the
    two-storage comparison the workload names, 512 for the headline lattice), T
    cooling linearly 1.05 -> 0.98 over 10^4 steps (temperature(t), R:2828-2829),
    2-D V'(phi, T) table 4096 x 256 (bilinear), hash noise seed 1, the same initial
    field.  Both runs go through the graph-captured driver with the 10 observables
    reduced (FP64, fixed order) after every step.  Reports the error of every
    observable against the FP64 run (max over the 10^4 steps), the converted-fraction
    curve of both runs and their largest difference, and each storage's step
    throughput (site-updates/s, algorithmic HBM GB/s) timed without the
    observables."""
    import torch
    from thermal_inflation_phase_transition_b200 import driver as D
    from thermal_inflation_phase_transition_b200.observables import OBS_NAMES, OBS_INDEX

    torch.cuda.set_device(0)
    n = args.size
    shape = (n, n, n)
    steps = args.prec_steps
    tab = D.Table2D.build(D.toy_vprime, 0.0, 3.0, 4096, 0.97, 1.06, 256)
    sched = D.linear_cooling(T_START, T_END, N_COOL, steps, dt=DT)
    kw = dict(table=tab, schedule=sched, seed=1, init_seed=7, graph_steps=100)
    res, rate = {}, {}
    for storage in ("f64", "f32c"):
        sim = D.Simulation(shape, storage=storage, **kw)
        t0 = time.perf_counter()
        res[storage] = sim.run(steps)
        wall = time.perf_counter() - t0
        # step throughput without the observables (fresh instance, same workload)
        s2 = D.Simulation(shape, storage=storage, **kw)
        s2.run(100, observe=False)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        s2.run(200, observe=False)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / 200
        rate[storage] = {"ms_per_step": ms, "site_updates_per_s": n ** 3 / (ms / 1e3),
                         "hbm_gbs_algorithmic": BYTES_PER_SITE[storage] * n ** 3 / (ms / 1e3) / 1e9,
                         "run_wall_s_with_observables": wall}
        del sim, s2
        torch.cuda.empty_cache()
    a, b = res["f64"], res["f32c"]
    errs = {}
    for q, name in enumerate(OBS_NAMES):
        if name == "n_nonfinite":
            continue
        d = np.abs(b[:, q] - a[:, q])
        scale = np.maximum(np.abs(a[:, q]), 1e-300)
        errs[name] = {"max_abs": float(d.max()), "max_rel": float((d / scale).max()),
                      "final_rel": float(d[-1] / scale[-1])}
    kf = OBS_INDEX["frac_above"]
    every = max(1, steps // 40)
    idx = np.arange(every - 1, steps, every)
    line = {
        "metric": "compensated-FP32 error against FP64 (max over the run)", "unit": "relative",
        "value": errs["phi2_mean"]["max_rel"], "higher_is_better": False,
        "workload": "precision", "steps": steps, "n_gpus": 1, "data": "synthetic",
        "config": {"workload": f"real scalar field {n}^3 periodic, T cooling 1.05->0.98 over "
                               f"1e4 steps, 2-D V' table 4096x256, hash noise seed 1, "
                               "f32c and f64 from the same initial field",
                   "lattice": [n, n, n], "dt": DT},
        "phi2_mean_max_rel_err": errs["phi2_mean"]["max_rel"],
        "phi2_mean_target": 1e-6,
        "observable_errors_vs_f64": errs,
        "frac_above_1": {"steps": idx.tolist(), "f64": a[idx, kf].tolist(),
                         "f32c": b[idx, kf].tolist(),
                         "max_abs_diff_all_steps": float(np.abs(b[:, kf] - a[:, kf]).max())},
        "throughput": rate,
    }
    print(json.dumps(line), flush=True)


def run_complex_bench(args):
    """Complex field, 512^3 compensated FP32, V = D(T^2-T0^2)|Phi|^2 - E T |Phi|^3
    + lam/4 |Phi|^4 tabulated in |Phi| (4096 points on [0, 3]) plus eps Re(Phi^4) analytic
    (eps = 1e-3), T = 0.98 (below T0: the U(1) breaks and strings form), hash noise per
    component, seed 2; tile shape from the autotuner.  One step = one midpoint dt-step of
    the whole lattice.  The plaquette winding (all three orientations, string length) runs
    every 500 steps; it is timed separately and amortised into `ms_per_step_with_winding`."""
    import torch
    from thermal_inflation_phase_transition_b200 import autotune as AT
    from thermal_inflation_phase_transition_b200 import complex_field as CF
    from thermal_inflation_phase_transition_b200 import real_field as RF
    from thermal_inflation_phase_transition_b200._common import table_source
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    n = args.size
    shape = (n, n, n)
    N = n ** 3
    T = 0.98
    x = np.linspace(PHI_LO, PHI_HI, NPHI)
    tab = torch.from_numpy(toy_vprime(x, T)).to(dev)
    vs = table_source(tab, PHI_LO, 1.0 / ((PHI_HI - PHI_LO) / (NPHI - 1)), NPHI)
    ns = noise_scale(T)
    tiles = AT.apply(shape, "f32c", field="complex", tune_if_missing=True)
    g = torch.Generator(device=dev)
    g.manual_seed(2)
    cur = [RF.to_f32c(0.01 * torch.randn(shape, dtype=torch.float64, device=dev, generator=g))
           for _ in range(2)]
    cur += [torch.zeros_like(cur[0]), torch.zeros_like(cur[0])]
    nxt = [torch.empty_like(a) for a in cur]

    def step(k):
        nonlocal cur, nxt
        CF.rk2_step_table_into(cur, nxt, DT, DX, ETA, 1.0, 1.0, vs, eps4=1e-3, noise_scale=ns,
                               noise_step=k, seed=2)
        cur, nxt = nxt, cur

    total = args.warmup + args.steps
    for k in range(args.warmup):
        step(k)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(0) as clk:
        time.sleep(0.3)
        torch.cuda.synchronize()
        ev0.record()
        for k in range(args.warmup, total):
            step(k)
        ev1.record()
        torch.cuda.synchronize()
    per_step_ms = ev0.elapsed_time(ev1) / args.steps
    # winding on the evolved field (all orientations, pierced-plaquette counts)
    for _ in range(2):
        wr = CF.compute_winding_number_full(cur[0], cur[1], w_site=False, w3=False)
    torch.cuda.synchronize()
    ev0.record()
    for _ in range(5):
        wr = CF.compute_winding_number_full(cur[0], cur[1], w_site=False, w3=False)
    ev1.record()
    torch.cuda.synchronize()
    wind_ms = ev0.elapsed_time(ev1) / 5
    counts = wr.host_counts()
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak = json.load(open(peaks_path))["hbm_gbs"] if os.path.exists(peaks_path) else 6650.0
    bps = 64
    achieved = bps * N / (per_step_ms / 1000.0) / 1e9
    line = {
        "metric": "complex site-updates/s", "value": N / (per_step_ms / 1000.0),
        "unit": "site-updates/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": per_step_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32c", "data": "synthetic",
        "config": {"workload": f"complex field {n}^3 periodic, FP32-compensated, V'(|Phi|) "
                               "table 4096 + eps Re(Phi^4) eps=1e-3, T=0.98, hash noise "
                               "per component seed 2", "lattice": [n, n, n],
                   "tiles": list(tiles) if tiles else "heuristic",
                   "l2": "inputs larger than L2 (state %.1f GB)" % (bps * N / 1e9)},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "algorithmic_bytes_per_site": bps,
                     "kernel": "complex rk2 fused midpoint stage"},
        "winding": {"ms": wind_ms, "every_steps": 500, "string_length": counts["string_length"],
                    "pierced": [counts["pierced_xy"], counts["pierced_xz"], counts["pierced_yz"]]},
        "ms_per_step_with_winding": per_step_ms + wind_ms / 500.0,
        "gpu_launches": args.steps, "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)


def _dev_ms(fn, reps, warm=3):
    """Mean device time of fn() over reps calls (CUDA events, after warm-up)."""
    import torch
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def run_extras_bench(args):
    """The components beyond the RK2 stepper, each on the device with a CPU path of the
    reference's algorithm timed beside it on the host:
      * overdamped Euler-Maruyama and BAOAB (R:2115, R:1974), 512^3 compensated FP32,
        1-D V' table (4096 points) at T = 1.0, hash noise; algorithmic bytes per site:
        16 (overdamped: phi hi+lo read and written) and 32 (BAOAB: phi and pi);
        CPU: the numpy simultaneous-update restatement on a 96^3 sample, one thread;
      * connected-component labelling of |phi| > 1 (scipy.ndimage.label's numbering) on
        a 512^3 compensated-FP32 field of smooth bubbles (band-limited noise); CPU:
        scipy.ndimage.label on a 256^3 field of the same kind;
      * thermal V': dJ_B + dJ_F quadrature on the 256-point grid and a 4096 x 256 (phi, T)
        table; CPU: scipy.integrate.quad of the same integrands on 16 grid points;
      * snapshot: device->host copy and npz write of a 256^3 compensated-FP32 state.
    One JSON line per component (none is the headline metric)."""
    import torch
    from oracle import integrators as OI
    from oracle import oracle as O
    from thermal_inflation_phase_transition_b200 import labels as LB
    from thermal_inflation_phase_transition_b200 import real_field as RF
    from thermal_inflation_phase_transition_b200 import thermal as TH
    from thermal_inflation_phase_transition_b200.snapshots import SnapshotWriter
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak = json.load(open(peaks_path))["hbm_gbs"] if os.path.exists(peaks_path) else 6650.0
    n = args.size
    N = n ** 3
    tab_np, tmin, dinv = O.build_table(lambda x: toy_vprime(x, 1.0), PHI_LO, PHI_HI, NPHI)
    tab = torch.from_numpy(tab_np).to(dev)
    ns = noise_scale(1.0)
    lines = []

    # ---- integrators
    g = torch.Generator(device=dev)
    g.manual_seed(7)
    phi = RF.to_f32c(0.01 * torch.randn((n, n, n), dtype=torch.float64, device=dev, generator=g))
    pi = torch.zeros_like(phi)
    ptmp, qtmp = torch.empty_like(phi), torch.empty_like(pi)
    step = [0]

    def od():
        RF.overdamped_euler_step_table(phi, DT, DX, ETA, 1.0, 1.0, tab, tmin, dinv, NPHI, ns,
                                       step[0], phi_tmp=ptmp)
        step[0] += 1

    def ba():
        RF.baoab_step_table(phi, pi, DT, DX, ETA, 1.0, 1.0, tab, tmin, dinv, NPHI, ns, step[0],
                            phi_tmp=ptmp, pi_tmp=qtmp)
        step[0] += 1

    m = 96
    rng = np.random.default_rng(3)
    cphi, cpi = rng.normal(0.0, 0.01, (m, m, m)), np.zeros((m, m, m))
    for name, fn, bps, cpu_fn in (
            ("overdamped Euler-Maruyama step", od, 16,
             lambda: OI.overdamped_step_table(cphi, DT, DX, ETA, 1.0, 1.0, tab_np, tmin, dinv,
                                              NPHI, ns, 1, sweep="jacobi")),
            ("BAOAB step", ba, 32,
             lambda: OI.baoab_step_table(cphi, cpi, DT, DX, ETA, 1.0, 1.0, tab_np, tmin, dinv,
                                         NPHI, ns, 1, sweep="jacobi"))):
        ms = _dev_ms(fn, 20)
        t0 = time.perf_counter()
        cpu_fn()
        cpu_s = time.perf_counter() - t0
        ach = bps * N / (ms / 1e3) / 1e9
        lines.append({
            "metric": f"{name} site-updates/s", "value": N / (ms / 1e3), "unit": "site-updates/s",
            "ms_per_step": ms, "dtype": "f32c", "data": "synthetic",
            "config": {"workload": f"{name}, {n}^3 compensated FP32, 1-D V' table 4096, hash noise",
                       "lattice": [n, n, n]},
            "roofline": {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s",
                         "frac": ach / peak, "algorithmic_bytes_per_site": bps},
            "cpu_baseline": {"value": m ** 3 / cpu_s, "unit": "site-updates/s", "cores": 1,
                             "kind": "port", "sample": f"one step of the numpy simultaneous-update "
                                                       f"restatement on {m}^3"}})
    assert int(RF.from_f32c(phi).isfinite().all()) == 1
    del phi, pi, ptmp, qtmp
    torch.cuda.empty_cache()

    # ---- labelling
    def bubbles(side, dev_):
        gen = torch.Generator(device=dev_)
        gen.manual_seed(11)
        w = torch.randn((side, side, side), dtype=torch.float32, device=dev_, generator=gen)
        f = torch.fft.rfftn(w)
        k = [torch.fft.fftfreq(side, device=dev_)] * 2 + [torch.fft.rfftfreq(side, device=dev_)]
        k2 = k[0][:, None, None] ** 2 + k[1][None, :, None] ** 2 + k[2][None, None, :] ** 2
        f *= torch.exp(-k2 * (side / 6.0) ** 2)
        x = torch.fft.irfftn(f, s=(side, side, side))
        return (x / x.std()).double()  # unit variance: |x| > 1 covers about a third

    fld = RF.to_f32c(bubbles(n, dev))
    lab_n = [0]

    def lab():
        lab_n[0] = LB.label(fld, 1.0)[1]

    ms = _dev_ms(lab, 5, warm=2)
    from scipy import ndimage
    c = 256
    cf = np.abs(bubbles(c, dev).cpu().numpy()) > 1.0
    t0 = time.perf_counter()
    _, nc = ndimage.label(cf)
    cpu_s = time.perf_counter() - t0
    lines.append({
        "metric": "labelling sites/s", "value": N / (ms / 1e3), "unit": "sites/s", "ms": ms,
        "dtype": "f32c", "data": "synthetic",
        "config": {"workload": f"|phi| > 1 components, {n}^3 field of smooth bubbles "
                               "(band-limited noise), face connectivity, open lattice",
                   "lattice": [n, n, n], "components": lab_n[0]},
        "cpu_baseline": {"value": c ** 3 / cpu_s, "unit": "sites/s", "cores": 1,
                         "kind": "reference", "sample": f"scipy.ndimage.label on a {c}^3 field "
                                                       f"of the same kind ({nc} components)"}})
    del fld
    torch.cuda.empty_cache()

    # ---- thermal V'
    tp = [None]

    def therm():
        tp[0] = TH.ThermalPotential(counterterm=(1.0, 1000.0), device=dev)
        tp[0].table_2d(0.0, 3000.0, 4096, 900.0, 1100.0, 256)

    t0 = time.perf_counter()
    therm()
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    therm()
    torch.cuda.synchronize()
    gpu_s = time.perf_counter() - t1
    from scipy import integrate
    us = np.linspace(0.0, 100.0, 16)
    t0 = time.perf_counter()
    for u in us:
        for sgn in (-1.0, 1.0):
            integrate.quad(lambda y: y * y * u / (math.sqrt(y * y + u * u) *
                                                  (math.exp(math.sqrt(y * y + u * u)) + sgn))
                           if y * y + u * u > 0 else 0.0, 0.0, 100.0, limit=200)
    cpu_s = time.perf_counter() - t0
    lines.append({
        "metric": "thermal V' build seconds", "value": gpu_s, "unit": "s",
        "higher_is_better": False, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "dJ_B + dJ_F quadrature on the 256-point u grid with the lattice "
                               "counterterm, not-a-knot splines, 4096 x 256 (phi, T) V' table"},
        "cpu_baseline": {"value": cpu_s * 512 / 32, "unit": "s", "cores": 1, "kind": "reference",
                         "sample": "scipy.integrate.quad of the same two integrands on 16 of "
                                   "the 256 grid points, scaled to 256 points x 2 integrands "
                                   "(the table and counterterm not included)"}})

    # ---- snapshot
    sn = 256
    st = RF.to_f32c(0.01 * torch.randn((sn, sn, sn), dtype=torch.float64, device=dev))
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        w = SnapshotWriter(d, background=False)
        t0 = time.perf_counter()
        path = w.save_real(0, 0.0, 1.0, st, st)
        wall = time.perf_counter() - t0
        size = os.path.getsize(path)
    lines.append({
        "metric": "snapshot write seconds", "value": wall, "unit": "s", "higher_is_better": False,
        "dtype": "f32c", "data": "synthetic",
        "config": {"workload": f"checkpoint (phi and pi, float64 hi+lo plus lo planes, "
                               f"compressed npz) of a {sn}^3 compensated-FP32 state",
                   "file_bytes": size}})
    for ln in lines:
        print(json.dumps(ln), flush=True)


def run_surrogate_bench(args):
    """Surrogate-steered scan over T/T0 in [0.97, 1.02], E in [0.03, 0.07], D in [0.05, 0.15],
    lam in [0.05, 0.2]: 2x10^4 training replicas (128^2 2-D, 48^3, 64^3) from the ensemble
    engine, training by the library's BF16 kernels, 64 lam* proposals on a 4x4x4 (T, E, D)
    grid for 64^3, each re-verified by a plain 256-replica ensemble; cost against a dense
    plain scan of 16 lam values per point."""
    import torch
    from thermal_inflation_phase_transition_b200 import scan as SC
    torch.cuda.set_device(0)
    t0 = time.perf_counter()
    rep = SC.steered_scan(n_train=20000, n_points=64, n_verify=256, fit_iters=4000, seed=5,
                          log=lambda m: print(m, file=sys.stderr, flush=True))
    wall = time.perf_counter() - t0
    rep.pop("net")
    v = rep["verify"]
    line = {
        "metric": "surrogate Gamma error vs plain 256-replica ensembles; GPU-hours saved vs dense scan",
        "value": v["median_abs_rel_err"], "unit": "median |Gamma_sur/Gamma_plain - 1|",
        "n_gpus": 1, "higher_is_better": False, "vs_baseline": None, "dtype": "bf16/fp32",
        "data": "synthetic",
        "config": {"workload": "surrogate-steered scan of T/T0, E, D, lam with 64^3 "
                               "verification", "train_replicas": 20000,
                   "scan_points": 64, "verify_replicas": 256, "scan_lattice": [64, 64, 64]},
        "report": rep, "wall_s": wall,
    }
    print(json.dumps(line, default=lambda o: o.item() if hasattr(o, "item") else str(o)),
          flush=True)


if __name__ == "__main__":
    main()
