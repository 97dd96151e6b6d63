"""Batched ensembles of independent replicas and nucleation-rate estimates.

The reference studies nucleation by running one lattice per invocation and
reading the converted fraction off its snapshots.  ``Ensemble`` runs many
replicas with uneven sizes, seeds, temperatures and couplings at once: every
step is one persistent launch over a chunk work-list (``tipt_ensemble_step``);
every ``check_every`` steps a per-replica reduction records the converted
fraction (sites with phi > thr), records the first-passage step of replicas
whose fraction exceeds ``stop_frac`` and retires those whose fraction exceeds
``retire_frac`` (default: ``stop_frac``; a larger value lets the conversion
curve run on after the first passage).  The check interval is
captured once into a CUDA graph (device step counter) and replayed.

``plain_first_passage`` runs the same replicas one at a time (one lattice per
launch, graph-captured loops) -- the per-replica baseline.

``gamma_mle`` turns first-passage times into a nucleation rate per volume:
the exponential (Poisson) maximum-likelihood estimate with right censoring,
Gamma = n_events / (V * sum_i t_i), relative error 1/sqrt(n_events).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib as L
from ._common import ptr, step_params, stream_handle

__all__ = ["Ensemble", "ReplicaSpec", "toy_coefficients", "gamma_mle", "mixed_lattice_specs",
           "plain_first_passage"]


def toy_coefficients(T, E, D=0.1, lam=0.1, T0=1.0):
    """V'(phi) = c1 phi + c2 phi^2 + c3 phi^3 of V = D(T^2-T0^2)phi^2 - E T phi^3 + lam/4 phi^4."""
    return 2.0 * D * (T * T - T0 * T0), -3.0 * E * T, lam


def _magic(d):
    return 0 if d == 1 else (1 << 32) // d + (1 if (1 << 32) % d else 0)


@dataclass
class ReplicaSpec:
    shape: tuple
    T: float
    E: float
    seed: int
    D: float = 0.1
    lam: float = 0.1
    T0: float = 1.0


def mixed_lattice_specs(n128=1024, n64=512, n96=256, seed=4, T_range=(0.98, 1.01),
                  E_range=(0.04, 0.06)):
    """The 1792-replica ensemble: 1024 x 128^2 (2-D), 512 x 64^3, 256 x 96^3, seed = replica
    id, T ~ U[0.98, 1.01], E ~ U[0.04, 0.06] (fixed host RNG)."""
    rng = np.random.default_rng(seed)
    shapes = [(128, 128, 1)] * n128 + [(64, 64, 64)] * n64 + [(96, 96, 96)] * n96
    T = rng.uniform(*T_range, len(shapes))
    E = rng.uniform(*E_range, len(shapes))
    return [ReplicaSpec(tuple(s), float(t), float(e), r) for r, (s, t, e) in
            enumerate(zip(shapes, T, E))]


def _canonical(shape):
    nx, ny, nz = shape
    if nz == 1:
        return (1, nx, ny) if ny > 1 else (1, 1, nx)
    return (nx, ny, nz)


class Ensemble:
    """Replicas stepped together; see the module docstring."""

    def __init__(self, specs, *, storage="f32c", dt=0.05, dx=1.0, eta=1.0, mu=1.0, inv_a2=1.0,
                 thr=1.0, stop_frac=0.5, retire_frac=None, init_sigma=0.01, init_seed=0,
                 chunk_sites=8192, check_every=10, use_march=True, device="cuda"):
        if storage not in ("f32c", "f64"):
            raise ValueError("ensemble storage is 'f32c' or 'f64'")
        self.specs = list(specs)
        self.R = len(self.specs)
        self.storage = storage
        self.st = L.TIPT_F32C if storage == "f32c" else L.TIPT_F64
        self.dev = torch.device(device)
        self.dt, self.dx, self.eta, self.mu, self.inv_a2 = dt, dx, eta, mu, inv_a2
        self.thr, self.stop_frac, self.check_every = thr, stop_frac, max(2, check_every & ~1)
        self.retire_frac = stop_frac if retire_frac is None else max(retire_frac, stop_frac)
        reps = (L.Replica * self.R)()
        chunks = []
        off = 0
        self.sizes = np.zeros(self.R, np.int64)
        self.offsets = np.zeros(self.R, np.int64)
        # Replica offsets are multiples of 4 sites (16-byte aligned rows for the bulk
        # copies of the marching stage).
        for r, sp in enumerate(self.specs):
            n0, n1, n2 = _canonical(sp.shape)
            n = n0 * n1 * n2
            if n * max(n1, n2) >= 1 << 32:
                raise ValueError("replica too large for the 32-bit site decomposition")
            c1, c2, c3 = toy_coefficients(sp.T, sp.E, sp.D, sp.lam, sp.T0)
            ns = math.sqrt(2.0 * eta * sp.T * dt / dx ** 3)
            reps[r] = L.Replica(n0, n1, n2, _magic(n1), _magic(n2), 0, off, c1, c2, c3, ns,
                                int(sp.seed) & (2 ** 64 - 1))
            self.sizes[r] = n
            self.offsets[r] = off
            off += (n + 3) & ~3
        self.n_total = off
        # 3-D shape classes in compensated storage step on the marching stage (shared-
        # memory tiles fed by bulk copies), one launch per class; the rest (2-D
        # lattices, FP64, shapes without marching tiles) on the chunk work-list kernel
        classes = {}
        for r, sp in enumerate(self.specs):
            n0, n1, n2 = _canonical(sp.shape)
            n = n0 * n1 * n2
            if self.st == L.TIPT_F32C and use_march and \
                    L.lib().tipt_ensemble_march_supported(n0, n1, n2):
                classes.setdefault((n0, n1, n2), []).append(r)
                continue
            for b in range(0, n, chunk_sites):
                chunks.append((r, min(chunk_sites, n - b), b))
        # per class: all its replica ids, the active ones (compacted at the start of
        # every check interval) and their device count
        self._march = [(shape, torch.tensor(rids, dtype=torch.int32, device=self.dev),
                        torch.empty(len(rids), dtype=torch.int32, device=self.dev),
                        torch.zeros(1, dtype=torch.int32, device=self.dev))
                       for shape, rids in classes.items()]
        self._reps = torch.frombuffer(bytearray(bytes(reps)), dtype=torch.uint8).to(self.dev)
        ch = (L.Chunk * max(len(chunks), 1))(*[L.Chunk(*c) for c in chunks])
        self._chunks = torch.frombuffer(bytearray(bytes(ch)), dtype=torch.uint8).to(self.dev)
        self.n_chunks = len(chunks)
        phi = torch.zeros(self.n_total, dtype=torch.float64, device=self.dev)
        for r, sp in enumerate(self.specs):
            n, o = int(self.sizes[r]), int(self.offsets[r])
            phi[o:o + n] = replica_initial_phi(n, sp.seed, init_seed, init_sigma, self.dev)
        if storage == "f32c":
            hi = phi.float()
            lo = (phi - hi.double()).float()
            self.phi = [torch.stack([hi, lo]).contiguous(), None]
            self.pi = [torch.zeros((2, self.n_total), dtype=torch.float32, device=self.dev), None]
        else:
            self.phi = [phi, None]
            self.pi = [torch.zeros(self.n_total, dtype=torch.float64, device=self.dev), None]
        self.phi[1] = torch.empty_like(self.phi[0])
        self.pi[1] = torch.empty_like(self.pi[0])
        self.active = torch.ones(self.R, dtype=torch.int32, device=self.dev)
        self.n_active = torch.tensor([self.R], dtype=torch.int32, device=self.dev)
        self.first_step = torch.full((self.R,), -1, dtype=torch.int64, device=self.dev)
        self.frac = torch.zeros(self.R, dtype=torch.float64, device=self.dev)
        self._counter = torch.zeros(1, dtype=torch.int64, device=self.dev)
        self._sp = step_params(dt, dx, eta, mu, inv_a2, 0.0, 0, 0)
        self.steps_done = 0
        self.curves = []  # (step, frac[R]) per check
        self._graph = None

    def _chunk(self, K):
        lib = L.lib()
        st = stream_handle()
        for _, rids, act, n_act in self._march:
            L.check(lib.tipt_ensemble_compact(ptr(rids), rids.numel(), ptr(self.active), ptr(act),
                                              ptr(n_act), st), "tipt_ensemble_compact")
        for q in range(K):
            a, b = q & 1, (q + 1) & 1
            for (n0, n1, n2), rids, act, n_act in self._march:
                L.check(lib.tipt_ensemble_step_march(
                    ptr(self.phi[a]), ptr(self.pi[a]), ptr(self.phi[b]), ptr(self.pi[b]),
                    self.n_total, ptr(self._reps), ptr(act), act.numel(), ptr(n_act), n0, n1,
                    n2, ptr(self.active), self._sp, ptr(self._counter), q, st),
                    "tipt_ensemble_step_march")
            L.check(lib.tipt_ensemble_step(
                self.st, ptr(self.phi[a]), ptr(self.pi[a]), ptr(self.phi[b]), ptr(self.pi[b]),
                self.n_total, ptr(self._reps), ptr(self._chunks), self.n_chunks,
                ptr(self.active), self._sp, ptr(self._counter), q, st), "tipt_ensemble_step")
        # K is even: the state is back in buffer 0; the check records step counter + K - 1
        L.check(lib.tipt_ensemble_observe(
            self.st, ptr(self.phi[0]), self.n_total, ptr(self._reps), self.R, ptr(self.active),
            ptr(self.n_active), float(self.thr), float(self.stop_frac), float(self.retire_frac),
            0, ptr(self._counter),
            K - 1, ptr(self.first_step), ptr(self.frac), st), "tipt_ensemble_observe")
        L.check(lib.tipt_counter_add(ptr(self._counter), K, st), "tipt_counter_add")

    def run(self, max_steps, *, use_graphs=True, poll_every=10, record_curves=True):
        """Step until every replica converted or max_steps; returns first-passage steps
        (-1 = censored at max_steps).  Polls the active count every poll_every checks."""
        K = self.check_every
        checks = 0
        while self.steps_done + K <= max_steps:
            if use_graphs:
                if self._graph is None:
                    s = torch.cuda.Stream()
                    s.wait_stream(torch.cuda.current_stream())
                    g = torch.cuda.CUDAGraph()
                    with torch.cuda.graph(g, stream=s):
                        self._chunk(K)
                    torch.cuda.current_stream().wait_stream(s)
                    self._graph = g
                self._graph.replay()
            else:
                self._chunk(K)
            self.steps_done += K
            checks += 1
            if record_curves:
                self.curves.append((self.steps_done - 1, self.frac.clone()))
            if checks % poll_every == 0 and int(self.n_active.item()) == 0:
                break
        torch.cuda.synchronize(self.dev)
        return self.first_step.cpu().numpy()

    def frac_curves(self):
        """(steps, frac[n_checks][R]) on the host."""
        if not self.curves:
            return np.zeros(0), np.zeros((0, self.R))
        steps = np.array([c[0] for c in self.curves])
        return steps, torch.stack([c[1] for c in self.curves]).cpu().numpy()

    def replica_state(self, r):
        """(phi, pi) of replica r as FP64 tensors with its canonical shape."""
        n0, n1, n2 = _canonical(self.specs[r].shape)
        o = int(self.offsets[r])
        n = int(self.sizes[r])

        def f64(t):
            if self.storage == "f32c":
                return (t[0, o:o + n].double() + t[1, o:o + n].double()).reshape(n0, n1, n2)
            return t[o:o + n].reshape(n0, n1, n2)
        return f64(self.phi[0]), f64(self.pi[0])


def replica_initial_phi(n, replica_seed, init_seed, init_sigma, device):
    """phi ~ N(0, init_sigma^2) of one replica from its own generator (independent of the
    replica's position in an ensemble)."""
    g = torch.Generator(device=device)
    g.manual_seed((int(init_seed) * 1000003 + int(replica_seed)) & (2 ** 63 - 1))
    return init_sigma * torch.randn(n, dtype=torch.float64, device=device, generator=g)


def gamma_mle(first_steps, max_steps, volume, dt):
    """Exponential first-passage MLE with censoring: (Gamma, rel_err, n_events).

    first_steps: step of first passage (-1 if none by max_steps); volume: sites x dx^d."""
    fs = np.asarray(first_steps)
    ev = fs >= 0
    t = np.where(ev, fs + 1, max_steps) * dt
    n = int(ev.sum())
    total = float(volume) * float(t.sum())
    gam = n / total if total > 0 else float("nan")
    return gam, (1.0 / math.sqrt(n) if n else float("inf")), n


def plain_first_passage(specs, max_steps, *, storage="f32c", dt=0.05, dx=1.0, eta=1.0,
                        thr=1.0, stop_frac=0.5, check_every=10, init_sigma=0.01, init_seed=0,
                        device="cuda", timing=None):
    """The per-replica baseline: each replica alone through the single-lattice driver
    (marching kernel where the shape allows, graph-captured check intervals, a host poll
    per check).  Same arithmetic, noise and initial state as the batched ensemble, so
    the first-passage steps agree exactly.  Returns first-passage steps (-1 = none).
    ``timing`` (a dict) receives the seconds spent in setup (state upload, first graph
    capture) and in stepping, separately."""
    import time
    from .driver import Simulation, constant_temperature
    K = max(2, check_every & ~1)
    out = []
    if timing is not None:
        timing.setdefault("setup_s", 0.0)
        timing.setdefault("run_s", 0.0)
    for sp in specs:
        t0 = time.perf_counter()
        shape = _canonical(sp.shape)
        n = shape[0] * shape[1] * shape[2]
        phi0 = replica_initial_phi(n, sp.seed, init_seed, init_sigma, device)
        sim = Simulation(shape, storage=storage, dt=dt, dx=dx, eta=eta, table=None,
                         vpoly=toy_coefficients(sp.T, sp.E, sp.D, sp.lam, sp.T0),
                         schedule=constant_temperature(sp.T, 1, dt=dt, eta=eta, dx_phys=dx),
                         seed=sp.seed, phi0=phi0.reshape(shape).cpu().numpy(),
                         obs_threshold=thr, graph_steps=K, device=device)
        if timing is not None:
            sim.prepare_graphs(K)
            torch.cuda.synchronize(device)
            t1 = time.perf_counter()
            timing["setup_s"] += t1 - t0
        out.append(sim.run_until(stop_frac, max_steps, check_every=K))
        if timing is not None:
            torch.cuda.synchronize(device)
            timing["run_s"] += time.perf_counter() - t1
    return np.array(out)
