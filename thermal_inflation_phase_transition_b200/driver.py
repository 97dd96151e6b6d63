"""Host step driver: the reference's per-step loop (R:3619-3880) on the GPU.

The reference recomputes T(t), the noise amplitude and the table on the host
every step and calls one numba kernel.  Here the per-step scalars for the whole
run are computed once in FP64 on the host (``schedule``), uploaded, and read by
the kernels through a device step counter, so a chunk of K steps (each step a
fused midpoint launch, optionally followed by the observables reduction) is
captured once into a CUDA graph and replayed; the graph ends by advancing the
counter.  No host synchronisation happens inside a chunk.

    sim = Simulation((256, 256, 1), storage="f64", table=Table1D(...),
                     schedule=constant_temperature(1.02, 2000, dt=0.05))
    history = sim.run(2000)          # (2000, 10) observables, FP64, on the host
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib as L
from ._common import poly_source, ptr, step_params, stream_handle, table_source
from .observables import OBS_INDEX, OBS_NAMES, workspace_bytes
from .real_field import to_f32c

__all__ = ["Table1D", "Table2D", "Simulation", "constant_temperature", "linear_cooling",
           "hubble_expansion", "hubble_param", "toy_vprime", "OBS_NAMES", "OBS_INDEX",
           "G_STAR", "M_PL", "DEL_V"]

# The reference's expanding background (R:424-427): SM relativistic degrees of
# freedom, reduced Planck mass (GeV), vacuum energy of the inflation background (GeV^4).
G_STAR = 106.75
M_PL = 2.4e18
DEL_V = 1e36 / 4


def toy_vprime(phi, T, D=0.1, E=0.05, lam=0.1, T0=1.0):
    """V'(phi) of V = D(T^2-T0^2) phi^2 - E T phi^3 + (lam/4) phi^4."""
    phi = np.asarray(phi, np.float64)
    return 2.0 * D * (T * T - T0 * T0) * phi - 3.0 * E * T * phi * phi + lam * phi ** 3


@dataclass
class Table1D:
    """Uniform V' table at one temperature (R:840-849 build_vprime_table)."""
    values: np.ndarray
    tmin: float
    dinv: float

    @classmethod
    def build(cls, fn, T, lo, hi, n):
        x = np.linspace(lo, hi, n, dtype=np.float64)
        return cls(np.ascontiguousarray(fn(x, T), np.float64), float(lo),
                   1.0 / ((hi - lo) / (n - 1)))


@dataclass
class Table2D:
    """V'(phi, T) on a uniform (T, phi) grid, rows blended at the step's T."""
    values: np.ndarray  # [nT][nphi]
    tmin: float
    dinv: float
    T_min: float
    T_dinv: float

    @classmethod
    def build(cls, fn, lo, hi, n_phi, T_lo, T_hi, n_T):
        x = np.linspace(lo, hi, n_phi, dtype=np.float64)
        Ts = np.linspace(T_lo, T_hi, n_T, dtype=np.float64)
        v = np.stack([fn(x, T) for T in Ts]).astype(np.float64)
        return cls(np.ascontiguousarray(v), float(lo), 1.0 / ((hi - lo) / (n_phi - 1)),
                   float(T_lo), 1.0 / ((T_hi - T_lo) / (n_T - 1)))


def noise_amplitude(T, eta, dt, dx_phys=1.0, mu=1.0, a=1.0):
    """ns = sqrt(2 eta T dt a^-3 / (mu^2 dx_phys^3))  (R:3714-3718)."""
    return math.sqrt(max(2.0 * eta * T * dt / (a ** 3) / (mu * mu * dx_phys ** 3), 0.0))


def constant_temperature(T, n_steps, *, dt, eta=1.0, dx_phys=1.0, mu=1.0, noise=True):
    """(n_steps, 2) schedule of (T, ns) at fixed T (the reference's --no_hubble run)."""
    ns = noise_amplitude(T, eta, dt, dx_phys, mu) if noise else 0.0
    return np.tile(np.array([[T, ns]], np.float64), (n_steps, 1))


def linear_cooling(T_start, T_end, n_cool, n_steps, *, dt, eta=1.0, dx_phys=1.0, mu=1.0,
                   noise=True):
    """T(t) = max(T_start - rate t, 0) with rate = (T_start - T_end)/(n_cool dt)
    (the temperature(t) form of R:2828-2829), t = n dt."""
    rate = (T_start - T_end) / (n_cool * dt)
    n = np.arange(n_steps, dtype=np.float64)
    T = np.maximum(T_start - rate * (n * dt), 0.0)
    ns = np.array([noise_amplitude(t, eta, dt, dx_phys, mu) if noise else 0.0 for t in T])
    return np.ascontiguousarray(np.stack([T, ns], axis=1), np.float64)


def hubble_param(T, g_star=G_STAR, m_pl=M_PL, del_v=DEL_V):
    """H(T) = sqrt((T^4 g* pi^2 / 30 + del_V) / (3 M_pl^2)) in GeV (R:706-710, the
    form the step loop evaluates, R:3625)."""
    T4 = T * T * T * T
    return math.sqrt((T4 * (g_star * math.pi ** 2 / 30.0) + del_v) * (1.0 / (3.0 * m_pl ** 2)))


def hubble_expansion(T0, n_steps, *, dt, eta, mu, dx_phys=1.0, scale_factor=True, noise=True,
                     a0=1.0, g_star=G_STAR, m_pl=M_PL, del_v=DEL_V):
    """(n_steps, 4) schedule of (T, ns, eta_eff, inv_a2) on the reference's expanding
    background (R:3621-3636, noise amplitude R:3714-3718): at step n, T = T0 / a,
    H = H(T), eta_eff = eta + 3H/mu and inv_a2 = 1/a^2 (eta_eff = eta, inv_a2 =
    inv_a3 = 1 when ``scale_factor`` is False, the reference's --no_scale_factor),
    ns = sqrt(2 eta_eff T dt inv_a3 / (mu^2 dx_phys^3)); then a += a H dt / mu.
    Returns the schedule and the scale factor after the last step."""
    out = np.empty((n_steps, 4), np.float64)
    chig = g_star * math.pi ** 2 / 30.0
    inv3 = 1.0 / (3.0 * m_pl ** 2)
    a = float(a0)
    for n in range(n_steps):
        T = T0 / a
        T4 = T * T * T * T
        H = math.sqrt((T4 * chig + del_v) * inv3)
        if scale_factor:
            eta_eff, inv_a2, inv_a3 = eta + 3.0 * H / mu, 1.0 / (a * a), 1.0 / (a * a * a)
        else:
            eta_eff, inv_a2, inv_a3 = eta, 1.0, 1.0
        ns = math.sqrt(2.0 * eta_eff * T * dt * inv_a3 / (mu ** 2 * dx_phys ** 3)) if noise else 0.0
        out[n] = (T, ns, eta_eff, inv_a2)
        a += a * H * (dt / mu)
    return out, a


class Simulation:
    """A real scalar field on a periodic lattice, stepped by graph-captured chunks.

    storage: "f64", "f32" (the reference's float32 mode) or "f32c" (compensated).
    table: Table1D / Table2D, or None with vpoly = (c1, c2, c3) for the polynomial
    V'(phi) = c1 phi + c2 phi^2 + c3 phi^3.
    schedule: (n, 2) rows (T, ns) per step, or (n, 4) rows (T, ns, eta_eff, inv_a2)
    for an expanding background (``hubble_expansion``); the observables' gradient
    energy uses the constructor's inv_a2.
    phi0/pi0: initial fields (numpy, FP64); default phi ~ N(0, init_sigma^2), pi = 0.
    """

    def __init__(self, shape, *, storage="f32c", dt=0.05, dx=1.0, eta=1.0, mu=1.0, inv_a2=1.0,
                 table, schedule, seed=0, phi0=None, pi0=None, init_sigma=0.01, init_seed=0,
                 obs_threshold=1.0, graph_steps=50, vpoly=None, device="cuda"):
        self.shape = tuple(int(x) for x in shape)
        self.storage = storage
        self.dev = torch.device(device)
        self.dt, self.dx, self.eta, self.mu, self.inv_a2 = dt, dx, eta, mu, inv_a2
        self.seed = seed
        self.thr = obs_threshold
        self.graph_steps = max(2, graph_steps + (graph_steps & 1))  # even: state ends in buffer 0
        self.schedule = np.ascontiguousarray(schedule, np.float64)
        if self.schedule.ndim != 2 or self.schedule.shape[1] not in (2, 4):
            raise ValueError("schedule must be (n_steps, 2) (T, ns) or (n_steps, 4) "
                             "(T, ns, eta_eff, inv_a2) per step")
        self._sched_fn = ("tipt_rk2_step_table_sched" if self.schedule.shape[1] == 2
                          else "tipt_rk2_step_table_sched4")
        self._sched = torch.from_numpy(self.schedule).to(self.dev)
        if table is None:
            if vpoly is None:
                raise ValueError("give a table or vpoly")
            self._table = None
            self._vs = poly_source(*vpoly)
        elif isinstance(table, Table2D):
            self._table = torch.from_numpy(np.asarray(table.values)).to(self.dev)
            self._vs = table_source(self._table, table.tmin, table.dinv, table.values.shape[1],
                                    float(self.schedule[0, 0]), table.T_min, table.T_dinv)
        else:
            self._table = torch.from_numpy(np.asarray(table.values)).to(self.dev)
            self._vs = table_source(self._table, table.tmin, table.dinv, table.values.shape[0])
        if phi0 is None:
            phi0 = np.random.default_rng(init_seed).normal(0.0, init_sigma, self.shape)
        if pi0 is None:
            pi0 = np.zeros(self.shape)
        self.phi = [self._to_storage(phi0), None]
        self.pi = [self._to_storage(pi0), None]
        self.phi[1] = torch.empty_like(self.phi[0])
        self.pi[1] = torch.empty_like(self.pi[0])
        self._counter = torch.zeros(1, dtype=torch.int64, device=self.dev)
        self._ws = torch.empty(workspace_bytes(self.shape) // 8 + 1, dtype=torch.float64,
                               device=self.dev)
        self._sp = step_params(dt, dx, eta, mu, inv_a2, 0.0, 0, seed)
        self.steps_done = 0
        self._graphs = {}

    # ------------------------------------------------------------- state
    def _to_storage(self, a):
        t = torch.from_numpy(np.ascontiguousarray(a, np.float64)).to(self.dev)
        if self.storage == "f64":
            return t
        if self.storage == "f32":
            return t.to(torch.float32).contiguous()
        if self.storage == "f32c":
            return to_f32c(t)
        raise ValueError(f"unknown storage {self.storage}")

    def fields(self):
        """Current (phi, pi) as FP64 CUDA tensors."""
        def f64(t):
            if self.storage == "f32c":
                return t[0].double() + t[1].double()
            return t.double()
        return f64(self.phi[0]), f64(self.pi[0])

    # ------------------------------------------------------- checkpoints
    def snapshot(self, writer, *, energy_params=None):
        """Save the current state through a ``snapshots.SnapshotWriter`` in the
        reference's layout (R:3997-4018): labelled with the index n of the last step
        applied, time n dt, and that step's T; ``pi`` on the writer's checkpoint
        cadence.  ``energy_params = (lam, mphi)`` adds E_kin, E_grad, E_pot."""
        n = self.steps_done - 1
        T = float(self.schedule[min(max(n, 0), self.schedule.shape[0] - 1), 0])
        en = None
        if energy_params is not None:
            from .observables import observables
            lam, mphi = energy_params
            o = observables(self.phi[0], self.pi[0], dx=self.dx, inv_a2=self.inv_a2, lam=lam,
                            mphi=mphi, mu=self.mu).tolist()
            en = (o[0], o[1], o[2])
        return writer.save_real(n, n * self.dt, T, self.phi[0], self.pi[0], energies=en)

    def resume(self, ckpt):
        """Continue from a checkpoint (the dict of ``snapshots.latest_checkpoint``): the
        fields are copied into the current buffers (captured graphs stay valid) and the
        next step is the one after the saved step.  (The reference restarts its loop at
        the saved step index, applying that step a second time.)"""
        from .snapshots import load_fields
        phi, pi = load_fields(ckpt, ["phi", "pi"], self.storage, self.dev)
        self.phi[0].copy_(phi.reshape(self.phi[0].shape))
        self.pi[0].copy_(pi.reshape(self.pi[0].shape))
        self.steps_done = int(ckpt["step"]) + 1
        self._counter.fill_(self.steps_done)

    # ------------------------------------------------------------ stepping
    def _st(self):
        return {"f64": L.TIPT_F64, "f32": L.TIPT_F32, "f32c": L.TIPT_F32C}[self.storage]

    def _launch_chunk(self, K, obs, observe_last=False):
        """Enqueue K steps (+ observables into obs[q], or only after the last step into
        obs[0] with observe_last) and the counter advance."""
        lib = L.lib()
        st = stream_handle()
        nx, ny, nz = self.shape
        for q in range(K):
            a, b = q & 1, (q + 1) & 1
            rc = getattr(lib, self._sched_fn)(
                self._st(), ptr(self.phi[a]), ptr(self.pi[a]), ptr(self.phi[b]), ptr(self.pi[b]),
                nx, ny, nz, self._sp, self._vs, ptr(self._sched), self.schedule.shape[0],
                ptr(self._counter), q, st)
            L.check(rc, self._sched_fn)
            if obs is not None and (not observe_last or q == K - 1):
                rc = lib.tipt_observables(self._st(), ptr(self.phi[b]), ptr(self.pi[b]), nx, ny,
                                          nz, float(self.dx), float(self.inv_a2), 0.0, 0.0,
                                          float(self.mu), float(self.thr),
                                          ptr(obs[0 if observe_last else q]), ptr(self._ws),
                                          self._ws.numel() * 8, st)
                L.check(rc, "tipt_observables")
        L.check(lib.tipt_counter_add(ptr(self._counter), K, st), "tipt_counter_add")

    def _graph(self, K, observe):
        # a graph bakes the buffer pointers: an odd eager remainder exchanges the
        # two buffers, so the graph is keyed by which buffer holds the state
        key = (K, observe, self.phi[0].data_ptr())
        if key not in self._graphs:
            obs = torch.zeros((K, 10), dtype=torch.float64, device=self.dev) if observe else None
            s = torch.cuda.Stream()
            s.wait_stream(torch.cuda.current_stream())
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=s):
                self._launch_chunk(K, obs)
            torch.cuda.current_stream().wait_stream(s)
            self._graphs[key] = (g, obs)
        return self._graphs[key]

    def run(self, n_steps, *, observe=True, use_graphs=True):
        """Advance n_steps; returns the per-step observables (n_steps, 10) on the host
        (None if observe=False).  Steps beyond the schedule reuse its last (T, ns)."""
        K = self.graph_steps
        out = []
        done = 0
        while done < n_steps:
            k = min(K, n_steps - done)
            if use_graphs and k == K:
                g, obs = self._graph(K, observe)
                g.replay()
                if observe:
                    out.append(obs.clone())
            else:
                # remainder (or graphs off): eager launches in pairs keep the
                # state in buffer 0; an odd final step is followed by a swap
                obs = torch.zeros((k, 10), dtype=torch.float64, device=self.dev) if observe else None
                self._launch_chunk(k, obs)
                if k & 1:
                    self.phi.reverse()
                    self.pi.reverse()
                if observe:
                    out.append(obs)
            done += k
        self.steps_done += n_steps
        if not observe:
            return None
        return torch.cat(out).cpu().numpy()

    def run_until(self, stop_frac, max_steps, *, check_every=None):
        """Step in graph-captured chunks of check_every steps; after each chunk read the
        fraction of sites with phi > obs_threshold on the host and stop once it exceeds
        stop_frac.  Returns the 0-based index of that chunk's last step, or -1."""
        K = self.graph_steps if check_every is None else max(2, check_every & ~1)
        if K != self.graph_steps:
            self.graph_steps = K
            self._graphs = {}
        k_frac = OBS_INDEX["frac_above"]
        while self.steps_done + K <= max_steps:
            obs = self._run_chunk_observe_last(K)
            self.steps_done += K
            if float(obs[k_frac]) > stop_frac:
                return self.steps_done - 1
        return -1

    def prepare_graphs(self, K):
        """Capture (without running) the check-interval graph run_until replays."""
        self._last_graph(K)

    def _last_graph(self, K):
        key = ("last", K, self.phi[0].data_ptr())
        if key not in self._graphs:
            obs = torch.zeros((1, 10), dtype=torch.float64, device=self.dev)
            s = torch.cuda.Stream()
            s.wait_stream(torch.cuda.current_stream())
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=s):
                self._launch_chunk(K, obs, observe_last=True)
            torch.cuda.current_stream().wait_stream(s)
            self._graphs[key] = (g, obs)
        return self._graphs[key]

    def _run_chunk_observe_last(self, K):
        g, obs = self._last_graph(K)
        g.replay()
        return obs[0].cpu().numpy()

    def synchronize(self):
        torch.cuda.synchronize(self.dev)
