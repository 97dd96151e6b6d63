"""Command-line run of the complex-field (U(1) / Z_N) simulation with the reference
script's flags.

    python -m thermal_inflation_phase_transition_b200.run_complex --Nx 64 --Ny 64 --Nz 64 \\
        --Nt 2000 --steps 500 --zn_order 4 --zn_strength 1e11 --out runs

Mirrors simulation/latticeSimComplex_numba.py (C) end to end on this package's
GPU kernels: its command line (C:21-158, same names and defaults), the physical
setup (C:631-713: dx_phys = 1e-3, dt_phys = 2.5e-4 dt_factor, eta_phys = 1000,
lam = 1e-16, mu = mphi), the first-order integrator chosen automatically when
eta_phys exceeds 100 and no --integrator is given (C:654-669), _POT_COEFFS from
--potential_type (C:205-221), Z_N from --zn_order / --zn_strength with the
turn-on below --zn_turn_on_T (C:226-231, C:4254-4261), the initial state
r = init_rho |N(0, 1)|, theta uniform, pi = 0 (C:1272-1279), the expanding
background (always on, C:422; T = T0 / a, eta_eff = eta + 3H/mu, inv_a2 = 1/a^2,
noise amplitude without the a^-3 factor, C:4240-4249), the V'(rho) table rebuilt
when T drifts by 1e-4 or rho leaves its range (C:4263-4288), the --integrator
dispatch, the NaN / divergence guard (C:4540-4582), snapshots with rho, theta and
the plaquette windings in the reference's npz layout (C:4584-4654), --resume,
replay mode and simulation_metadata.npz (C:4757-4790).

Differences, by design: the Z_N turn-on reaches the kernels (the reference
writes its flag into a global that its compiled kernels froze at their first
compile, so there Z_N never turns on at run time); the two noise fields of a
step are the cos and sin members of one hash pair per site (the reference seeds
its second field with n + 1, the seed of the next step's first field); a resumed
or replayed run continues with the step after the checkpoint's; hash noise in
place of the per-thread Mersenne Twister; no figures; no bubble seeding.
"""
from __future__ import annotations

import argparse
import math
import os
import sys
import time

import numpy as np
import torch

from . import complex_field as CF
from . import real_field as RF
from .driver import DEL_V, G_STAR, M_PL
from .run import CHECKPOINT_EVERY, INTEGRATORS, RECORDED_NAME, TABLE_MARGIN_FRAC, TABLE_SIZE
from .run import _replay_params
from .snapshots import SnapshotWriter, latest_checkpoint, load_fields, write_metadata
from .thermal import ThermalPotential

PARAM_SET = "set6"              # C:3354
OVERDAMPED_AUTO_THRESHOLD = 100.0   # C:343
FIELDS = ("phi1", "phi2", "pi1", "pi2")


def build_parser():
    ap = argparse.ArgumentParser(description="Complex lattice field simulation (GPU)")
    ap.add_argument("--Nx", type=int, default=256)
    ap.add_argument("--Ny", type=int, default=256)
    ap.add_argument("--Nz", type=int, default=256)
    ap.add_argument("--Nt", type=int, default=100_000_000)
    ap.add_argument("--T0", type=float, default=7350.0)
    ap.add_argument("--steps", type=int, default=100_000)
    ap.add_argument("--resume", action="store_true")
    ap.add_argument("--dt_factor", type=float, default=1.0)
    ap.add_argument("--replay_dir", type=str, default=None)
    ap.add_argument("--start_step", type=int, default=None)
    ap.add_argument("--replay_steps", type=int, default=3000)
    ap.add_argument("--replay_save_every", type=int, default=10)
    ap.add_argument("--integrator", type=str, default=None, choices=INTEGRATORS)
    ap.add_argument("--phi_threshold", type=float, default=None)
    ap.add_argument("--steps_dense", type=int, default=None)
    ap.add_argument("--boson_coupling", type=float, default=None)
    ap.add_argument("--fermion_coupling", type=float, default=None)
    ap.add_argument("--counterterm", action="store_true")
    ap.add_argument("--potential_type", type=str, default="V_p",
                    choices=["V_p", "V_correct", "fermion_only"])
    ap.add_argument("--zn_order", type=int, default=0)
    ap.add_argument("--zn_strength", type=float, default=0.0)
    ap.add_argument("--zn_turn_on_T", type=float, default=0.0)
    ap.add_argument("--init_rho", type=float, default=0.01)
    # this package's own options
    ap.add_argument("--out", type=str, default="data/lattice")
    ap.add_argument("--storage", type=str, default="f32", choices=["f32", "f64", "f32c"])
    ap.add_argument("--init_seed", type=int, default=0)
    ap.add_argument("--range_check_every", type=int, default=1)
    ap.add_argument("--device", type=str, default="cuda")
    ap.add_argument("--quiet", action="store_true")
    return ap


def pot_coeffs(potential_type):
    """C:205-221: V_p (2, -1), V_correct (1, 1), fermion_only (0, 1)."""
    return {"V_p": (2.0, -1.0), "V_correct": (1.0, 1.0), "fermion_only": (0.0, 1.0)}[
        potential_type]


def integrator_of(args, eta_phys):
    """The integrator the script runs: --integrator, or the first-order one when
    eta_phys exceeds the threshold (C:654-669), else rk2_nonfused."""
    if args.integrator is not None:
        return args.integrator
    return "overdamped" if eta_phys > OVERDAMPED_AUTO_THRESHOLD else "rk2_nonfused"


class ComplexRun:
    """The complex script's state and step loop."""

    def __init__(self, args):
        self.args = args
        self.log = (lambda *a: None) if args.quiet else print
        self.replay = args.replay_dir is not None
        self.dx_phys, self.dt_phys = 1e-3, 2.5e-4 * args.dt_factor       # C:633-634
        self.eta_phys = 1000.0                                          # C:642
        if self.replay:
            if args.start_step is None:
                raise SystemExit("--start_step is required in replay mode")
            self.dx_phys, self.dt_phys, self.eta_phys, _ = _replay_params(args)
        self.shape = (args.Nx, args.Ny, args.Nz)
        self.lam, self.mphi = 1e-16, 1000.0                              # C:638-639
        self.T0 = args.T0
        self.mu = self.mphi
        self.dx, self.dt = self.mu * self.dx_phys, self.mu * self.dt_phys
        self.eta = self.eta_phys / self.mu
        self.cooling_rate = 1.0 / self.mu
        self.bms, self.gb, self.gbg, self.gf, self.gfg = 1.0e6, 1.09, 1.05, 1.09, 1.05
        if args.boson_coupling is not None:
            self.gb = args.boson_coupling
        if args.fermion_coupling is not None:
            self.gf = args.fermion_coupling
        self.integrator = integrator_of(args, self.eta_phys)
        self.name = RECORDED_NAME[self.integrator]
        self.uses_table = self.integrator in ("baoab", "rk2_nonfused", "rk2_fused_table",
                                              "overdamped")
        self.overdamped = self.integrator == "overdamped"
        # Z_N: (N, delta_V, active); active from the start unless a turn-on T is given
        self.zn = [float(args.zn_order), float(args.zn_strength),
                   1.0 if args.zn_order > 0 and args.zn_turn_on_T <= 0.0 else 0.0]
        self.dev = torch.device(args.device)
        self.tp = ThermalPotential(lam=self.lam, mphi=self.mphi, bosonMassSquared=self.bms,
                                   bosonCoupling=self.gb, bosonGaugeCoupling=self.gbg,
                                   fermionCoupling=self.gf, fermionGaugeCoupling=self.gfg,
                                   pot_coeffs=pot_coeffs(args.potential_type),
                                   counterterm=(self.dx_phys, self.T0) if args.counterterm
                                   else None, device=self.dev)
        self.Nt, self.steps = args.Nt, args.steps
        self.n_start, self.n_origin, self.a = 0, 0, 1.0
        self._paths()

    def _paths(self):
        a = self.args
        if self.replay:
            end = a.start_step + a.replay_steps
            self.save_path = os.path.join(a.replay_dir,
                                          f"detailed_replay/step_{a.start_step}_to_{end}")
            self.Nt, self.steps = end, a.replay_save_every
        else:
            tag = (f"{a.Nx}x{a.Ny}x{a.Nz}_T0_{int(self.T0)}_complex"
                   f"{'_ZN' + str(a.zn_order) if a.zn_order > 0 else ''}"
                   f"_dx_{self.dx_phys:g}_dtphys_{self.dt_phys:g}_interval_{self.steps}_3D_hubble"
                   f"_eta_{self.eta_phys:g}_gb_{self.gb:g}_gf_{self.gf:g}"
                   f"{'_OD' if self.overdamped else ''}_{self.name}"
                   f"{'_CT' if a.counterterm else ''}"
                   f"{'_' + a.potential_type if a.potential_type != 'V_p' else ''}")
            self.save_path = os.path.join(a.out, PARAM_SET, tag)
        self.state_path = os.path.join(self.save_path, "field_states")

    # ------------------------------------------------------------ state ---
    def _field(self, x):
        t = torch.from_numpy(np.ascontiguousarray(x, np.float64)).to(self.dev)
        if self.args.storage == "f64":
            return t
        if self.args.storage == "f32":
            return t.float().contiguous()
        return RF.to_f32c(t)

    def _v(self, t):
        return (RF.from_f32c(t) if t.dim() == 4 else t).double()

    def _rho_max(self):
        """max |Phi|: from the previous step's fused range when it has one
        (rk2_nonfused), else a reduction."""
        if getattr(self, "rrange", None) is not None and self._range_valid:
            return RF.PhiRange.decode(self.rrange.last.cpu().numpy())[1]
        p1, p2 = self._v(self.st[0]), self._v(self.st[1])
        return float(torch.sqrt(p1 * p1 + p2 * p2).max())

    def init_state(self):
        a = self.args
        if self.replay:
            f = os.path.join(a.replay_dir, "field_states", f"state_step_{a.start_step:010d}.npz")
            if not os.path.exists(f):
                raise SystemExit(f"checkpoint file not found: {f}")
            with np.load(f) as z:
                d = {k: z[k] for k in z.files}
            names = ["phi1", "phi2"] + ([] if self.overdamped else ["pi1", "pi2"])
            if any(k not in d or np.isnan(d[k]).any() for k in names):
                raise SystemExit(f"checkpoint {f} lacks pi or contains NaN")
            self._load(d, a.start_step)
            return
        rng = np.random.default_rng(a.init_seed)
        th = 2.0 * np.pi * rng.random(self.shape)                        # C:1273-1276
        r = a.init_rho * np.abs(rng.standard_normal(self.shape))
        zero = np.zeros(self.shape)
        self.st = [self._field(r * np.cos(th)), self._field(r * np.sin(th)), self._field(zero),
                   self._field(zero)]
        if a.resume:
            f, d = latest_checkpoint(self.state_path, need_pi=not self.overdamped,
                                     keys=("phi1", "phi2"), pi_keys=("pi1", "pi2"))
            if d is not None:
                self.log(f"resuming from {f} (step {int(d['step'])})")
                self._load(d, int(d["step"]))

    def _load(self, d, step):
        names = ["phi1", "phi2"] + ([] if self.overdamped else ["pi1", "pi2"])
        got = load_fields(d, names, self.args.storage, self.dev)
        shp = ((2,) + self.shape) if self.args.storage == "f32c" else self.shape
        self.st = [g.reshape(shp) for g in got]
        while len(self.st) < 4:
            self.st.append(self._field(np.zeros(self.shape)))
        self.n_start, self.n_origin = step + 1, step
        if "scale_factor" in d:
            self.a = float(d["scale_factor"])
        if "zn_active" in d:
            self.zn[2] = max(self.zn[2], float(d["zn_active"]))

    # ------------------------------------------------------------ table ---
    def _rebuild(self, T, T_mid):
        hi = self._rho_max()
        margin = max(max(hi, 1.0) * TABLE_MARGIN_FRAC, 20000.0)
        lo, hi = 0.0, hi + margin                                        # C:4279-4280
        self.tab = self.tp.table(T, lo, hi, TABLE_SIZE)
        self.tab_mid = self.tp.table(T_mid, lo, hi, TABLE_SIZE)
        self.t_hi, self.T_last = hi, T

    def _need_rebuild(self, n, T):
        if self.tab is None or abs(T - self.T_last) / max(abs(T), 1.0) > 1e-4:
            return True
        if (n - self.n_start) % self.args.range_check_every:
            return False
        return self._rho_max() > self.t_hi

    # ------------------------------------------------------------- loop ---
    def scalars(self, n):
        """T, T_mid, eta_eff, inv_a2, H of step n; advances a (C:4240-4249)."""
        T = self.T0 / self.a
        T4 = T * T * T * T
        H = math.sqrt((T4 * (G_STAR * np.pi ** 2 / 30.0) + DEL_V) * (1.0 / (3.0 * M_PL ** 2)))
        eta_eff = self.eta + 3.0 * H / self.mu
        inv_a2 = 1.0 / (self.a * self.a)
        self.a += self.a * H * (self.dt / self.mu)
        return T, self.T0 / self.a, eta_eff, inv_a2, H

    def step(self, n, T, T_mid, eta_eff, inv_a2):
        dt, dx, mu, st = self.dt, self.dx, self.mu, self.st
        zn = tuple(self.zn)
        c = (self.lam, self.mphi, self.bms, self.gb, self.gbg, self.gf, self.gfg)
        tab = self.tab + (TABLE_SIZE,) if self.uses_table else None
        if self.integrator == "overdamped":                               # C:4290-4301
            ns = math.sqrt(2.0 * T * dt / (eta_eff * mu ** 2 * self.dx_phys ** 3))
            CF.overdamped_euler_step_table(st[0], st[1], dt, dx, eta_eff, mu, inv_a2, *tab, ns,
                                           n, tmp=self.mid[:2], zn=zn)
            return
        if self.integrator == "baoab":                                    # C:4302-4322
            ns = math.sqrt(T / (mu ** 2 * self.dx_phys ** 3))
            CF.baoab_step_table(*st, dt, dx, eta_eff, mu, inv_a2, *tab, ns, n, tmp=self.mid,
                                zn=zn)
            return
        ns = math.sqrt(2.0 * eta_eff * T * dt / (mu ** 2 * self.dx_phys ** 3))
        if self.integrator == "rk2_fused_inline":
            CF.rk2_fused_single_pass(*st, dt, dx, eta_eff, T, T_mid, mu, *c, ns, n, *self.mid,
                                     inv_a2, zn=zn, splines=self.tp)
            return
        n1, n2 = self.noise
        RF.generate_noise_field(n1, ns, n, component=0)
        RF.generate_noise_field(n2, ns, n, component=1)
        if self.integrator == "rk2_nonfused":
            CF.rk2_step_table(*st, dt, dx, eta_eff, mu, n1, n2, *self.mid, inv_a2, *tab, zn=zn,
                              rho_range=self.rrange)
            self._range_valid = True
        elif self.integrator == "rk2_nonfused_inline":
            CF.rk2_step_inline(*st, dt, dx, eta_eff, T, mu, *c, n1, n2, *self.mid, inv_a2, zn=zn,
                               splines=self.tp)
        elif self.integrator == "rk2_fused_table":
            CF.rk2_fused_table(*st, dt, dx, eta_eff, mu, n1, n2, *self.mid, inv_a2, *tab,
                               *self.tab_mid, TABLE_SIZE, zn=zn)
        elif self.integrator == "rk2_fused":
            CF.rk2_step_fused(*st, dt, dx, eta_eff, T, T_mid, mu, *c, n1, n2, None, None, None,
                              None, *self.mid, inv_a2, zn=zn, splines=self.tp)
        else:                                                             # "rk2"
            h1, h2 = n1 * 0.5, n2 * 0.5
            for TT in (T, T_mid):
                CF.rk2_step(*st, 0.5 * dt, dx, eta_eff, TT, mu, *c, h1, h2, None, None, None,
                            None, *self.mid, inv_a2, zn=zn, splines=self.tp)

    def _finite_and_bounded(self):
        names = 2 if self.overdamped else 4
        ok = all(bool(torch.isfinite(t).all()) for t in self.st[:names])
        return ok and self._rho_max() <= 1e6                             # C:4555

    def run(self):
        a = self.args
        self.init_state()
        os.makedirs(self.state_path, exist_ok=True)
        self.mid = [torch.empty_like(t) for t in self.st]
        ndt = torch.float32 if a.storage == "f32" else torch.float64
        self.noise = [torch.empty(self.shape, dtype=ndt, device=self.dev) for _ in range(2)]
        self.tab = None
        # the default RK2 step folds |Phi|'s range as it writes (the table check)
        self.rrange = RF.PhiRange(self.dev) if self.integrator == "rk2_nonfused" else None
        self._range_valid = False
        writer = SnapshotWriter(self.state_path, checkpoint_every=CHECKPOINT_EVERY)
        dense_on = a.phi_threshold is not None and a.steps_dense is not None
        dense_active = False
        nan_every = 1000 if self.replay else 100000
        t_start = time.time()
        self.status = "completed"
        for n in range(self.n_start, self.Nt):
            t = n * self.dt
            T, T_mid, eta_eff, inv_a2, H = self.scalars(n)
            if a.zn_order > 0 and a.zn_turn_on_T > 0.0 and T < a.zn_turn_on_T and self.zn[2] < 0.5:
                self.zn[2] = 1.0                                          # C:4254-4261
                self.log(f"Z_{a.zn_order} breaking activated at T={T:.1f}")
            if self.uses_table and self._need_rebuild(n, T):
                self._rebuild(T, T_mid)
            self.step(n, T, T_mid, eta_eff, inv_a2)
            if n % nan_every == 0 and not self._finite_and_bounded():
                path = os.path.join(self.state_path, f"state_step_{n:010d}_NaN_debug.npz")
                d = {f: self._v(x).cpu().numpy() for f, x in zip(FIELDS, self.st)}
                np.savez(path, step=n, time=t, temperature=T, eta_eff=eta_eff, inv_a2=inv_a2, **d)
                self.log(f"NaN/Inf or divergence at step {n}; state written to {path}")
                self.status = "diverged"
                break
            cur = self.steps
            if dense_on and not dense_active and self._rho_max() > a.phi_threshold:
                dense_active = True
            if dense_active:
                cur = a.steps_dense
            due = (n - self.n_origin) % cur == 0 if self.replay else n % cur == 0
            if due:
                pis = (None, None) if self.overdamped else (self.st[2], self.st[3])
                writer.save_complex(n, t, T, self.st[0], self.st[1], *pis, zn_active=self.zn[2],
                                    scale_factor=self.a, hubble=H)
                el = time.time() - t_start
                self.log(f"Step {n}/{self.Nt} | T={T:.1f} | a={self.a:.6f} | "
                         f"{(n - self.n_start + 1) / el if el > 0 else 0.0:.1f} steps/s")
        torch.cuda.synchronize(self.dev)
        writer.wait()
        self.total_time = time.time() - t_start
        write_metadata(self.save_path, Nx=a.Nx, Ny=a.Ny, Nz=a.Nz, dx_phys=self.dx_phys,
                       dt_phys=self.dt_phys, mphi=self.mphi, lam=self.lam,
                       eta_phys=self.eta_phys, T0=self.T0, cooling_rate=self.cooling_rate,
                       Nt=self.Nt, steps=self.steps, total_time=self.total_time, mu=self.mu,
                       dx=self.dx, dt=self.dt, eta=self.eta,
                       vev=np.sqrt(self.mphi ** 2 / self.lam), seed_bubbles=False,
                       bubble_config=np.array([]), bubble_profile="none", bubble_wall_width=0.0,
                       integrator=self.name, counterterm=a.counterterm,
                       potential_type=a.potential_type, field_type="complex",
                       zn_order=a.zn_order, zn_strength=a.zn_strength,
                       zn_turn_on_T=a.zn_turn_on_T, init_rho=a.init_rho)
        return self.status


def main(argv=None):
    r = ComplexRun(build_parser().parse_args(argv))
    status = r.run()
    r.log(f"{status}: {r.save_path}")
    return 0 if status == "completed" else 1


if __name__ == "__main__":
    sys.exit(main())
