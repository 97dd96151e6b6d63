"""Command-line run of the real-field simulation with the reference script's flags.

    python -m thermal_inflation_phase_transition_b200.run --Nx 64 --Ny 64 --Nz 64 \\
        --Nt 2000 --steps 500 --no_hubble --out runs

Mirrors simulation/latticeSimeRescale_numba.py (R) end to end on this package's
GPU kernels: its command line (R:21-170, same names and defaults), the physical
setup (R:633-669: mu = mphi, dx = mu dx_phys, dt = mu dt_phys, eta = T0 / mu),
the thermal potential (_POT_COEFFS from --potential_type and --nb / --nf,
R:226-241, --counterterm R:755-797), the initial state phi = 0.01 N(0, 1), pi = 0
(R:1259-1260), the step loop (R:3619-3944: expanding background with T = T0 / a,
eta_eff = eta + 3H/mu, inv_a2 = 1/a^2 unless --no_hubble / --no_scale_factor;
the V' table rebuilt when T drifts by 1e-4 or phi leaves its range; the
--integrator dispatch; the NaN guard), snapshots and checkpoints in the
reference's npz layout with the dense-interval switch (R:3945-4018), --resume
(R:2960-3010), replay mode (R:180-222, R:2890-2958) and simulation_metadata.npz
(R:4126-4167).

Differences, by design: a resumed or replayed run continues with the step after
the checkpoint's (the reference restarts its loop at the checkpoint's step and
applies that step a second time); the noise is the counter-based hash noise
(generate_noise_field) instead of numba's per-thread Mersenne Twister, which no
run reproduces; the table range test reads phi's minimum and maximum every
--range_check_every steps (1, the default, is the reference's every step); no
figures are drawn; bubble seeding (off in the reference, R:356) is not offered.
The output directory name follows R:2856-2877 under --out instead of data/lattice.
"""
from __future__ import annotations

import argparse
import math
import os
import re
import sys
import time

import numpy as np
import torch

from . import real_field as RF
from .driver import DEL_V, G_STAR, M_PL
from .snapshots import SnapshotWriter, latest_checkpoint, load_fields, write_metadata
from .thermal import ThermalPotential

INTEGRATORS = ["baoab", "rk2_nonfused", "rk2_fused", "rk2_fused_table", "rk2_fused_inline", "rk2",
               "overdamped", "rk2_nonfused_inline"]
# the name each --integrator choice records (R:2839-2854)
RECORDED_NAME = {None: "rk2_nonfused_table", "rk2_nonfused": "rk2_nonfused_table",
                 "baoab": "baoab", "rk2_nonfused_inline": "rk2_nonfused_inline",
                 "rk2_fused_table": "rk2_fused_table", "rk2_fused_inline": "rk2_fused_inline",
                 "rk2_fused": "rk2_fused", "rk2": "rk2", "overdamped": "overdamped"}
TABLE_SIZE = 16384          # R:308
TABLE_MARGIN_FRAC = 1.0     # R:3604
CHECKPOINT_EVERY = 10       # R:395
PARAM_SET = "set8"          # R:2835


def build_parser():
    ap = argparse.ArgumentParser(description="Lattice scalar field simulation (GPU)")
    ap.add_argument("--Nx", type=int, default=256)
    ap.add_argument("--Ny", type=int, default=256)
    ap.add_argument("--Nz", type=int, default=256)
    ap.add_argument("--Nt", type=int, default=100_000_000)
    ap.add_argument("--T0", type=float, default=7350.0)
    ap.add_argument("--steps", type=int, default=100_000)
    ap.add_argument("--resume", action="store_true")
    ap.add_argument("--dt_factor", type=float, default=1.0,
                    help="accepted and reported; the reference does not apply it (R:639)")
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
    ap.add_argument("--potential_type", type=str, default="V_correct",
                    choices=["V_p", "V_correct", "fermion_only"])
    ap.add_argument("--no_scale_factor", action="store_true")
    ap.add_argument("--no_hubble", action="store_true")
    ap.add_argument("--diag_energy", action="store_true")
    ap.add_argument("--nb", type=int, default=20)
    ap.add_argument("--nf", type=int, default=20)
    ap.add_argument("--dx_phys", type=float, default=1e-3)
    ap.add_argument("--dt_phys", type=float, default=1e-4)
    # this package's own options
    ap.add_argument("--out", type=str, default="data/lattice",
                    help="root of the output directories (the reference's data/lattice)")
    ap.add_argument("--storage", type=str, default="f32", choices=["f32", "f64", "f32c"],
                    help="f32: the reference's float32 mode (R:348); f32c: compensated FP32")
    ap.add_argument("--init_seed", type=int, default=0, help="seed of the initial phi")
    ap.add_argument("--range_check_every", type=int, default=1)
    ap.add_argument("--device", type=str, default="cuda")
    ap.add_argument("--quiet", action="store_true")
    return ap


def pot_coeffs(potential_type, nb, nf):
    """R:226-241 as executed: V_correct and V_p both keep (1, 1), fermion_only
    (0, 1); then times (nb, nf)."""
    c = [1.0, 1.0]
    if potential_type == "fermion_only":
        c = [0.0, 1.0]
    return (c[0] * nb, c[1] * nf)


def _replay_params(args):
    """R:180-222: lattice and physical parameters of the run being replayed, from its
    simulation_metadata.npz or else from its directory name."""
    meta = os.path.join(args.replay_dir, "simulation_metadata.npz")
    if os.path.exists(meta):
        with np.load(meta) as m:
            args.Nx, args.Ny, args.Nz = int(m["Nx"]), int(m["Ny"]), int(m["Nz"])
            args.T0 = float(m["T0"])
            return float(m["dx_phys"]), float(m["dt_phys"]), float(m["eta_phys"]), True
    base = os.path.basename(args.replay_dir.rstrip("/"))
    mt = re.match(r"(\d+)x(\d+)x(\d+)_T0_(\d+)_dx_([\d.eE+-]+)_dtphys_([\d.eE+-]+)"
                  r"_interval_\d+_3D_(hubble|nohubble)_eta_([\d.eE+-]+)", base)
    if mt is None:
        raise SystemExit(f"cannot parse simulation parameters from directory name: {base}")
    args.Nx, args.Ny, args.Nz = int(mt.group(1)), int(mt.group(2)), int(mt.group(3))
    args.T0 = float(mt.group(4))
    return float(mt.group(5)), float(mt.group(6)), float(mt.group(8)), mt.group(7) == "hubble"


class Run:
    """The reference script's state and step loop."""

    def __init__(self, args):
        self.args = args
        self.log = (lambda *a: None) if args.quiet else print
        self.replay = args.replay_dir is not None
        eta_phys = None
        hubble = not args.no_hubble
        self.dx_phys, self.dt_phys = args.dx_phys, args.dt_phys
        if self.replay:
            if args.start_step is None:
                raise SystemExit("--start_step is required in replay mode")
            self.dx_phys, self.dt_phys, eta_phys, hubble = _replay_params(args)
        self.hubble = hubble
        self.shape = (args.Nx, args.Ny, args.Nz)
        self.lam, self.mphi = 1e-24, 1000.0                     # R:642-643
        self.T0 = args.T0
        self.eta_phys = args.T0 if eta_phys is None else eta_phys
        self.mu = self.mphi                                    # R:666
        self.dx = self.mu * self.dx_phys                       # R:668
        self.dt = self.mu * self.dt_phys                       # R:669
        self.eta = self.eta_phys / self.mu
        self.cooling_rate = 1.0 / self.mu
        self.bms, self.gb, self.gbg, self.gf, self.gfg = 1.0e6, 1.09, 1.05, 1.09, 1.05
        if args.boson_coupling is not None:
            self.gb = args.boson_coupling
        if args.fermion_coupling is not None:
            self.gf = args.fermion_coupling
        self.integrator = args.integrator or "rk2_nonfused"
        self.name = RECORDED_NAME[args.integrator]
        self.uses_table = self.integrator in ("baoab", "rk2_nonfused", "rk2_fused_table",
                                              "overdamped")
        self.overdamped = self.integrator == "overdamped"
        self.dev = torch.device(args.device)
        self.tp = ThermalPotential(lam=self.lam, mphi=self.mphi, bosonMassSquared=self.bms,
                                   bosonCoupling=self.gb, bosonGaugeCoupling=self.gbg,
                                   fermionCoupling=self.gf, fermionGaugeCoupling=self.gfg,
                                   pot_coeffs=pot_coeffs(args.potential_type, args.nb, args.nf),
                                   counterterm=(self.dx_phys, self.T0) if args.counterterm
                                   else None, device=self.dev)
        self.Nt, self.steps = args.Nt, args.steps
        self.n_start = 0
        self.n_origin = 0       # replay saves every --replay_save_every steps after this one
        self.a = 1.0
        self._paths()

    # ------------------------------------------------------------ paths ---
    def _paths(self):
        a = self.args
        if self.replay:
            end = a.start_step + a.replay_steps
            self.save_path = os.path.join(a.replay_dir,
                                          f"detailed_replay/step_{a.start_step}_to_{end}")
            self.Nt = end
            self.steps = a.replay_save_every
        else:
            tag = (f"{a.Nx}x{a.Ny}x{a.Nz}_T0_{int(self.T0)}_dx_{self.dx_phys:g}"
                   f"_dtphys_{self.dt_phys:g}_interval_{self.steps}_3D"
                   f"{'_hubble' if self.hubble else '_nohubble'}_eta_{self.eta_phys:g}"
                   f"_gb_{self.gb:g}_gf_{self.gf:g}_nb_{a.nb}_nf_{a.nf}"
                   f"{'_OD' if self.overdamped else ''}_{self.name}"
                   f"{'_CT' if a.counterterm else ''}"
                   f"{'_' + a.potential_type if a.potential_type != 'V_p' else ''}"
                   f"{'_noScaleFactor' if a.no_scale_factor else ''}")
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

    def init_state(self):
        a = self.args
        if self.replay:
            f = os.path.join(a.replay_dir, "field_states", f"state_step_{a.start_step:010d}.npz")
            if not os.path.exists(f):
                raise SystemExit(f"checkpoint file not found: {f}")
            with np.load(f) as z:
                d = {k: z[k] for k in z.files}
            if not self.overdamped and "pi" not in d:
                raise SystemExit(f"{f} has no 'pi' (lightweight snapshot)")
            names = ["phi"] + ([] if self.overdamped else ["pi"])
            if any(np.isnan(d[k]).any() for k in names):
                raise SystemExit(f"checkpoint {f} contains NaN")
            self._load(d, a.start_step)
            return
        rng = np.random.default_rng(a.init_seed)
        self.phi = self._field(0.01 * rng.standard_normal(self.shape))
        self.pi = self._field(np.zeros(self.shape))
        if a.resume:
            f, d = latest_checkpoint(self.state_path, need_pi=not self.overdamped)
            if d is not None:
                self.log(f"resuming from {f} (step {int(d['step'])})")
                self._load(d, int(d["step"]))

    def _load(self, d, step):
        names = ["phi"] + ([] if self.overdamped else ["pi"])
        fields = load_fields(d, names, self.args.storage, self.dev)
        self.phi = fields[0].reshape(self._shape_of())
        self.pi = fields[1].reshape(self._shape_of()) if len(fields) > 1 else \
            self._field(np.zeros(self.shape))
        self.n_start = step + 1                   # the step after the checkpoint's
        self.n_origin = step
        if self.hubble and "scale_factor" in d:
            self.a = float(d["scale_factor"])

    def _shape_of(self):
        return ((2,) + self.shape) if self.args.storage == "f32c" else self.shape

    def _values(self, t):
        return RF.from_f32c(t) if t.dim() == 4 else t

    # ------------------------------------------------------------ table ---
    def _rebuild(self, T, T_mid):
        v = self._values(self.phi)
        lo, hi = float(v.min()), float(v.max())
        margin = max(max(hi - lo, 1.0) * TABLE_MARGIN_FRAC, 20000.0)
        lo, hi = lo - margin, hi + margin
        self.tab = self.tp.table(T, lo, hi, TABLE_SIZE)
        self.tab_mid = self.tp.table(T_mid, lo, hi, TABLE_SIZE)
        self.t_lo, self.t_hi, self.T_last = lo, hi, T

    def _phi_range(self):
        """(min, max) of phi: from the previous step's fused range when it has one
        (rk2_nonfused), else two reductions."""
        if self.prange is not None and self._range_valid:
            lo, hi, _ = RF.PhiRange.decode(self.prange.last.cpu().numpy())
            return lo, hi
        v = self._values(self.phi)
        return float(v.min()), float(v.max())

    def _need_rebuild(self, n, T):
        if self.tab is None:
            return True
        if abs(T - self.T_last) / max(abs(T), 1.0) > 1e-4:
            return True
        if (n - self.n_start) % self.args.range_check_every:
            return False
        lo, hi = self._phi_range()
        return lo < self.t_lo or hi > self.t_hi

    # ------------------------------------------------------------- loop ---
    def scalars(self, n):
        """T, T_mid, eta_eff, inv_a2, inv_a3, H of step n; advances a (R:3621-3645)."""
        if self.hubble:
            T = self.T0 / self.a
            T4 = T * T * T * T
            H = math.sqrt((T4 * (G_STAR * np.pi ** 2 / 30.0) + DEL_V) * (1.0 / (3.0 * M_PL ** 2)))
            if self.args.no_scale_factor:
                eta_eff, inv_a2, inv_a3 = self.eta, 1.0, 1.0
            else:
                eta_eff = self.eta + 3.0 * H / self.mu
                inv_a2 = 1.0 / (self.a * self.a)
                inv_a3 = 1.0 / (self.a * self.a * self.a)
            self.a += self.a * H * (self.dt / self.mu)
            return T, self.T0 / self.a, eta_eff, inv_a2, inv_a3, H
        return self.T0, self.T0, self.eta, 1.0, 1.0, 0.0

    def step(self, n, T, T_mid, eta_eff, inv_a2, inv_a3):
        dt, dx, mu = self.dt, self.dx, self.mu
        c = (self.lam, self.mphi, self.bms, self.gb, self.gbg, self.gf, self.gfg)
        tab = self.tab + (TABLE_SIZE,) if self.uses_table else None
        if self.integrator == "overdamped":                                   # R:3676-3697
            ns = math.sqrt(2.0 * T * dt * inv_a3 / (eta_eff * mu ** 2 * self.dx_phys ** 3))
            RF.overdamped_euler_step_table(self.phi, dt, dx, eta_eff, mu, inv_a2, *tab, ns, n)
            return
        if self.integrator == "baoab":                                        # R:3698-3720
            ns = math.sqrt(T * inv_a3 / (mu ** 2 * self.dx_phys ** 3))
            RF.baoab_step_table(self.phi, self.pi, dt, dx, eta_eff, mu, inv_a2, *tab, ns, n)
            return
        ns = math.sqrt(2.0 * eta_eff * T * dt * inv_a3 / (mu ** 2 * self.dx_phys ** 3))
        if self.integrator == "rk2_fused_inline":                             # R:3728-3750
            RF.rk2_fused_single_pass(self.phi, self.pi, dt, dx, eta_eff, T, T_mid, mu, *c, ns, n,
                                     self.mid[0], self.mid[1], inv_a2, splines=self.tp)
            return
        RF.generate_noise_field(self.noise, ns, n)                            # R:3752-3757
        if self.integrator == "rk2_nonfused":
            RF.rk2_step_table(self.phi, self.pi, dt, dx, eta_eff, mu, self.noise, self.mid[0],
                              self.mid[1], inv_a2, *tab, phi_range=self.prange)
            self._range_valid = True
        elif self.integrator == "rk2_nonfused_inline":
            RF.rk2_step_inline(self.phi, self.pi, dt, dx, eta_eff, T, mu, *c, self.noise,
                               self.mid[0], self.mid[1], inv_a2, splines=self.tp)
        elif self.integrator == "rk2_fused_table":
            RF.rk2_fused_table(self.phi, self.pi, dt, dx, eta_eff, mu, self.noise, self.mid[0],
                               self.mid[1], inv_a2, *tab, *self.tab_mid, TABLE_SIZE)
        elif self.integrator == "rk2_fused":
            RF.rk2_step_fused(self.phi, self.pi, dt, dx, eta_eff, T, T_mid, mu, *c, self.noise,
                              None, None, self.mid[0], self.mid[1], inv_a2, splines=self.tp)
        else:                                                                 # "rk2", R:3837-3880
            half = self.noise * 0.5
            for TT in (T, T_mid):
                RF.rk2_step(self.phi, self.pi, 0.5 * dt, dx, eta_eff, TT, mu, *c, half, None,
                            None, self.mid[0], self.mid[1], inv_a2, splines=self.tp)

    def run(self):
        a = self.args
        self.init_state()
        os.makedirs(self.state_path, exist_ok=True)
        self.mid = [torch.empty_like(self.phi), torch.empty_like(self.pi)]
        ndt = torch.float32 if a.storage == "f32" else torch.float64
        self.noise = torch.empty(self.shape, dtype=ndt, device=self.dev)
        self.tab = None
        # the default integrator's step folds phi's range as it writes (the
        # per-step phi.min() / phi.max() of the table check, R:3655-3660)
        self.prange = RF.PhiRange(self.dev) if self.integrator == "rk2_nonfused" else None
        self._range_valid = False
        writer = SnapshotWriter(self.state_path, checkpoint_every=CHECKPOINT_EVERY)
        dense_on = a.phi_threshold is not None and a.steps_dense is not None
        dense_active = False
        nan_every = 1000 if self.replay else 100000
        t_start = time.time()
        self.status = "completed"
        for n in range(self.n_start, self.Nt):
            t = n * self.dt
            T, T_mid, eta_eff, inv_a2, inv_a3, H = self.scalars(n)
            if self.uses_table and self._need_rebuild(n, T):
                self._rebuild(T, T_mid)
            self.step(n, T, T_mid, eta_eff, inv_a2, inv_a3)
            if n % nan_every == 0 and not self._finite():                     # R:3882-3944
                path = os.path.join(self.state_path, f"state_step_{n:010d}_NaN_debug.npz")
                np.savez(path, phi=self._values(self.phi).double().cpu().numpy(), step=n,
                         time=t, temperature=T)
                self.log(f"NaN/Inf at step {n}; state written to {path}")
                self.status = "diverged"
                break
            cur = self.steps
            if dense_on and not dense_active:
                v = self._values(self.phi)
                if max(abs(float(v.min())), abs(float(v.max()))) > a.phi_threshold:
                    dense_active = True
                    cur = a.steps_dense
            elif dense_active:
                cur = a.steps_dense
            due = (n - self.n_origin) % cur == 0 if self.replay else n % cur == 0
            if due:
                en = None
                if a.diag_energy and not self.overdamped:
                    en = RF.compute_energy_densities(self.phi, self.pi, self.dx, inv_a2, self.lam,
                                                     self.mphi, self.mu)
                writer.save_real(n, t, T, self.phi, None if self.overdamped else self.pi,
                                 energies=en, scale_factor=self.a if self.hubble else None,
                                 hubble=H if self.hubble else None)
                done = n - self.n_start + 1
                el = time.time() - t_start
                self.log(f"Step {n}/{self.Nt} | t={t / self.mu:.2e} | T={T:.1f} | "
                         f"{done / el if el > 0 else 0.0:.1f} steps/s")
        torch.cuda.synchronize(self.dev)
        writer.wait()
        self.total_time = time.time() - t_start
        write_metadata(self.save_path, Nx=a.Nx, Ny=a.Ny, Nz=a.Nz, dx_phys=self.dx_phys,
                       dt_phys=self.dt_phys, mphi=self.mphi, lam=self.lam,
                       eta_phys=self.eta_phys, nb=a.nb, nf=a.nf, bosonCoupling=self.gb,
                       fermionCoupling=self.gf, T0=self.T0, cooling_rate=self.cooling_rate,
                       Nt=self.Nt, steps=self.steps, total_time=self.total_time, mu=self.mu,
                       dx=self.dx, dt=self.dt, eta=self.eta,
                       vev=np.sqrt(self.mphi ** 2 / self.lam), seed_bubbles=False,
                       bubble_config=np.array([]), bubble_profile="none", bubble_wall_width=0.0,
                       integrator=self.name, counterterm=a.counterterm,
                       potential_type=a.potential_type, no_scale_factor=a.no_scale_factor,
                       no_hubble=not self.hubble)
        return self.status

    def _finite(self):
        ok = bool(torch.isfinite(self.phi).all())
        if not self.overdamped:
            ok = ok and bool(torch.isfinite(self.pi).all())
        return ok


def main(argv=None):
    args = build_parser().parse_args(argv)
    r = Run(args)
    status = r.run()
    r.log(f"{status}: {r.save_path}")
    return 0 if status == "completed" else 1


if __name__ == "__main__":
    sys.exit(main())
