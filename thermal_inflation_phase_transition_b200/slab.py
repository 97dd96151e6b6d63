"""One lattice split into x-slabs across ranks (one process per GPU).

The reference decomposes only in CosmoLattice (MPI slabs along x,
simulation/run_cosmolattice.py:148-152); the numba stepper runs one lattice
on one node.  Here rank r of W owns lattice planes [i_lo, i_lo + nx_local)
(a balanced split of nx) in arrays of nx_local + 2 planes: plane 0 and plane
nx_local + 1 are ghost copies of the neighbouring ranks' edge planes (periodic
in x), filled by a halo exchange before every step.  The step itself is
``tipt_rk2_step_table_slab``: planes 1..nx_local with the hash noise keyed by
the lattice-wide site index, so the W ranks together reproduce the
single-lattice step bit for bit.  Observables reduce each slab over the
lattice's site count and combine with one all-reduce per quantity class.

The exchange is point-to-point: every field plane (hi and lo planes of a
compensated-FP32 field separately) goes to the neighbour that needs it as a
ghost, with ``torch.distributed`` send/receive (NCCL between GPUs, gloo on
CPU); with one rank the ghosts are local copies.  Sends to the upper
neighbour are issued before sends to the lower one and receives from the lower
neighbour before receives from the upper one, and the two directions carry
different tags, so the pairs match also when both neighbours are the same rank
(W = 2).
"""
from __future__ import annotations

import torch
import torch.distributed as dist

from . import _lib as L
from ._common import dims_of, need_cuda, ptr, step_params, storage_of, stream_handle

__all__ = ["Slab", "split_planes"]

_TAG_UP, _TAG_DOWN = 11, 12


def split_planes(nx: int, world: int, rank: int) -> tuple[int, int]:
    """(i_lo, nx_local) of rank `rank`: nx planes split into `world` runs whose
    lengths differ by at most one (the first nx % world ranks take one more)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank / world")
    base, extra = divmod(int(nx), int(world))
    if base < 1:
        raise ValueError(f"{nx} planes cannot be split over {world} ranks")
    nx_local = base + (1 if rank < extra else 0)
    i_lo = rank * base + min(rank, extra)
    return i_lo, nx_local


class Slab:
    """The slab of lattice `shape` = (nx, ny, nz) owned by this rank."""

    def __init__(self, shape, *, rank=None, world=None, group=None):
        nx, ny, nz = (int(x) for x in shape)
        if nz < 2:
            raise ValueError("slabs need nz >= 2 (a 2-D lattice is one GPU's work)")
        if world is None:
            world = dist.get_world_size(group) if dist.is_initialized() else 1
        if rank is None:
            rank = dist.get_rank(group) if dist.is_initialized() else 0
        self.shape = (nx, ny, nz)
        self.rank, self.world, self.group = int(rank), int(world), group
        self.i_lo, self.nx_local = split_planes(nx, self.world, self.rank)
        self.up = (self.rank + 1) % self.world
        self.down = (self.rank - 1) % self.world
        self.n_sites = nx * ny * nz

    # ----------------------------------------------------------- layout ---
    @property
    def local_shape(self):
        return (self.nx_local + 2, self.shape[1], self.shape[2])

    def empty(self, storage, device):
        """Uninitialised local field (ghost planes included)."""
        if storage == "f32c":
            return torch.empty((2,) + self.local_shape, dtype=torch.float32, device=device)
        dt = torch.float64 if storage == "f64" else torch.float32
        return torch.empty(self.local_shape, dtype=dt, device=device)

    def local_planes(self):
        """Lattice plane of every local plane, ghosts included."""
        nx = self.shape[0]
        return [(self.i_lo - 1 + q) % nx for q in range(self.nx_local + 2)]

    def scatter(self, field):
        """This rank's local field (ghosts filled) cut from a whole-lattice field
        (float (nx, ny, nz) or compensated (2, nx, ny, nz))."""
        idx = torch.tensor(self.local_planes(), device=field.device)
        dim = 1 if field.dim() == 4 else 0
        return field.index_select(dim, idx).contiguous()

    def interior(self, local):
        """View of the computed planes 1..nx_local."""
        if local.dim() == 4:
            return local[:, 1:self.nx_local + 1]
        return local[1:self.nx_local + 1]

    def gather(self, local):
        """The whole-lattice field from every rank's interior (all ranks get it)."""
        mine = self.interior(local).contiguous()
        if self.world == 1:
            return mine
        dim = 1 if local.dim() == 4 else 0
        sizes = [split_planes(self.shape[0], self.world, r)[1] for r in range(self.world)]
        parts = []
        for r, n in enumerate(sizes):
            shp = list(mine.shape)
            shp[dim] = n
            parts.append(torch.empty(shp, dtype=mine.dtype, device=mine.device))
        if len(set(sizes)) == 1:
            dist.all_gather(parts, mine, group=self.group)
        else:  # uneven slabs: pad to the largest, gather, trim
            big = max(sizes)
            shp = list(mine.shape)
            shp[dim] = big
            pad = torch.zeros(shp, dtype=mine.dtype, device=mine.device)
            pad.narrow(dim, 0, mine.shape[dim]).copy_(mine)
            bufs = [torch.empty_like(pad) for _ in sizes]
            dist.all_gather(bufs, pad, group=self.group)
            parts = [b.narrow(dim, 0, n) for b, n in zip(bufs, sizes)]
        return torch.cat(parts, dim=dim)

    # --------------------------------------------------------- exchange ---
    def _planes(self, t):
        return [t[0], t[1]] if t.dim() == 4 else [t]

    def exchange(self, *fields):
        """Fill the ghost planes of each local field from the neighbouring ranks."""
        n = self.nx_local
        if self.world == 1:
            for t in fields:
                for a in self._planes(t):
                    a[0].copy_(a[n])
                    a[n + 1].copy_(a[1])
            return
        ops = []
        for t in fields:
            for a in self._planes(t):
                ops.append(dist.P2POp(dist.isend, a[n], self.up, self.group, _TAG_UP))
                ops.append(dist.P2POp(dist.isend, a[1], self.down, self.group, _TAG_DOWN))
        for t in fields:
            for a in self._planes(t):
                ops.append(dist.P2POp(dist.irecv, a[0], self.down, self.group, _TAG_UP))
                ops.append(dist.P2POp(dist.irecv, a[n + 1], self.up, self.group, _TAG_DOWN))
        for w in dist.batch_isend_irecv(ops):
            w.wait()

    # ------------------------------------------------------------- step ---
    def step(self, phi, pi, phi_out, pi_out, dt, dx, eta_eff, mu, inv_a2, vsource, *,
             noise_scale=0.0, noise_step=0, seed=0, stream=None, stepper=None, overlap=True):
        """Halo exchange of (phi, pi), then one midpoint step of the local planes
        into (phi_out, pi_out) (rk2_step_table, R:1875-1966, hash noise).

        With ``overlap`` (and at least three local planes) the exchange runs on a
        second stream while the interior planes 2 .. nx_local - 1, which read no
        ghost plane, are stepped; the two edge planes follow the exchange.  The
        result is the same either way.  `stepper`, if given, replaces the library
        call with the same arguments after a plain exchange (the CPU tests pass
        the oracle)."""
        kw = dict(noise_scale=noise_scale, noise_step=noise_step, seed=seed)
        if stepper is not None:
            self.exchange(phi, pi)
            return stepper(self, phi, pi, phi_out, pi_out, dt, dx, eta_eff, mu, inv_a2, vsource,
                           noise_scale, noise_step, seed)
        args = (phi, pi, phi_out, pi_out, dt, dx, eta_eff, mu, inv_a2, vsource)
        n = self.nx_local
        if not overlap or n < 3:
            self.exchange(phi, pi)
            self.step_local(*args, stream=stream, **kw)
            return
        main = torch.cuda.current_stream(phi.device) if stream is None else stream
        if getattr(self, "_comm", None) is None:
            self._comm = torch.cuda.Stream(device=phi.device)
        ready = torch.cuda.Event()
        ready.record(main)                      # the inputs are complete on the main stream
        self._comm.wait_event(ready)
        with torch.cuda.stream(self._comm):
            self.exchange(phi, pi)
        done = torch.cuda.Event()
        done.record(self._comm)
        self.step_local(*args, stream=main, planes=(2, n), **kw)      # interior planes
        main.wait_event(done)
        self.step_local(*args, stream=main, planes=(1, 2), **kw)      # edge planes
        self.step_local(*args, stream=main, planes=(n, n + 1), **kw)

    def step_local(self, phi, pi, phi_out, pi_out, dt, dx, eta_eff, mu, inv_a2, vsource, *,
                   noise_scale=0.0, noise_step=0, seed=0, stream=None, planes=None):
        """The step of the local planes alone (ghost planes already filled);
        ``planes = (b, e)`` restricts it to the array planes [b, e) of
        [1, nx_local + 1)."""
        need_cuda(phi, pi, phi_out, pi_out, names=["phi", "pi", "phi_out", "pi_out"])
        nxl, ny, nz = dims_of(phi)
        if (nxl, ny, nz) != self.local_shape:
            raise ValueError(f"local fields must be {self.local_shape}, got {(nxl, ny, nz)}")
        b, e = planes if planes is not None else (1, self.nx_local + 1)
        sp = step_params(dt, dx, eta_eff, mu, inv_a2, noise_scale, noise_step, seed)
        L.call("tipt_rk2_step_table_slab_planes", storage_of(phi), ptr(phi), ptr(pi),
               ptr(phi_out), ptr(pi_out), self.nx_local, ny, nz, self.i_lo, self.shape[0], int(b),
               int(e), sp, vsource, stream_handle(stream))

    # ------------------------------------------------------ observables ---
    def observables(self, phi, pi=None, *, dx=1.0, inv_a2=1.0, lam=0.0, mphi=0.0, mu=1.0,
                    thr=1.0, workspace=None, stream=None, exchange=True):
        """The lattice's 10 observables (observables.OBS_NAMES), identical on every
        rank: the upper ghost plane of phi is refreshed (exchange=True), each rank
        reduces its planes over the lattice's site count, and the partial results
        are combined (sums; min; max) across ranks."""
        if exchange:
            self.exchange(phi)
        return self.combine(self.observables_local(phi, pi, dx=dx, inv_a2=inv_a2, lam=lam,
                                                   mphi=mphi, mu=mu, thr=thr,
                                                   workspace=workspace, stream=stream))

    def observables_local(self, phi, pi=None, *, dx=1.0, inv_a2=1.0, lam=0.0, mphi=0.0, mu=1.0,
                          thr=1.0, workspace=None, stream=None):
        """This slab's share of the observables (means over the lattice's site
        count; min / max / non-finite count of the slab), ghost planes as they are."""
        need_cuda(phi, pi, names=["phi", "pi"])
        nxl, ny, nz = self.local_shape
        out = torch.empty(10, dtype=torch.float64, device=phi.device)
        wb = int(L.lib().tipt_observables_workspace_size(nxl, ny, nz))
        if workspace is None:
            workspace = torch.empty(max(wb, 8) // 8 + 1, dtype=torch.float64, device=phi.device)
        L.call("tipt_observables_slab", storage_of(phi), ptr(phi), ptr(pi), self.nx_local, ny,
               nz, self.n_sites, float(dx), float(inv_a2), float(lam), float(mphi), float(mu),
               float(thr), ptr(out), ptr(workspace),
               workspace.numel() * workspace.element_size(), stream_handle(stream))
        return out

    def combine(self, out):
        """Combine per-rank slab observables: sums of the means and counts, min, max."""
        if self.world == 1:
            return out
        sums = out.clone()
        sums[7:9] = 0.0
        mn, mx = out[7:8].clone(), out[8:9].clone()
        dist.all_reduce(sums, op=dist.ReduceOp.SUM, group=self.group)
        dist.all_reduce(mn, op=dist.ReduceOp.MIN, group=self.group)
        dist.all_reduce(mx, op=dist.ReduceOp.MAX, group=self.group)
        sums[7] = mn[0]
        sums[8] = mx[0]
        return sums
