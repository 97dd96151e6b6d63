"""Real scalar field kernels with the reference's names and positional signatures.

Reference: simulation/latticeSimeRescale_numba.py (R).  Fields are CUDA tensors:
float64 (nx,ny,nz) [FP64], float32 (nx,ny,nz) [the reference's FP32 storage],
or float32 (2,nx,ny,nz) hi/lo planes [FP32-compensated, value hi + lo].  Calls are enqueued on
the current CUDA stream and do not synchronise.

Extensions over the reference signatures are keyword-only:
  noise=None   -> inline counter-based hash noise (R:2511-2522) with amplitude
                  ``noise_scale``, step counter ``noise_step`` and ``seed``
                  (seed=0 is the reference key);
  a 2-D ``vp_table`` with ``vp_T, vp_T_min, vp_T_dinv`` -> (phi, T) table.
"""
from __future__ import annotations

import torch

from . import _lib as L
from ._common import (dims_of, need_cuda, poly_source, ptr, same_layout, step_params,
                      storage_of, stream_handle, swap_storage, table_source)

K_PASS2 = L.K_PASS2
K_PASS4 = L.K_PASS4


def _noise_check(noise, phi, storage):
    if noise is None:
        return
    need_cuda(noise, names=["noise"])
    want = torch.float32 if storage == L.TIPT_F32 else torch.float64
    if noise.dtype != want or tuple(noise.shape) != dims_of(phi):
        raise ValueError(f"noise must be {want} with shape {dims_of(phi)}")


def hash_rng_pair(keys: torch.Tensor):
    """R:2322 _hash_rng_pair for a CUDA uint64/int64 key tensor -> (u1, u2, z)."""
    need_cuda(keys, names=["keys"])
    if keys.dtype not in (torch.int64, torch.uint64):
        raise TypeError("keys must be 64-bit integers")
    u1 = torch.empty(keys.shape, dtype=torch.float64, device=keys.device)
    u2 = torch.empty_like(u1)
    z = torch.empty_like(u1)
    L.call("tipt_hash_rng_pair", ptr(keys), keys.numel(), ptr(u1), ptr(u2), ptr(z),
           stream_handle())
    return u1, u2, z


def generate_noise_field(noise, scale, seed, *, mul=K_PASS2, hash_seed=0, component=0):
    """Counter-based replacement of R:1348 generate_noise_field(noise, scale, seed).

    The reference seeds MT19937 with ``seed`` (the step number, R:3748) and is not
    reproducible across thread counts; here noise = scale * z(site, seed, mul,
    hash_seed), identical for any launch configuration."""
    need_cuda(noise, names=["noise"])
    st = storage_of(noise)
    if st == L.TIPT_F32C:
        raise TypeError("noise fields are float64 or float32")
    nx, ny, nz = dims_of(noise)
    L.call("tipt_generate_noise_field", st, ptr(noise), nx, ny, nz, float(scale),
           int(seed) & (2 ** 64 - 1), int(mul), int(hash_seed) & (2 ** 64 - 1), int(component),
           stream_handle())


def rk2_step_table(phi, pi, dt, dx, eta_eff, mu, noise, phi_tmp, pi_tmp, inv_a2, vp_table,
                   vp_tmin, vp_dinv, vp_npts, *, noise_scale=0.0, noise_step=0, seed=0,
                   vp_T=None, vp_T_min=None, vp_T_dinv=None, phi_range=None):
    """R:1875 rk2_step_table: one midpoint RK2 step, updating phi and pi in place.

    The fused kernel writes the new state into phi_tmp / pi_tmp and the tensors
    then exchange storages, so on return phi, pi hold the new state (the
    reference's in-place result) and phi_tmp, pi_tmp hold the old one (the
    reference leaves the midpoint state there; both are scratch).  ``phi_range``
    (a PhiRange) receives the new phi's minimum and maximum from the same launch
    (the reference's per-step phi.min() / phi.max())."""
    st = storage_of(phi)
    need_cuda(phi, pi, phi_tmp, pi_tmp, names=["phi", "pi", "phi_tmp", "pi_tmp"])
    same_layout(phi, pi, phi_tmp, pi_tmp, names=["pi", "phi_tmp", "pi_tmp"])
    _noise_check(noise, phi, st)
    nx, ny, nz = dims_of(phi)
    vs = table_source(vp_table, vp_tmin, vp_dinv, vp_npts, vp_T, vp_T_min, vp_T_dinv)
    sp = step_params(dt, dx, eta_eff, mu, inv_a2, noise_scale, noise_step, seed)
    if phi_range is None:
        L.call("tipt_rk2_step_table", st, ptr(phi), ptr(pi), ptr(phi_tmp), ptr(pi_tmp), nx, ny,
               nz, sp, vs, ptr(noise), stream_handle())
    else:
        cur, nxt = phi_range.next_pair()
        L.call("tipt_rk2_step_table_range", st, ptr(phi), ptr(pi), ptr(phi_tmp), ptr(pi_tmp), nx,
               ny, nz, sp, vs, ptr(noise), ptr(cur), ptr(nxt), stream_handle())
    swap_storage(phi, phi_tmp)
    swap_storage(pi, pi_tmp)


def rk2_step_inline(phi, pi, dt, dx, eta_eff, T, mu, lam_val, mphi_val, bosonMassSquared,
                    bosonCoupling, bosonGaugeCoupling, fermionCoupling, fermionGaugeCoupling,
                    noise, phi_tmp, pi_tmp, inv_a2, *, splines=None, noise_scale=0.0,
                    noise_step=0, seed=0):
    """R:2654 rk2_step_inline: rk2_step_table's midpoint step with the thermal V'
    evaluated inline per site at T (R:2201-2266 _vprime_inline) instead of a table;
    phi and pi are updated in place.  ``noise`` is the reference's noise array (or
    None for inline hash noise with the keywords); the dJ splines come from
    ``splines`` (a thermal.ThermalPotential), by default the reference script's."""
    from .thermal import default_potential
    st = storage_of(phi)
    need_cuda(phi, pi, phi_tmp, pi_tmp, names=["phi", "pi", "phi_tmp", "pi_tmp"])
    same_layout(phi, pi, phi_tmp, pi_tmp, names=["pi", "phi_tmp", "pi_tmp"])
    _noise_check(noise, phi, st)
    nx, ny, nz = dims_of(phi)
    tp = splines if splines is not None else default_potential(phi.device)
    vs = tp.source(T, lam=lam_val, mphi=mphi_val, bosonMassSquared=bosonMassSquared,
                   bosonCoupling=bosonCoupling, bosonGaugeCoupling=bosonGaugeCoupling,
                   fermionCoupling=fermionCoupling, fermionGaugeCoupling=fermionGaugeCoupling)
    sp = step_params(dt, dx, eta_eff, mu, inv_a2, noise_scale, noise_step, seed)
    L.call("tipt_rk2_step_table", st, ptr(phi), ptr(pi), ptr(phi_tmp), ptr(pi_tmp), nx, ny, nz,
           sp, vs, ptr(noise), stream_handle())
    swap_storage(phi, phi_tmp)
    swap_storage(pi, pi_tmp)


def rk2_step_table_into(phi, pi, phi_out, pi_out, dt, dx, eta_eff, mu, inv_a2, vsource, *,
                        noise=None, noise_scale=0.0, noise_step=0, seed=0, stream=None,
                        phi_range=None):
    """Ping-pong form of rk2_step_table: (phi, pi) -> (phi_out, pi_out), no swap.

    ``vsource`` is a prepared V' source (``table_source`` / ``poly_source``);
    ``phi_range`` (a PhiRange) receives the range of phi_out from the same launch."""
    st = storage_of(phi)
    nx, ny, nz = dims_of(phi)
    sp = step_params(dt, dx, eta_eff, mu, inv_a2, noise_scale, noise_step, seed)
    if phi_range is None:
        L.call("tipt_rk2_step_table", st, ptr(phi), ptr(pi), ptr(phi_out), ptr(pi_out), nx, ny,
               nz, sp, vsource, ptr(noise), stream_handle(stream))
        return
    cur, nxt = phi_range.next_pair()
    L.call("tipt_rk2_step_table_range", st, ptr(phi), ptr(pi), ptr(phi_out), ptr(pi_out), nx, ny,
           nz, sp, vsource, ptr(noise), ptr(cur), ptr(nxt), stream_handle(stream))


class PhiRange:
    """Range of phi after each step, folded by the step kernel itself (the reference
    loop reads phi.min() and phi.max() every step, R:3655-3660, for its V' table
    check).  Two 3-word device buffers alternate: a step writes one and resets the
    other for the next step, so reading a step's range needs no extra launch.

        rng = PhiRange(device)
        rk2_step_table_into(phi, pi, po, qo, ..., vs, phi_range=rng)
        lo, hi, nonfinite = rng.decode(rng.last.cpu())     # or copy rng.last to a host buffer

    A CUDA graph bakes the two buffers into its launches: capture an even number of
    steps per graph, so that each buffer is written by one step and reset by the
    other on every replay."""

    def __init__(self, device="cuda"):
        self.buf = torch.empty((2, 4), dtype=torch.int32, device=device)
        self.buf[:, 0] = -1          # 0xFFFFFFFF: minimum code not yet seen
        self.buf[:, 1:] = 0
        self.k = 0
        self.last = self.buf[1]

    def next_pair(self):
        """(this step's words, the next step's words) and advance."""
        cur, nxt = self.buf[self.k], self.buf[self.k ^ 1]
        self.k ^= 1
        self.last = cur
        return cur, nxt

    @staticmethod
    def decode(words):
        """(min, max, nonfinite) from a step's 3 (or 4) int32 words on the host."""
        import numpy as np
        w = np.asarray(words, dtype=np.int64).astype(np.uint32)

        def f(c):
            c = int(c)
            u = c & 0x7FFFFFFF if c & 0x80000000 else (~c) & 0xFFFFFFFF
            return float(np.array([u], np.uint32).view(np.float32)[0])
        return f(w[0]), f(w[1]), bool(w[2])


def rk2_fused_table(phi, pi, dt, dx, eta_eff, mu, noise, phi_tmp, pi_tmp, inv_a2, vp_table_T,
                    vp_tmin_T, vp_dinv_T, vp_npts_T, vp_table_Tm, vp_tmin_Tm, vp_dinv_Tm,
                    vp_npts_Tm, *, noise_scale=0.0, noise_step=0, seed=0):
    """R:1708 rk2_fused_table: two dt/2 midpoint halves (tables at T, then T_mid).

    Half one runs (phi, pi) -> (phi_tmp, pi_tmp), half two (phi_tmp, pi_tmp) ->
    (phi, pi): the update is in place with no exchange.  noise=None uses the
    inline hash of rk2_fused_single_pass (0.5*ns*z, multipliers 73856093 then
    19349669)."""
    st = storage_of(phi)
    need_cuda(phi, pi, phi_tmp, pi_tmp, names=["phi", "pi", "phi_tmp", "pi_tmp"])
    same_layout(phi, pi, phi_tmp, pi_tmp, names=["pi", "phi_tmp", "pi_tmp"])
    _noise_check(noise, phi, st)
    nx, ny, nz = dims_of(phi)
    va = table_source(vp_table_T, vp_tmin_T, vp_dinv_T, vp_npts_T)
    vb = table_source(vp_table_Tm, vp_tmin_Tm, vp_dinv_Tm, vp_npts_Tm)
    sp = step_params(dt, dx, eta_eff, mu, inv_a2, noise_scale, noise_step, seed)
    L.call("tipt_rk2_fused_table", st, ptr(phi), ptr(pi), ptr(phi), ptr(pi), ptr(phi_tmp),
           ptr(pi_tmp), nx, ny, nz, sp, va, vb, ptr(noise), stream_handle())


def rk2_fused_single_pass(phi, pi, dt, dx, eta_eff, T, T_mid, mu, lam, mphi, bosonMassSquared,
                          bosonCoupling, bosonGaugeCoupling, fermionCoupling,
                          fermionGaugeCoupling, noise_scale, noise_seed, phi_tmp, pi_tmp,
                          inv_a2, *, seed=0, splines=None):
    """R:2339 rk2_fused_single_pass: 4-pass RK2 with inline V' and inline hash noise.

    ``noise_seed`` is the reference's name for the step counter (R:3742).  The
    inline V' is the reference's _vprime_inline (R:2201-2266) evaluated per site at T
    in the first half and T_mid in the second; its dJ splines are those of
    ``splines`` (a thermal.ThermalPotential), by default the reference script's
    module-level splines (thermal.default_potential).  With all four couplings zero
    it reduces to lam phi^3 - mphi^2 phi (R:2228), evaluated as a polynomial."""
    st = storage_of(phi)
    need_cuda(phi, pi, phi_tmp, pi_tmp, names=["phi", "pi", "phi_tmp", "pi_tmp"])
    same_layout(phi, pi, phi_tmp, pi_tmp, names=["pi", "phi_tmp", "pi_tmp"])
    nx, ny, nz = dims_of(phi)
    sp = step_params(dt, dx, eta_eff, mu, inv_a2, noise_scale, noise_seed, seed)
    if all(float(c) == 0.0 for c in (bosonCoupling, bosonGaugeCoupling, fermionCoupling,
                                     fermionGaugeCoupling)) and splines is None:
        va = vb = poly_source(-float(mphi) * float(mphi), 0.0, float(lam))
    else:
        from .thermal import default_potential
        tp = splines if splines is not None else default_potential(phi.device)
        kw = dict(lam=lam, mphi=mphi, bosonMassSquared=bosonMassSquared,
                  bosonCoupling=bosonCoupling, bosonGaugeCoupling=bosonGaugeCoupling,
                  fermionCoupling=fermionCoupling, fermionGaugeCoupling=fermionGaugeCoupling)
        va, vb = tp.source(T, **kw), tp.source(T_mid, **kw)
    L.call("tipt_rk2_fused_table", st, ptr(phi), ptr(pi), ptr(phi), ptr(pi), ptr(phi_tmp),
           ptr(pi_tmp), nx, ny, nz, sp, va, vb, None, stream_handle())


def laplacian_periodic(out, a, dx):
    """R:1364 laplacian_periodic: out = periodic 7-point Laplacian of a (out has a's
    storage; a float32 pair of planes is evaluated in FP64 and stored as hi/lo)."""
    need_cuda(out, a, names=["out", "a"])
    same_layout(a, out, names=["out"])
    L.call("tipt_laplacian_periodic", storage_of(a), ptr(a), ptr(out), *dims_of(a), float(dx),
           stream_handle())
    return out


def cubic_eval_uniform(x, x_min, h, nseg, c0, c1, c2, c3):
    """R:1415 cubic_eval_uniform at the points x (a float64 CUDA tensor of any shape;
    a Python number gives a Python float): segment trunc((x - x_min) / h) clamped
    to [0, nseg - 1], Horner in x - x_i.  c0 .. c3 are float64 CUDA tensors."""
    scalar = not isinstance(x, torch.Tensor)
    dev = c0.device
    xt = torch.tensor([float(x)], dtype=torch.float64, device=dev) if scalar else x
    need_cuda(xt, c0, c1, c2, c3, names=["x", "c0", "c1", "c2", "c3"])
    for c in (xt, c0, c1, c2, c3):
        if c.dtype != torch.float64 or not c.is_contiguous():
            raise ValueError("cubic_eval_uniform takes contiguous float64 tensors")
    if min(c.numel() for c in (c0, c1, c2, c3)) < int(nseg):
        raise ValueError("coefficient arrays are shorter than nseg")
    out = torch.empty_like(xt)
    L.call("tipt_cubic_eval_uniform", ptr(xt), xt.numel(), float(x_min), float(h), int(nseg),
           ptr(c0), ptr(c1), ptr(c2), ptr(c3), ptr(out), stream_handle())
    return float(out.item()) if scalar else out


def Vprime_field(out, phi, T, lam, mphi, bosonMassSquared, bosonCoupling, bosonGaugeCoupling,
                 fermionCoupling, fermionGaugeCoupling, *, splines=None):
    """R:1435 Vprime_field: out = V'(phi, T) per site (FP64 arithmetic; out float64,
    or float32 as the reference's float32 arrays).  The dJ splines come from
    ``splines`` (a thermal.ThermalPotential), by default the reference script's."""
    from .thermal import ThermalPotential, default_potential
    need_cuda(out, phi, names=["out", "phi"])
    if tuple(out.shape) != dims_of(phi) or out.dtype not in (torch.float64, torch.float32):
        raise ValueError(f"out must be float64/float32 with shape {dims_of(phi)}")
    tp = splines if splines is not None else default_potential(phi.device)
    q = tp.params
    th = L.Thermal(float(lam), float(mphi), float(bosonMassSquared), float(bosonCoupling),
                   float(bosonGaugeCoupling), float(fermionCoupling), float(fermionGaugeCoupling),
                   q.coeff_b, q.coeff_f, q.x_min, q.h, q.nseg, 1, q.spline)
    o = out if out.dtype == torch.float64 and out.is_contiguous() else \
        torch.empty(dims_of(phi), dtype=torch.float64, device=phi.device)
    L.call("tipt_thermal_vprime_field", storage_of(phi), ptr(phi), float(T), th, ptr(o),
           *dims_of(phi), stream_handle())
    if o is not out:
        out.copy_(o)
    return out


def _thermal_pair(phi, T_list, lam, mphi, bosonMassSquared, bosonCoupling, bosonGaugeCoupling,
                  fermionCoupling, fermionGaugeCoupling, splines):
    from .thermal import default_potential
    tp = splines if splines is not None else default_potential(phi.device)
    kw = dict(lam=lam, mphi=mphi, bosonMassSquared=bosonMassSquared, bosonCoupling=bosonCoupling,
              bosonGaugeCoupling=bosonGaugeCoupling, fermionCoupling=fermionCoupling,
              fermionGaugeCoupling=fermionGaugeCoupling, form="field")
    return [tp.source(T, **kw) for T in T_list]


def rk2_step(phi, pi, dt, dx, eta_eff, T, mu, lam, mphi, bosonMassSquared, bosonCoupling,
             bosonGaugeCoupling, fermionCoupling, fermionGaugeCoupling, noise, lap, Vp,
             phi_mid_buf, pi_mid_buf, inv_a2, *, splines=None):
    """R:1489 rk2_step: the un-fused midpoint step (laplacian_periodic and
    Vprime_field at phi, then at the midpoint; phi += dt pi~, pi += dt k~ + noise),
    in place, as one fused launch with V' in the Vprime_field form.  ``lap`` and
    ``Vp`` are the reference's scratch arrays and are not written;
    ``phi_mid_buf`` / ``pi_mid_buf`` exchange storage with phi / pi."""
    st = storage_of(phi)
    need_cuda(phi, pi, phi_mid_buf, pi_mid_buf, names=["phi", "pi", "phi_mid_buf", "pi_mid_buf"])
    same_layout(phi, pi, phi_mid_buf, pi_mid_buf, names=["pi", "phi_mid_buf", "pi_mid_buf"])
    _noise_check(noise, phi, st)
    (vs,) = _thermal_pair(phi, [T], lam, mphi, bosonMassSquared, bosonCoupling,
                          bosonGaugeCoupling, fermionCoupling, fermionGaugeCoupling, splines)
    sp = step_params(dt, dx, eta_eff, mu, inv_a2)
    L.call("tipt_rk2_step_table", st, ptr(phi), ptr(pi), ptr(phi_mid_buf), ptr(pi_mid_buf),
           *dims_of(phi), sp, vs, ptr(noise), stream_handle())
    swap_storage(phi, phi_mid_buf)
    swap_storage(pi, pi_mid_buf)


def rk2_step_fused(phi, pi, dt, dx, eta_eff, T, T_mid, mu, lam, mphi, bosonMassSquared,
                   bosonCoupling, bosonGaugeCoupling, fermionCoupling, fermionGaugeCoupling,
                   noise, lap, Vp, phi_mid_buf, pi_mid_buf, inv_a2, *, splines=None):
    """R:1553 rk2_step_fused: two dt/2 midpoint halves with V' (Vprime_field form)
    at T, then T_mid, and 0.5 * noise in each half, in place (two launches; the
    state between the halves lives in phi_mid_buf / pi_mid_buf).  ``lap`` and
    ``Vp`` are the reference's scratch arrays and are not written."""
    st = storage_of(phi)
    need_cuda(phi, pi, phi_mid_buf, pi_mid_buf, names=["phi", "pi", "phi_mid_buf", "pi_mid_buf"])
    same_layout(phi, pi, phi_mid_buf, pi_mid_buf, names=["pi", "phi_mid_buf", "pi_mid_buf"])
    _noise_check(noise, phi, st)
    va, vb = _thermal_pair(phi, [T, T_mid], lam, mphi, bosonMassSquared, bosonCoupling,
                           bosonGaugeCoupling, fermionCoupling, fermionGaugeCoupling, splines)
    sp = step_params(dt, dx, eta_eff, mu, inv_a2)
    L.call("tipt_rk2_fused_table", st, ptr(phi), ptr(pi), ptr(phi), ptr(pi), ptr(phi_mid_buf),
           ptr(pi_mid_buf), *dims_of(phi), sp, va, vb, ptr(noise), stream_handle())


def _vsource_1d(vp_table, vp_tmin, vp_dinv, vp_npts, vpoly):
    if vpoly is not None:
        return poly_source(*[float(c) for c in vpoly])
    return table_source(vp_table, vp_tmin, vp_dinv, vp_npts)


def overdamped_euler_step_table(phi, dt, dx, eta_eff, mu, inv_a2, vp_table, vp_tmin, vp_dinv,
                                vp_npts, noise_scale, seed, *, phi_tmp=None, hash_seed=0,
                                vpoly=None):
    """R:2115 overdamped_euler_step_table: phi += dt/eta_eff F(phi) + noise_scale z, in place.

    ``seed`` is the reference's per-step seed (the step number): here it is the hash
    noise step; ``hash_seed`` selects an independent stream.  The update is simultaneous
    over the lattice (the new field goes to ``phi_tmp``, then the storages swap);
    ``phi_tmp`` is allocated when not given.  ``vpoly = (c1, c2, c3)`` replaces the
    table by V' = c1 phi + c2 phi^2 + c3 phi^3."""
    st = storage_of(phi)
    need_cuda(phi, names=["phi"])
    tmp = torch.empty_like(phi) if phi_tmp is None else phi_tmp
    same_layout(phi, tmp, names=["phi_tmp"])
    nx, ny, nz = dims_of(phi)
    vs = _vsource_1d(vp_table, vp_tmin, vp_dinv, vp_npts, vpoly)
    sp = step_params(dt, dx, eta_eff, mu, inv_a2, noise_scale, seed, hash_seed)
    L.call("tipt_overdamped_step_table", st, ptr(phi), ptr(tmp), nx, ny, nz, sp, vs,
           stream_handle())
    swap_storage(phi, tmp)


def baoab_step_table(phi, pi, dt, dx, gamma, mu, inv_a2, vp_table, vp_tmin, vp_dinv, vp_npts,
                     noise_scale, seed, *, phi_tmp=None, pi_tmp=None, hash_seed=0, vpoly=None):
    """R:1974 baoab_step_table: one BAOAB step of (phi, pi) in place (B A O A B,
    c1 = exp(-gamma dt), c2 = sqrt(1 - c1^2) noise_scale); arguments as
    overdamped_euler_step_table."""
    st = storage_of(phi)
    need_cuda(phi, pi, names=["phi", "pi"])
    pt = torch.empty_like(phi) if phi_tmp is None else phi_tmp
    qt = torch.empty_like(pi) if pi_tmp is None else pi_tmp
    same_layout(phi, pi, pt, qt, names=["pi", "phi_tmp", "pi_tmp"])
    nx, ny, nz = dims_of(phi)
    vs = _vsource_1d(vp_table, vp_tmin, vp_dinv, vp_npts, vpoly)
    sp = step_params(dt, dx, gamma, mu, inv_a2, noise_scale, seed, hash_seed)
    L.call("tipt_baoab_step_table", st, ptr(phi), ptr(pi), ptr(pt), ptr(qt), nx, ny, nz, sp, vs,
           stream_handle())
    swap_storage(phi, pt)
    swap_storage(pi, qt)


def compute_energy_densities(phi, pi, dx, inv_a2, lam_val, mphi_val, mu):
    """R:2270 compute_energy_densities -> (E_kin, E_grad, E_pot) as Python floats."""
    from .observables import observables
    o = observables(phi, pi, dx=dx, inv_a2=inv_a2, lam=lam_val, mphi=mphi_val, mu=mu)
    v = o.tolist()
    return v[0], v[1], v[2]


# ------------------------------------------------------------ state helpers
def to_f32c(x: torch.Tensor) -> torch.Tensor:
    """float64 field -> float32 (2, ...) hi/lo planes (exact to 48 bits)."""
    hi = x.to(torch.float32)
    lo = (x - hi.to(torch.float64)).to(torch.float32)
    return torch.stack([hi, lo], dim=0).contiguous()


def from_f32c(x: torch.Tensor) -> torch.Tensor:
    """float32 (2, ...) hi/lo planes -> float64 field."""
    return x[0].to(torch.float64) + x[1].to(torch.float64)
