"""Complex scalar field kernels with the reference's names and positional signatures.

Reference: simulation/latticeSimComplex_numba.py (C).  Phi = phi1 + i phi2; each
component is a CUDA tensor in one of the three storages (see real_field).

Extensions over the reference signatures are keyword-only:
  zn=(N, delta_V, active) -> the reference's _ZN_PARAMS (C:226-231), passed
                             per call instead of frozen into the compiled kernel;
  eps4                    -> eps * Re(Phi^4) symmetry breaking;
  noise1=noise2=None      -> inline hash noise, one pair per site (C:2958-2974).
"""
from __future__ import annotations

import torch

from . import _lib as L
from ._common import (dims_of, need_cuda, poly_source, ptr, same_layout, step_params, storage_of,
                      stream_handle, swap_storage, table_source)


def rk2_step_table(phi1, phi2, pi1, pi2, dt, dx, eta_eff, mu, noise1, noise2, phi1_tmp,
                   phi2_tmp, pi1_tmp, pi2_tmp, inv_a2, vp_table, vp_tmin, vp_dinv, vp_npts, *,
                   zn=(0.0, 0.0, 0.0), eps4=0.0, noise_scale=0.0, noise_step=0, seed=0,
                   rho_range=None):
    """C:2067 rk2_step_table (complex): one midpoint step, in place (storage exchange
    with the *_tmp tensors, as real_field.rk2_step_table).  ``rho_range`` (a
    real_field.PhiRange) receives the new |Phi|'s minimum and maximum from the same
    launch (the complex loop's per-step rho check, C:4263-4288)."""
    st = storage_of(phi1)
    arrs = (phi1, phi2, pi1, pi2, phi1_tmp, phi2_tmp, pi1_tmp, pi2_tmp)
    names = ("phi1", "phi2", "pi1", "pi2", "phi1_tmp", "phi2_tmp", "pi1_tmp", "pi2_tmp")
    need_cuda(*arrs, names=names)
    same_layout(phi1, *arrs[1:], names=names[1:])
    if (noise1 is None) != (noise2 is None):
        raise ValueError("give both noise1 and noise2, or neither")
    if noise1 is not None:
        need_cuda(noise1, noise2, names=["noise1", "noise2"])
        want = torch.float32 if st == L.TIPT_F32 else torch.float64
        for n in (noise1, noise2):
            if n.dtype != want or tuple(n.shape) != dims_of(phi1):
                raise ValueError(f"noise arrays must be {want} with shape {dims_of(phi1)}")
    nx, ny, nz = dims_of(phi1)
    vs = table_source(vp_table, vp_tmin, vp_dinv, vp_npts)
    sp = step_params(dt, dx, eta_eff, mu, inv_a2, noise_scale, noise_step, seed)
    ct = L.ComplexTerms(float(zn[0]), float(zn[1]), float(zn[2]), float(eps4))
    args = (st, ptr(phi1), ptr(phi2), ptr(pi1), ptr(pi2), ptr(phi1_tmp), ptr(phi2_tmp),
            ptr(pi1_tmp), ptr(pi2_tmp), nx, ny, nz, sp, vs, ct, ptr(noise1), ptr(noise2))
    if rho_range is None:
        L.call("tipt_complex_rk2_step_table", *args, stream_handle())
    else:
        cur, nxt = rho_range.next_pair()
        L.call("tipt_complex_rk2_step_table_range", *args, ptr(cur), ptr(nxt), stream_handle())
    for a, b in ((phi1, phi1_tmp), (phi2, phi2_tmp), (pi1, pi1_tmp), (pi2, pi2_tmp)):
        swap_storage(a, b)


def _check_noise_pair(noise1, noise2, st, phi1):
    if (noise1 is None) != (noise2 is None):
        raise ValueError("give both noise1 and noise2, or neither")
    if noise1 is not None:
        need_cuda(noise1, noise2, names=["noise1", "noise2"])
        want = torch.float32 if st == L.TIPT_F32 else torch.float64
        for n in (noise1, noise2):
            if n.dtype != want or tuple(n.shape) != dims_of(phi1):
                raise ValueError(f"noise arrays must be {want} with shape {dims_of(phi1)}")


def _fused(state, tmp, dt, dx, eta_eff, mu, inv_a2, va, vb, zn, eps4, noise1, noise2,
           noise_scale, noise_step, seed):
    """Two dt/2 halves in place: state -> tmp (first half) -> state (second half)."""
    st = storage_of(state[0])
    names = ("phi1", "phi2", "pi1", "pi2", "phi1_tmp", "phi2_tmp", "pi1_tmp", "pi2_tmp")
    need_cuda(*state, *tmp, names=names)
    same_layout(state[0], *state[1:], *tmp, names=names[1:])
    _check_noise_pair(noise1, noise2, st, state[0])
    nx, ny, nz = dims_of(state[0])
    sp = step_params(dt, dx, eta_eff, mu, inv_a2, noise_scale, noise_step, seed)
    ct = L.ComplexTerms(float(zn[0]), float(zn[1]), float(zn[2]), float(eps4))
    L.call("tipt_complex_rk2_fused_table", st, *[ptr(a) for a in state],
           *[ptr(a) for a in state], *[ptr(a) for a in tmp], nx, ny, nz, sp, va, vb, ct,
           ptr(noise1), ptr(noise2), stream_handle())


def rk2_fused_table(phi1, phi2, pi1, pi2, dt, dx, eta_eff, mu, noise1, noise2, phi1_tmp,
                    phi2_tmp, pi1_tmp, pi2_tmp, inv_a2, vp_table_T, vp_tmin_T, vp_dinv_T,
                    vp_npts_T, vp_table_Tm, vp_tmin_Tm, vp_dinv_Tm, vp_npts_Tm, *,
                    zn=(0.0, 0.0, 0.0), eps4=0.0, noise_scale=0.0, noise_step=0, seed=0):
    """C:1789 rk2_fused_table (complex): two dt/2 halves with the V'(rho) tables at T
    and T_mid, 0.5*noise in each half, in place; noise1 = noise2 = None selects the
    inline hash pairs (keywords)."""
    va = table_source(vp_table_T, vp_tmin_T, vp_dinv_T, vp_npts_T)
    vb = table_source(vp_table_Tm, vp_tmin_Tm, vp_dinv_Tm, vp_npts_Tm)
    _fused((phi1, phi2, pi1, pi2), (phi1_tmp, phi2_tmp, pi1_tmp, pi2_tmp), dt, dx, eta_eff, mu,
           inv_a2, va, vb, zn, eps4, noise1, noise2, noise_scale, noise_step, seed)


def _thermal_kw(lam, mphi, bosonMassSquared, bosonCoupling, bosonGaugeCoupling, fermionCoupling,
                fermionGaugeCoupling):
    return dict(lam=lam, mphi=mphi, bosonMassSquared=bosonMassSquared,
                bosonCoupling=bosonCoupling, bosonGaugeCoupling=bosonGaugeCoupling,
                fermionCoupling=fermionCoupling, fermionGaugeCoupling=fermionGaugeCoupling)


def rk2_fused_single_pass(phi1, phi2, pi1, pi2, dt, dx, eta_eff, T, T_mid, mu, lam, mphi,
                          bosonMassSquared, bosonCoupling, bosonGaugeCoupling, fermionCoupling,
                          fermionGaugeCoupling, noise_scale, noise_seed, phi1_tmp, phi2_tmp,
                          pi1_tmp, pi2_tmp, inv_a2, *, zn=(0.0, 0.0, 0.0), eps4=0.0,
                          splines=None, seed=0):
    """C:2765 rk2_fused_single_pass (complex): two dt/2 halves with the inline V'(rho)
    (C:2605-2680 _vprime_complex_inline) at T, then T_mid, and one inline hash pair per
    site per half (multipliers 73856093, 19349669; ``noise_seed`` is the step counter),
    in place.  The dJ splines come from ``splines`` (a thermal.ThermalPotential), by
    default the complex script's (its _POT_COEFFS = (2, -1), C:215)."""
    from .thermal import default_potential
    tp = splines if splines is not None else default_potential(phi1.device, (2.0, -1.0))
    kw = _thermal_kw(lam, mphi, bosonMassSquared, bosonCoupling, bosonGaugeCoupling,
                     fermionCoupling, fermionGaugeCoupling)
    _fused((phi1, phi2, pi1, pi2), (phi1_tmp, phi2_tmp, pi1_tmp, pi2_tmp), dt, dx, eta_eff, mu,
           inv_a2, tp.source(T, **kw), tp.source(T_mid, **kw), zn, eps4, None, None,
           noise_scale, noise_seed, seed)


def rk2_step_inline(phi1, phi2, pi1, pi2, dt, dx, eta_eff, T, mu, lam_val, mphi_val,
                    bosonMassSquared, bosonCoupling, bosonGaugeCoupling, fermionCoupling,
                    fermionGaugeCoupling, noise1, noise2, phi1_tmp, phi2_tmp, pi1_tmp, pi2_tmp,
                    inv_a2, *, zn=(0.0, 0.0, 0.0), eps4=0.0, splines=None, noise_scale=0.0,
                    noise_step=0, seed=0):
    """C:3140 rk2_step_inline (complex): rk2_step_table's midpoint step with the inline
    V'(rho) at T, in place (storage exchange with the *_tmp tensors); noise arrays as
    the reference passes them, or None for the inline hash pair (keywords)."""
    from .thermal import default_potential
    st = storage_of(phi1)
    arrs = (phi1, phi2, pi1, pi2, phi1_tmp, phi2_tmp, pi1_tmp, pi2_tmp)
    names = ("phi1", "phi2", "pi1", "pi2", "phi1_tmp", "phi2_tmp", "pi1_tmp", "pi2_tmp")
    need_cuda(*arrs, names=names)
    same_layout(phi1, *arrs[1:], names=names[1:])
    _check_noise_pair(noise1, noise2, st, phi1)
    tp = splines if splines is not None else default_potential(phi1.device, (2.0, -1.0))
    vs = tp.source(T, **_thermal_kw(lam_val, mphi_val, bosonMassSquared, bosonCoupling,
                                    bosonGaugeCoupling, fermionCoupling, fermionGaugeCoupling))
    nx, ny, nz = dims_of(phi1)
    sp = step_params(dt, dx, eta_eff, mu, inv_a2, noise_scale, noise_step, seed)
    ct = L.ComplexTerms(float(zn[0]), float(zn[1]), float(zn[2]), float(eps4))
    L.call("tipt_complex_rk2_step_table", st, *[ptr(a) for a in arrs], nx, ny, nz, sp, vs, ct,
           ptr(noise1), ptr(noise2), stream_handle())
    for a, b in ((phi1, phi1_tmp), (phi2, phi2_tmp), (pi1, pi1_tmp), (pi2, pi2_tmp)):
        swap_storage(a, b)


def _field_sources(phi1, Ts, lam, mphi, bosonMassSquared, bosonCoupling, bosonGaugeCoupling,
                   fermionCoupling, fermionGaugeCoupling, splines):
    from .thermal import default_potential
    tp = splines if splines is not None else default_potential(phi1.device, (2.0, -1.0))
    kw = _thermal_kw(lam, mphi, bosonMassSquared, bosonCoupling, bosonGaugeCoupling,
                     fermionCoupling, fermionGaugeCoupling)
    return [tp.source(T, form="field", **kw) for T in Ts]


def Vprime_field(out1, out2, phi1_arr, phi2_arr, T, lam, mphi, bosonMassSquared, bosonCoupling,
                 bosonGaugeCoupling, fermionCoupling, fermionGaugeCoupling, *,
                 zn=(0.0, 0.0, 0.0), splines=None):
    """C:1452 Vprime_field of the complex field: (out1, out2) = V'(rho) phi_a / rho
    (+ the Z_N term of ``zn``), FP64 arithmetic; out float64 (or float32).  The dJ
    splines default to the complex script's (pot_coeffs (2, -1))."""
    from .thermal import default_potential
    need_cuda(out1, out2, phi1_arr, phi2_arr, names=["out1", "out2", "phi1", "phi2"])
    same_layout(phi1_arr, phi2_arr, names=["phi2"])
    shape = dims_of(phi1_arr)
    for o in (out1, out2):
        if tuple(o.shape) != shape or o.dtype not in (torch.float64, torch.float32):
            raise ValueError(f"outputs must be float64/float32 with shape {shape}")
    tp = splines if splines is not None else default_potential(phi1_arr.device, (2.0, -1.0))
    q = tp.params
    th = L.Thermal(float(lam), float(mphi), float(bosonMassSquared), float(bosonCoupling),
                   float(bosonGaugeCoupling), float(fermionCoupling), float(fermionGaugeCoupling),
                   q.coeff_b, q.coeff_f, q.x_min, q.h, q.nseg, 1, q.spline)
    ct = L.ComplexTerms(float(zn[0]), float(zn[1]), float(zn[2]), 0.0)
    tmp = [o if o.dtype == torch.float64 and o.is_contiguous() else
           torch.empty(shape, dtype=torch.float64, device=phi1_arr.device) for o in (out1, out2)]
    L.call("tipt_thermal_vprime_field_complex", storage_of(phi1_arr), ptr(phi1_arr),
           ptr(phi2_arr), float(T), th, ct, ptr(tmp[0]), ptr(tmp[1]), *shape, stream_handle())
    for o, t in zip((out1, out2), tmp):
        if o is not t:
            o.copy_(t)
    return out1, out2


def rk2_step(phi1, phi2, pi1, pi2, dt, dx, eta_eff, T, mu, lam, mphi, bosonMassSquared,
             bosonCoupling, bosonGaugeCoupling, fermionCoupling, fermionGaugeCoupling, noise1,
             noise2, lap1, lap2, Vp1, Vp2, phi1_mid_buf, phi2_mid_buf, pi1_mid_buf, pi2_mid_buf,
             inv_a2, *, zn=(0.0, 0.0, 0.0), eps4=0.0, splines=None):
    """C:1533 rk2_step (complex): the un-fused midpoint step with Vprime_field
    (C:1452) at phi, then at the midpoint, in place, as one fused launch; the
    scratch arrays lap1 .. Vp2 are accepted and not written; the *_mid_buf tensors
    exchange storage with phi1 .. pi2."""
    st = storage_of(phi1)
    arrs = (phi1, phi2, pi1, pi2, phi1_mid_buf, phi2_mid_buf, pi1_mid_buf, pi2_mid_buf)
    names = ("phi1", "phi2", "pi1", "pi2", "phi1_mid_buf", "phi2_mid_buf", "pi1_mid_buf",
             "pi2_mid_buf")
    need_cuda(*arrs, names=names)
    same_layout(phi1, *arrs[1:], names=names[1:])
    _check_noise_pair(noise1, noise2, st, phi1)
    (vs,) = _field_sources(phi1, [T], lam, mphi, bosonMassSquared, bosonCoupling,
                           bosonGaugeCoupling, fermionCoupling, fermionGaugeCoupling, splines)
    sp = step_params(dt, dx, eta_eff, mu, inv_a2)
    ct = L.ComplexTerms(float(zn[0]), float(zn[1]), float(zn[2]), float(eps4))
    L.call("tipt_complex_rk2_step_table", st, *[ptr(a) for a in arrs], *dims_of(phi1), sp, vs, ct,
           ptr(noise1), ptr(noise2), stream_handle())
    for a, b in zip(arrs[:4], arrs[4:]):
        swap_storage(a, b)


def rk2_step_fused(phi1, phi2, pi1, pi2, dt, dx, eta_eff, T, T_mid, mu, lam, mphi,
                   bosonMassSquared, bosonCoupling, bosonGaugeCoupling, fermionCoupling,
                   fermionGaugeCoupling, noise1, noise2, lap1, lap2, Vp1, Vp2, phi1_mid_buf,
                   phi2_mid_buf, pi1_mid_buf, pi2_mid_buf, inv_a2, *, zn=(0.0, 0.0, 0.0),
                   eps4=0.0, splines=None):
    """C:1610 rk2_step_fused (complex): two dt/2 halves with Vprime_field at T, then
    T_mid, and 0.5 * noise in each, in place (two launches; the state between the
    halves lives in the *_mid_buf tensors); lap1 .. Vp2 are accepted and not written."""
    va, vb = _field_sources(phi1, [T, T_mid], lam, mphi, bosonMassSquared, bosonCoupling,
                            bosonGaugeCoupling, fermionCoupling, fermionGaugeCoupling, splines)
    _fused((phi1, phi2, pi1, pi2), (phi1_mid_buf, phi2_mid_buf, pi1_mid_buf, pi2_mid_buf), dt, dx,
           eta_eff, mu, inv_a2, va, vb, zn, eps4, noise1, noise2, 0.0, 0, 0)


def rk2_step_table_into(state, out, dt, dx, eta_eff, mu, inv_a2, vsource, *, zn=(0.0, 0.0, 0.0),
                        eps4=0.0, noise_scale=0.0, noise_step=0, seed=0, stream=None,
                        rho_range=None):
    """Ping-pong form: state=(phi1, phi2, pi1, pi2) -> out=(phi1', phi2', pi1', pi2');
    ``rho_range`` (a real_field.PhiRange) receives the range of the new |Phi|."""
    st = storage_of(state[0])
    nx, ny, nz = dims_of(state[0])
    sp = step_params(dt, dx, eta_eff, mu, inv_a2, noise_scale, noise_step, seed)
    ct = L.ComplexTerms(float(zn[0]), float(zn[1]), float(zn[2]), float(eps4))
    args = (st, *[ptr(a) for a in state], *[ptr(a) for a in out], nx, ny, nz, sp, vsource, ct,
            None, None)
    if rho_range is None:
        L.call("tipt_complex_rk2_step_table", *args, stream_handle(stream))
    else:
        cur, nxt = rho_range.next_pair()
        L.call("tipt_complex_rk2_step_table_range", *args, ptr(cur), ptr(nxt),
               stream_handle(stream))


def _vsource_1d(vp_table, vp_tmin, vp_dinv, vp_npts, vpoly):
    if vpoly is not None:
        return poly_source(*[float(c) for c in vpoly])
    return table_source(vp_table, vp_tmin, vp_dinv, vp_npts)


def overdamped_euler_step_table(phi1, phi2, dt, dx, eta_eff, mu, inv_a2, vp_table, vp_tmin,
                                vp_dinv, vp_npts, noise_scale, seed, *, tmp=None,
                                zn=(0.0, 0.0, 0.0), eps4=0.0, hash_seed=0, vpoly=None):
    """C:2422 overdamped_euler_step_table (complex), in place; ``seed`` is the hash noise
    step (the reference's per-step seed); ``tmp`` = two scratch fields (allocated when
    not given)."""
    st = storage_of(phi1)
    need_cuda(phi1, phi2, names=["phi1", "phi2"])
    t = tmp if tmp is not None else [torch.empty_like(phi1), torch.empty_like(phi2)]
    same_layout(phi1, phi2, *t, names=["phi2", "tmp1", "tmp2"])
    nx, ny, nz = dims_of(phi1)
    vs = _vsource_1d(vp_table, vp_tmin, vp_dinv, vp_npts, vpoly)
    sp = step_params(dt, dx, eta_eff, mu, inv_a2, noise_scale, seed, hash_seed)
    ct = L.ComplexTerms(float(zn[0]), float(zn[1]), float(zn[2]), float(eps4))
    L.call("tipt_complex_overdamped_step_table", st, ptr(phi1), ptr(phi2), ptr(t[0]), ptr(t[1]),
           nx, ny, nz, sp, vs, ct, stream_handle())
    swap_storage(phi1, t[0])
    swap_storage(phi2, t[1])


def baoab_step_table(phi1, phi2, pi1, pi2, dt, dx, gamma, mu, inv_a2, vp_table, vp_tmin, vp_dinv,
                     vp_npts, noise_scale, seed, *, tmp=None, zn=(0.0, 0.0, 0.0), eps4=0.0,
                     hash_seed=0, vpoly=None):
    """C:2223 baoab_step_table (complex): one BAOAB step in place; ``tmp`` = four scratch
    fields (allocated when not given)."""
    st = storage_of(phi1)
    arrs = (phi1, phi2, pi1, pi2)
    need_cuda(*arrs, names=["phi1", "phi2", "pi1", "pi2"])
    t = tmp if tmp is not None else [torch.empty_like(a) for a in arrs]
    same_layout(phi1, *arrs[1:], *t, names=["phi2", "pi1", "pi2", "t1", "t2", "t3", "t4"])
    nx, ny, nz = dims_of(phi1)
    vs = _vsource_1d(vp_table, vp_tmin, vp_dinv, vp_npts, vpoly)
    sp = step_params(dt, dx, gamma, mu, inv_a2, noise_scale, seed, hash_seed)
    ct = L.ComplexTerms(float(zn[0]), float(zn[1]), float(zn[2]), float(eps4))
    L.call("tipt_complex_baoab_step_table", st, *[ptr(a) for a in arrs], *[ptr(a) for a in t],
           nx, ny, nz, sp, vs, ct, stream_handle())
    for a, b in zip(arrs, t):
        swap_storage(a, b)


class WindingResult:
    """Device outputs of compute_winding_number_full."""

    def __init__(self, w_site, w3, pierced, counts):
        self.w_site, self.w3, self.pierced, self.counts = w_site, w3, pierced, counts

    def host_counts(self):
        c = self.counts.tolist()
        return {"pierced_xy": c[0], "pierced_xz": c[1], "pierced_yz": c[2], "n_strings": c[3],
                "listed": c[4], "string_length": c[0] + c[1] + c[2]}


def compute_winding_number(phi1, phi2, winding_out):
    """C:2683 compute_winding_number(phi1, phi2, winding_out): per-site winding
    (sum over the XY, XZ, YZ plaquettes) into float32 ``winding_out``."""
    need_cuda(phi1, phi2, winding_out, names=["phi1", "phi2", "winding_out"])
    st = storage_of(phi1)
    if winding_out.dtype != torch.float32 or tuple(winding_out.shape) != dims_of(phi1):
        raise ValueError("winding_out must be float32 with the lattice shape")
    counts = torch.empty(5, dtype=torch.int64, device=phi1.device)
    L.call("tipt_compute_winding_number", st, ptr(phi1), ptr(phi2), *dims_of(phi1),
           ptr(winding_out), None, None, 0, ptr(counts), stream_handle())
    return winding_out


def compute_winding_number_full(phi1, phi2, *, w_site=True, w3=True, pierced_cap=0,
                                stream=None):
    """Winding with per-orientation int8 windings, a compacted list of pierced
    plaquettes (site*3 + orientation, XY=0, XZ=1, YZ=2) and device counts."""
    need_cuda(phi1, phi2, names=["phi1", "phi2"])
    st = storage_of(phi1)
    shape = dims_of(phi1)
    dev = phi1.device
    ws = torch.empty(shape, dtype=torch.float32, device=dev) if w_site else None
    w3t = torch.empty((3,) + shape, dtype=torch.int8, device=dev) if w3 else None
    pl = torch.empty(max(pierced_cap, 1), dtype=torch.int32, device=dev) if pierced_cap else None
    counts = torch.empty(5, dtype=torch.int64, device=dev)
    L.call("tipt_compute_winding_number", st, ptr(phi1), ptr(phi2), *shape, ptr(ws), ptr(w3t),
           ptr(pl), int(pierced_cap), ptr(counts), stream_handle(stream))
    return WindingResult(ws, w3t, pl, counts)


# C:1387 laplacian_periodic and C:1438 cubic_eval_uniform are the real script's
# kernels (R:1364, R:1415) verbatim.
from .real_field import cubic_eval_uniform, laplacian_periodic  # noqa: E402,F401
