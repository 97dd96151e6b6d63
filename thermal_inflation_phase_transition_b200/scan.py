"""Surrogate-steered scans of the nucleation rate over the parameter box.

No reference counterpart: the reference scans parameters by running one lattice
per invocation.  The pipeline here:

1. ``generate_rows``: replicas with parameters drawn uniformly from the box
   (T/T0, E, D, lam) and a mix of lattice shapes run in the batched ensemble
   engine (retired at a high converted fraction so that the conversion curve
   runs on after the first passage); each replica gives one training row: its
   first-passage event flag, its exposure (volume x time to first passage or
   to censoring) and its converted fraction at 16 fixed times.
2. ``SurrogateNet.fit`` trains the network on those rows.
3. ``critical_lambda``: for each scan point (T/T0, E, D) the network proposes
   the quartic coupling lam* at which the mean first-passage time of a given
   lattice equals a target t* (Gamma V t* = 1), by bisection of its log Gamma.
4. ``verify``: every proposal is re-measured by a plain ensemble of
   ``n_verify`` replicas (the exponential MLE with censoring); the relative
   error of the surrogate's Gamma = 1/(V t*) against that estimate is the
   surrogate's error, the Poisson error of the estimate is stated beside it.
5. The cost of the steered scan (training rows + verification) is compared
   with a dense plain scan that runs ``n_verify`` replicas at every point of a
   lam grid of ``dense_lams`` values for every scan point.
"""
from __future__ import annotations

import math
import time

import numpy as np
import torch

from . import ensemble as EN
from .surrogate import N_CURVE, PARAM_BOX, SurrogateNet, features

__all__ = ["sample_box", "run_replicas", "training_rows", "critical_lambda", "choose_target",
           "verify", "dense_scan_cost", "steered_scan"]


def sample_box(n, rng):
    return {k: rng.uniform(lo, hi, n) for k, (lo, hi) in PARAM_BOX.items()}


def _volume(shape):
    return int(np.prod(shape))


def _dim(shape):
    return 2 if 1 in shape else 3


def run_replicas(shapes, T, E, D, lam, seeds, *, max_steps, dt=0.05, check_every=10,
                 retire_frac=0.95, batch_sites=1_500_000_000, storage="f32c",
                 record_curves=True, device="cuda"):
    """Run replicas in ensembles of at most batch_sites sites.  Returns (first_step[n],
    curves[n][16] or None, site_updates, seconds); curve k is the converted fraction
    after (k + 1) max_steps / 16 steps (max_steps must be a multiple of 16 check_every)."""
    n = len(shapes)
    K = max(2, check_every & ~1)
    if record_curves and max_steps % (N_CURVE * K):
        raise ValueError("max_steps must be a multiple of 16 * check_every")
    first = np.full(n, -1, np.int64)
    curves = np.zeros((n, N_CURVE)) if record_curves else None
    order = np.argsort([_volume(s) for s in shapes], kind="stable")
    site_updates = 0
    seconds = 0.0
    pos = 0
    while pos < n:
        idx, sites = [], 0
        while pos < n and (not idx or sites + _volume(shapes[order[pos]]) <= batch_sites):
            idx.append(int(order[pos]))
            sites += _volume(shapes[order[pos]])
            pos += 1
        specs = [EN.ReplicaSpec(tuple(shapes[i]), float(T[i]), float(E[i]), int(seeds[i]),
                                D=float(D[i]), lam=float(lam[i])) for i in idx]
        ens = EN.Ensemble(specs, storage=storage, dt=dt, check_every=K, stop_frac=0.5,
                          retire_frac=retire_frac, device=device)
        torch.cuda.synchronize(device)
        t0 = time.perf_counter()
        fs = ens.run(max_steps, poll_every=10, record_curves=record_curves)
        seconds += time.perf_counter() - t0
        first[idx] = fs
        # site updates actually spent: a replica stops costing once retired
        if ens.retire_frac == ens.stop_frac:
            steps_run = np.where(fs >= 0, fs + 1, ens.steps_done)
        else:
            steps_run = np.full(len(idx), ens.steps_done)
        if record_curves:
            steps, fr = ens.frac_curves()
            want = (np.arange(1, N_CURVE + 1) * max_steps // N_CURVE) - 1
            for k, s in enumerate(want):
                c = np.searchsorted(steps, s)
                curves[idx, k] = fr[min(c, len(steps) - 1)] if len(steps) else 0.0
            if ens.retire_frac != ens.stop_frac:
                over = fr > ens.retire_frac
                has = over.any(axis=0)
                steps_run = np.where(has, steps[np.argmax(over, axis=0)] + 1, ens.steps_done)
        site_updates += int(sum(_volume(specs[j].shape) * int(steps_run[j])
                                for j in range(len(idx))))
        del ens
        torch.cuda.empty_cache()
    return first, curves, site_updates, seconds


def training_rows(shapes, T, E, D, lam, first, curves, *, max_steps, dt, exposure_unit):
    """Network inputs x[n][6] and targets tgt[n][20] of replica results."""
    vol = np.array([_volume(s) for s in shapes], np.float64)
    dim = np.array([_dim(s) for s in shapes], np.float64)
    x = features(T, E, D, lam, vol, dim)
    ev = first >= 0
    t = np.where(ev, first + 1, max_steps) * dt
    tgt = np.zeros((len(shapes), 4 + N_CURVE), np.float32)
    tgt[:, 0] = ev
    tgt[:, 1] = vol * t / exposure_unit
    tgt[:, 2] = 1.0
    tgt[:, 3] = 1.0 if curves is not None else 0.0
    if curves is not None:
        tgt[:, 4:] = np.clip(curves, 0.0, 1.0)
    return x, tgt


def critical_lambda(net, T, E, D, volume, dim, t_target, *, iters=40):
    """lam in the box with surrogate Gamma(lam) V t_target = 1, by bisection (Gamma
    decreasing in lam is not assumed: the bracket is found on a grid first).  Returns
    (lam*, bracketed[bool])."""
    lo_b, hi_b = PARAM_BOX["lam"]
    target = -math.log(volume * t_target)
    T = np.atleast_1d(np.asarray(T, np.float64))
    E = np.broadcast_to(np.asarray(E, np.float64), T.shape)
    D = np.broadcast_to(np.asarray(D, np.float64), T.shape)
    grid = np.linspace(lo_b, hi_b, 33)
    n = T.size
    f = net.log_gamma(np.repeat(T, grid.size), np.repeat(E, grid.size), np.repeat(D, grid.size),
                      np.tile(grid, n), volume, dim).reshape(n, grid.size) - target
    lam_star = np.full(n, np.nan)
    ok = np.zeros(n, bool)
    a = np.empty(n)
    b = np.empty(n)
    for i in range(n):
        s = np.nonzero(np.sign(f[i, :-1]) != np.sign(f[i, 1:]))[0]
        if s.size:
            ok[i] = True
            a[i], b[i] = grid[s[0]], grid[s[0] + 1]
        else:
            a[i] = b[i] = grid[np.argmin(np.abs(f[i]))]
    fa = None
    for _ in range(iters):
        m = 0.5 * (a + b)
        fm = net.log_gamma(T, E, D, m, volume, dim) - target
        if fa is None:
            fa = net.log_gamma(T, E, D, a, volume, dim) - target
        same = np.sign(fm) == np.sign(fa)
        a = np.where(same & ok, m, a)
        fa = np.where(same & ok, fm, fa)
        b = np.where(~same & ok, m, b)
    lam_star = np.where(ok, 0.5 * (a + b), a)
    return lam_star, ok


def choose_target(net, T, E, D, volume, dim, candidates_steps, dt):
    """Among candidate target times (steps), the one for which the surrogate brackets lam*
    at the most scan points (ties: the shortest, which is cheapest to verify)."""
    lo_b, hi_b = PARAM_BOX["lam"]
    T = np.asarray(T, np.float64)
    g_lo = net.log_gamma(T, E, D, np.full(T.size, lo_b), volume, dim)
    g_hi = net.log_gamma(T, E, D, np.full(T.size, hi_b), volume, dim)
    best, best_n = candidates_steps[0], -1
    for c in sorted(candidates_steps):
        tgt = -math.log(volume * c * dt)
        n = int(np.sum((np.minimum(g_lo, g_hi) < tgt) & (tgt < np.maximum(g_lo, g_hi))))
        if n > best_n:
            best, best_n = c, n
    return best


def verify(shape, T, E, D, lam, *, n_verify=256, max_steps, dt=0.05, check_every=10,
           seed0=10_000_000, storage="f32c", batch_sites=1_500_000_000):
    """Plain-ensemble Gamma estimates (censored exponential MLE) at each point.
    Returns (gamma[n], n_events[n], site_updates, seconds)."""
    n = len(T)
    shapes = [tuple(shape)] * (n * n_verify)
    rep = lambda a: np.repeat(np.asarray(a, np.float64), n_verify)  # noqa: E731
    seeds = seed0 + np.arange(n * n_verify)
    first, _, su, sec = run_replicas(shapes, rep(T), rep(E), rep(D), rep(lam), seeds,
                                     max_steps=max_steps, dt=dt, check_every=check_every,
                                     retire_frac=0.5, record_curves=False, storage=storage,
                                     batch_sites=batch_sites)
    V = _volume(shape)
    gam = np.zeros(n)
    nev = np.zeros(n, np.int64)
    for i in range(n):
        g, _, k = EN.gamma_mle(first[i * n_verify:(i + 1) * n_verify], max_steps, V, dt)
        gam[i], nev[i] = g, k
    return gam, nev, su, sec


def dense_scan_cost(gamma_fn, T, E, D, *, volume, n_verify, max_steps, dt, dense_lams):
    """Site updates of a dense plain scan: n_verify replicas at each of dense_lams lam
    values per scan point, each replica running to its first passage or censoring
    (expected steps (1 - exp(-G V c)) / (G V) for rate G and censoring time c)."""
    grid = np.linspace(*PARAM_BOX["lam"], dense_lams)
    total = 0.0
    c = max_steps * dt
    for i in range(len(T)):
        g = np.exp(gamma_fn(np.full(dense_lams, T[i]), np.full(dense_lams, E[i]),
                            np.full(dense_lams, D[i]), grid))
        rate = g * volume
        mean_t = np.where(rate * c > 1e-9, -np.expm1(-rate * c) / np.maximum(rate, 1e-300), c)
        total += float((n_verify * volume * mean_t / dt).sum())
    return total


def steered_scan(*, n_train=20000, train_shapes=((128, 128, 1), (48, 48, 48), (64, 64, 64)),
                 train_mix=(0.3, 0.3, 0.4), scan_shape=(64, 64, 64), n_points=64,
                 t_target_steps=None, train_steps=4800, verify_steps=None, n_verify=256,
                 dense_lams=16, dt=0.05, fit_iters=3000, seed=5, log=print):
    """The full pipeline (module docstring); returns a report dict."""
    rng = np.random.default_rng(seed)
    report = {}
    # 1. training rows from the ensemble engine
    mix = np.asarray(train_mix, np.float64) / np.sum(train_mix)
    which = rng.choice(len(train_shapes), n_train, p=mix)
    shapes = [tuple(train_shapes[w]) for w in which]
    box = sample_box(n_train, rng)
    seeds = np.arange(n_train) + 1_000_000 * (seed + 1)
    first, curves, su_train, sec_train = run_replicas(
        shapes, box["T"], box["E"], box["D"], box["lam"], seeds, max_steps=train_steps, dt=dt)
    log(f"training rows: {n_train} replicas, {int((first >= 0).sum())} events, "
        f"{su_train:.3e} site updates in {sec_train:.1f} s")
    exposure_unit = float(_volume(scan_shape)) * train_steps * dt / 8.0
    x, tgt = training_rows(shapes, box["T"], box["E"], box["D"], box["lam"], first, curves,
                           max_steps=train_steps, dt=dt, exposure_unit=exposure_unit)
    # 2. training (held-out tenth for the validation loss)
    n_val = n_train // 10
    net = SurrogateNet(seed=seed, exposure_unit=exposure_unit, horizon=train_steps * dt)
    ev_rate = tgt[:, 0].sum() / tgt[:, 1].sum()
    with torch.no_grad():
        b3 = net.params.numel() - 32
        net.params[b3] = float(np.log(max(ev_rate, 1e-6)))
        mc = np.clip(tgt[:, 4:].mean(axis=0), 1e-3, 1 - 1e-3)
        net.params[b3 + 1:b3 + 17] = torch.from_numpy(np.log(mc / (1 - mc)).astype(np.float32))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    hist = net.fit(x[n_val:], tgt[n_val:], iters=fit_iters, lr=2e-3, lr_final=5e-5,
                   batch=min(4096, n_train - n_val), seed=seed)
    sec_fit = time.perf_counter() - t0
    report["fit"] = {"rows": n_train - n_val, "iters": fit_iters, "seconds": sec_fit,
                     "loss_first": float(hist[0]), "loss_last": float(hist[-1]),
                     "val_loss": net.loss(x[:n_val], tgt[:n_val])}
    log(f"fit: {fit_iters} iters in {sec_fit:.1f} s, loss {hist[0]:.4f} -> {hist[-1]:.4f}, "
        f"validation {report['fit']['val_loss']:.4f}")
    # 3. proposals on a (T, E, D) grid: 4 x 4 x 4 points, lam* from the surrogate
    m = round(n_points ** (1 / 3))
    axes = [np.linspace(*PARAM_BOX[k], m + 2)[1:-1] for k in ("T", "E", "D")]
    TT, EE, DD = (a.reshape(-1) for a in np.meshgrid(*axes, indexing="ij"))
    V = _volume(scan_shape)
    dim = _dim(scan_shape)
    if t_target_steps is None:
        t_target_steps = choose_target(net, TT, EE, DD, V, dim,
                                       [train_steps // 16 * k for k in range(1, 9)], dt)
    if verify_steps is None:
        # censoring at four mean first-passage times: about 98 % of replicas convert
        verify_steps = 4 * t_target_steps
    report["target_steps"] = t_target_steps
    report["verify_steps"] = verify_steps
    t_target = t_target_steps * dt
    lam_star, ok = critical_lambda(net, TT, EE, DD, V, dim, t_target)
    report["proposals"] = {"points": int(TT.size), "bracketed": int(ok.sum())}
    log(f"proposals: {int(ok.sum())}/{TT.size} bracketed in lam")
    sel = np.nonzero(ok)[0]
    # 4. verification by plain ensembles
    g_hat, n_ev, su_ver, sec_ver = verify(scan_shape, TT[sel], EE[sel], DD[sel], lam_star[sel],
                                          n_verify=n_verify, max_steps=verify_steps, dt=dt)
    g_sur = np.exp(net.log_gamma(TT[sel], EE[sel], DD[sel], lam_star[sel], V, dim))
    rel = g_sur / g_hat - 1.0
    poisson = 1.0 / np.sqrt(np.maximum(n_ev, 1))
    report["verify"] = {
        "points": int(sel.size), "replicas_per_point": n_verify, "seconds": sec_ver,
        "site_updates": su_ver,
        "median_abs_rel_err": float(np.median(np.abs(rel))),
        "mean_abs_rel_err": float(np.mean(np.abs(rel))),
        "frac_within_10pct": float(np.mean(np.abs(rel) <= 0.10)),
        "median_poisson_err": float(np.median(poisson)),
        "frac_within_10pct_or_2sigma": float(np.mean(np.abs(rel) <= np.maximum(0.10, 2 * poisson))),
        "events_median": float(np.median(n_ev)),
        "rows": [{"T": float(TT[i]), "E": float(EE[i]), "D": float(DD[i]),
                  "lam": float(lam_star[i]), "gamma_surrogate": float(g_sur[k]),
                  "gamma_plain": float(g_hat[k]), "events": int(n_ev[k])}
                 for k, i in enumerate(sel)]}
    log(f"verify: median |err| {report['verify']['median_abs_rel_err']:.3f}, within 10%: "
        f"{report['verify']['frac_within_10pct']:.2f}, median Poisson err "
        f"{report['verify']['median_poisson_err']:.3f}")
    # 5. cost against a dense plain scan of the same points
    rate_sites = (su_train + su_ver) / max(sec_train + sec_ver, 1e-9)
    dense_su = dense_scan_cost(lambda T_, E_, D_, L_: net.log_gamma(T_, E_, D_, L_, V, dim),
                               TT[sel], EE[sel], DD[sel], volume=V, n_verify=n_verify,
                               max_steps=verify_steps, dt=dt, dense_lams=dense_lams)
    steered_s = sec_train + sec_fit + sec_ver
    dense_s = dense_su / rate_sites
    report["cost"] = {
        "steered_gpu_hours": steered_s / 3600.0, "dense_gpu_hours": dense_s / 3600.0,
        "saved_gpu_hours": (dense_s - steered_s) / 3600.0, "ratio": dense_s / steered_s,
        "dense_site_updates": dense_su, "steered_site_updates": su_train + su_ver,
        "engine_site_updates_per_s": rate_sites, "dense_lams": dense_lams}
    log(f"cost: steered {steered_s:.0f} s vs dense {dense_s:.0f} s "
        f"({dense_s / steered_s:.1f}x)")
    report["net"] = net
    return report
