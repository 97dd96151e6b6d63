"""Long-run statistical parity with the reference: the mean nucleation time and
the string density of long runs agree with the reference's own kernels within
the ensembles' statistical error (trajectories of two implementations cannot be
compared step by step over thousands of steps: rounding differences grow, so
the comparison is of ensemble statistics).

The reference side is tests/golden/longrun.npz (make_golden_longrun.py): 64
real-field replicas stepped by the reference's rk2_step_table (R:1875-1966) on
float32 arrays until the converted fraction exceeds 1/2, and 16 complex-field
quenches stepped by its complex rk2_step_table (C:2067-2215) with the string
voxel fraction of compute_winding_number (C:2683-2744, tools/winding.py:67-70)
every 100 steps.  This side runs independent replicas (other seeds) through the
batched ensemble engine and the compensated-FP32 complex stepper."""
import math

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from thermal_inflation_phase_transition_b200 import complex_field as CF  # noqa: E402
from thermal_inflation_phase_transition_b200 import ensemble as EN  # noqa: E402
from thermal_inflation_phase_transition_b200 import real_field as RF  # noqa: E402
from thermal_inflation_phase_transition_b200._common import table_source  # noqa: E402

N_REAL = 256
N_CPLX = 32


def test_mean_nucleation_time_vs_reference(golden):
    g = golden("longrun.npz")
    T, shape = float(g["real_T"]), tuple(int(x) for x in g["real_shape"])
    max_steps, K = int(g["real_max_steps"]), int(g["real_check_every"])
    specs = [EN.ReplicaSpec(shape, T, 0.05, 5001 + r) for r in range(N_REAL)]
    ens = EN.Ensemble(specs, storage="f32c", thr=float(g["real_thr"]),
                      stop_frac=float(g["real_stop_frac"]), check_every=K, init_seed=9)
    f_gpu = ens.run(max_steps, poll_every=5)
    f_ref = g["real_first_passage"]
    # the same check convention: a first passage is the last step of a check interval
    for f in (f_gpu, f_ref):
        assert ((f[f >= 0] + 1) % K == 0).all()
    # both sides are censored at the same max_steps: compare the first-passage
    # times restricted to max_steps (a replica still unconverted counts max_steps)
    ref = np.where(f_ref >= 0, f_ref + 1, max_steps).astype(np.float64)
    fs = np.where(f_gpu >= 0, f_gpu + 1, max_steps).astype(np.float64)
    assert (f_ref >= 0).mean() > 0.9 and (f_gpu >= 0).mean() > 0.9
    mr, sr = ref.mean(), ref.std(ddof=1)
    mg, sg = fs.mean(), fs.std(ddof=1)
    se = math.sqrt(sr ** 2 / ref.size + sg ** 2 / fs.size)
    assert abs(mg - mr) < 3.0 * se, (mg, mr, se)
    # the spread too: the sample standard deviations within three of their standard errors
    se_s = math.sqrt(sr ** 2 / (2 * (ref.size - 1)) + sg ** 2 / (2 * (fs.size - 1)))
    assert abs(sg - sr) < 3.0 * se_s, (sg, sr, se_s)
    # and the whole first-passage distribution: two-sample Kolmogorov-Smirnov
    from scipy.stats import ks_2samp
    assert ks_2samp(ref, fs).pvalue > 1e-3


def test_string_density_vs_reference(golden):
    g = golden("longrun.npz")
    ref = g["complex_string_fraction"]  # [replica][checkpoint]
    T, shape = float(g["complex_T"]), tuple(int(x) for x in g["complex_shape"])
    steps, every = int(g["complex_steps"]), int(g["complex_every"])
    dt = 0.05
    ns = math.sqrt(2.0 * T * dt)
    x = torch.linspace(0.0, 4.0, 4096, dtype=torch.float64, device="cuda")
    tab = 2.0 * 0.1 * (T * T - 1.0) * x - 3.0 * 0.05 * T * x * x + 0.1 * x ** 3
    vs = table_source(tab, 0.0, 4095 / 4.0, 4096)
    n_sites = shape[0] * shape[1] * shape[2]
    got = np.zeros((N_CPLX, steps // every))
    for r in range(N_CPLX):
        seed = 6001 + r
        gen = torch.Generator(device="cuda").manual_seed(seed)
        th = (torch.rand(shape, dtype=torch.float64, device="cuda", generator=gen) * 2 - 1) \
            * math.pi
        rho = 0.05 * torch.abs(1.0 + 0.3 * torch.randn(shape, dtype=torch.float64, device="cuda",
                                                        generator=gen))
        st = [RF.to_f32c(rho * torch.cos(th)), RF.to_f32c(rho * torch.sin(th)),
              torch.zeros((2,) + shape, dtype=torch.float32, device="cuda"),
              torch.zeros((2,) + shape, dtype=torch.float32, device="cuda")]
        out = [torch.empty_like(a) for a in st]
        for n in range(steps):
            CF.rk2_step_table_into(st, out, dt, 1.0, 1.0, 1.0, 1.0, vs, noise_scale=ns,
                                   noise_step=n, seed=seed)
            st, out = out, st
            if (n + 1) % every == 0:
                res = CF.compute_winding_number_full(st[0], st[1], w_site=True, w3=False)
                got[r, (n + 1) // every - 1] = res.host_counts()["n_strings"] / n_sites
    mr, mg = ref.mean(0), got.mean(0)
    se = np.sqrt(ref.var(0, ddof=1) / ref.shape[0] + got.var(0, ddof=1) / got.shape[0])
    assert (np.abs(mg - mr) < 4.0 * se).all(), (mg, mr, se)
    assert mr[-1] > 0.005  # a string network is still present at the end
