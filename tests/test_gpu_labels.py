"""GPU connected-component labelling against scipy.ndimage.label (the
reference's post-processing labeller) and the reference's per-cluster formulas
(postprocess/revisualize_snapshots.py:171-214, :360-392)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
ndimage = pytest.importorskip("scipy.ndimage")

pytestmark = pytest.mark.gpu

from thermal_inflation_phase_transition_b200 import labels as LB  # noqa: E402
from thermal_inflation_phase_transition_b200.real_field import to_f32c  # noqa: E402


@pytest.mark.parametrize("shape,density", [((20, 17, 13), 0.2), ((20, 17, 13), 0.35),
                                           ((64, 64, 64), 0.3), ((1, 40, 50), 0.5),
                                           ((33, 1, 70), 0.6), ((96, 96, 96), 0.25)])
def test_labels_equal_scipy(shape, density):
    rng = np.random.default_rng(int(density * 100) + shape[0])
    f = rng.uniform(-1.0, 1.0, shape)
    thr = 1.0 - density
    lab, n = LB.label(torch.from_numpy(f).cuda(), thr)
    ref, nref = ndimage.label(np.abs(f) > thr)
    assert n == nref
    np.testing.assert_array_equal(lab.cpu().numpy(), ref)


def test_periodic_joins_across_the_boundary():
    f = np.zeros((6, 6, 6))
    f[0, 2, 2] = f[5, 2, 2] = 1.0           # neighbours only through the x wrap
    f[3, 0, 4] = f[3, 5, 4] = 1.0           # through the y wrap
    f[1, 1, 0] = f[1, 1, 5] = 1.0           # through the z wrap
    t = torch.from_numpy(f).cuda()
    _, n_open = LB.label(t, 0.5)
    lab, n_per = LB.label(t, 0.5, periodic=True)
    assert n_open == 6 and n_per == 3
    lab = lab.cpu().numpy()
    assert lab[0, 2, 2] == lab[5, 2, 2] and lab[3, 0, 4] == lab[3, 5, 4]


def test_bubbles_match_reference_formulas():
    rng = np.random.default_rng(7)
    phi = rng.normal(0.0, 1.0, (40, 36, 30))
    phi = ndimage.gaussian_filter(phi, 1.5) * 8.0
    esc = 1.0
    got = LB.identify_bubbles(to_f32c(torch.from_numpy(phi).cuda()), esc, dx_phys=0.5)
    mask = np.abs(phi) > esc
    lab, n = ndimage.label(mask)
    ref = []
    for cid in range(1, n + 1):
        coords = np.argwhere(lab == cid)
        vol = len(coords)
        c = coords.mean(axis=0)
        vals = phi[lab == cid]
        ref.append(dict(centroid=c, volume=vol, r_eff=(3.0 * vol / (4.0 * np.pi)) ** (1 / 3),
                        r_rms=np.sqrt(np.mean(np.sum((coords - c) ** 2, axis=1))),
                        sign=1 if np.mean(vals) >= 0 else -1, peak=float(np.max(np.abs(vals)))))
    ref.sort(key=lambda b: b["volume"], reverse=True)
    assert len(got) == len(ref) > 3
    for a, b in zip(got, ref):
        assert a["volume"] == b["volume"] and a["sign"] == b["sign"]
        np.testing.assert_allclose(a["centroid"], b["centroid"], rtol=0, atol=1e-12)
        assert abs(a["r_rms"] - b["r_rms"]) < 1e-9 and abs(a["r_eff"] - b["r_eff"]) < 1e-12
        assert abs(a["peak"] - b["peak"]) <= 1e-12 * b["peak"]
        assert abs(a["r_phys"] - 0.5 * b["r_eff"]) < 1e-12


def test_strings_match_reference_formulas():
    rng = np.random.default_rng(9)
    w = rng.choice([-1.0, 0.0, 0.0, 0.0, 1.0, 2.0], size=(24, 24, 24)).astype(np.float32)
    lab_g, got = LB.identify_strings(torch.from_numpy(w).cuda())
    mask = np.abs(w) > 0.5
    lab, n = ndimage.label(mask)
    np.testing.assert_array_equal(lab_g, lab)
    labels = np.arange(1, n + 1)
    counts = np.bincount(lab.ravel(), minlength=n + 1)[1:]
    centers = ndimage.center_of_mass(mask, lab, labels)
    means = ndimage.mean(w, lab, labels)
    maxes = ndimage.maximum(np.abs(w), lab, labels)
    ref = [dict(loop_id=int(l), n_voxels=int(counts[i]), centroid=np.asarray(centers[i]),
                winding_sign=1 if float(means[i]) >= 0 else -1, max_winding=float(maxes[i]))
           for i, l in enumerate(labels)]
    ref.sort(key=lambda s: s["n_voxels"], reverse=True)
    assert len(got) == len(ref)
    for a, b in zip(got, ref):
        assert (a["loop_id"], a["n_voxels"], a["winding_sign"]) == \
               (b["loop_id"], b["n_voxels"], b["winding_sign"])
        assert a["max_winding"] == b["max_winding"]
        np.testing.assert_allclose(a["centroid"], b["centroid"], rtol=0, atol=1e-12)
