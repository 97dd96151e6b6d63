"""Snapshot/checkpoint files in the reference's .npz layout (host tensors; the
GPU path is covered by tests/test_gpu_snapshots.py)."""
import numpy as np
import torch

from thermal_inflation_phase_transition_b200 import snapshots as SN
from thermal_inflation_phase_transition_b200.real_field import to_f32c

REAL_KEYS = {"phi", "step", "time", "temperature", "phi_min", "phi_max"}
CPLX_KEYS = {"phi1", "phi2", "rho", "theta", "winding", "step", "time", "temperature",
             "rho_min", "rho_max", "zn_active"}


def test_real_schema_and_checkpoint_cadence(tmp_path):
    w = SN.SnapshotWriter(str(tmp_path), checkpoint_every=3)
    rng = np.random.default_rng(0)
    phi = torch.from_numpy(rng.normal(size=(4, 5, 6)))
    pi = torch.from_numpy(rng.normal(size=(4, 5, 6)))
    for n in range(7):
        w.save_real(100 * n, 0.5 * n, 1.02, phi, pi, energies=(1.0, 2.0, 3.0))
    w.wait()
    for n in range(7):
        with np.load(SN.snapshot_name(str(tmp_path), 100 * n)) as z:
            keys = set(z.files)
            assert REAL_KEYS | {"E_kin", "E_grad", "E_pot"} <= keys
            assert ("pi" in keys) == (n % 3 == 0)
            assert int(z["step"]) == 100 * n and float(z["temperature"]) == 1.02
            np.testing.assert_array_equal(z["phi"], phi.numpy())
            assert float(z["phi_max"]) == phi.max().item()


def test_latest_checkpoint_skips_nan_and_pi_less(tmp_path):
    w = SN.SnapshotWriter(str(tmp_path), checkpoint_every=2, background=False)
    good = torch.ones((2, 2, 2), dtype=torch.float64)
    bad = good.clone()
    bad[0, 0, 0] = float("nan")
    w.save_real(10, 0, 1, good, good)   # checkpoint
    w.save_real(20, 0, 1, good, good)   # no pi
    w.save_real(30, 0, 1, bad, good)    # checkpoint with NaN phi
    w.save_real(40, 0, 1, good, good)   # no pi
    path, d = SN.latest_checkpoint(str(tmp_path))
    assert path.endswith("state_step_0000000010.npz") and int(d["step"]) == 10
    path, d = SN.latest_checkpoint(str(tmp_path), need_pi=False)
    assert int(d["step"]) == 40


def test_f32c_round_trip_is_exact(tmp_path):
    rng = np.random.default_rng(1)
    x = torch.from_numpy(rng.normal(size=(3, 4, 5)) * 7.0)
    s = to_f32c(x)
    w = SN.SnapshotWriter(str(tmp_path), background=False)
    w.save_real(5, 0.1, 1.0, s, s)
    _, d = SN.latest_checkpoint(str(tmp_path))
    assert d["phi"].dtype == np.float64 and "phi_lo" in d
    back = SN.load_fields(d, ["phi", "pi"], "f32c", device="cpu")
    assert torch.equal(back[0], s) and torch.equal(back[1], s)


def test_complex_schema(tmp_path):
    rng = np.random.default_rng(2)
    a = torch.from_numpy(rng.normal(size=(3, 4, 5)))
    b = torch.from_numpy(rng.normal(size=(3, 4, 5)))
    w = SN.SnapshotWriter(str(tmp_path), background=False)
    wind = np.zeros((3, 4, 5), np.float32)
    w.save_complex(7, 0.2, 0.98, a, b, a, b, zn_active=1.0, winding=wind)
    with np.load(SN.snapshot_name(str(tmp_path), 7)) as z:
        assert CPLX_KEYS | {"pi1", "pi2"} <= set(z.files)
        assert z["rho"].dtype == np.float32 and z["theta"].dtype == np.float32
        np.testing.assert_allclose(z["rho"], np.hypot(a.numpy(), b.numpy()).astype(np.float32))
        assert float(z["zn_active"]) == 1.0
    p = SN.write_metadata(str(tmp_path), Nx=3, Ny=4, Nz=5, dt=0.05, integrator="rk2_nonfused")
    with np.load(p) as z:
        assert int(z["Nx"]) == 3 and str(z["integrator"]) == "rk2_nonfused"


def test_compressed_and_stored_archives_hold_the_same_arrays(tmp_path):
    """compress=True deflates the members as the reference's np.savez_compressed;
    the default stores them; np.load returns the same keys and arrays."""
    import zipfile
    rng = np.random.default_rng(1)
    phi = to_f32c(torch.from_numpy(rng.normal(size=(3, 4, 8))))
    pi = to_f32c(torch.from_numpy(rng.normal(size=(3, 4, 8))))
    out = {}
    for comp in (False, True):
        d = tmp_path / str(comp)
        w = SN.SnapshotWriter(str(d), background=False, compress=comp)
        path = w.save_real(5, 0.25, 1.0, phi, pi)
        with zipfile.ZipFile(path) as zf:
            kinds = {i.compress_type for i in zf.infolist()}
        assert kinds == ({zipfile.ZIP_DEFLATED} if comp else {zipfile.ZIP_STORED})
        with np.load(path) as z:
            out[comp] = {k: z[k] for k in z.files}
    assert out[False].keys() == out[True].keys()
    for k in out[False]:
        np.testing.assert_array_equal(out[False][k], out[True][k])
