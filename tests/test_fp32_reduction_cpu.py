"""The angle reductions of the FP32 Box-Muller transform (tipt_device.cuh:
half_turn_reduce, angle_reduce) against their direct form, in numpy float32:
the remainder t - q 2^k with q = round(t / 2^k) is the low k bits of t read as a
signed number, so (int)(t << (32 - k)) times (c 2^(k - 32)) gives the bits of
(float)(t - q 2^k) times c, and the parity of q is bit 31 of (t + 2^(k-1)) << 1."""
import numpy as np

C_HALF = np.float32(np.ldexp(0x1921FB6, -24 - 29 + 0))  # pi 2^-30 (0x1.921fb6p-29)
C_QUART = C_HALF                                        # (pi/2) 2^-29, the same bits


def _samples():
    rng = np.random.default_rng(5)
    t = rng.integers(0, 2 ** 31, size=1 << 22, dtype=np.uint64)
    edges = []
    for k in (28, 29, 30):
        for m in range(0, 2 ** 31, 1 << k):
            for d in (-2, -1, 0, 1, 2):
                if 0 <= m + d < 2 ** 31:
                    edges.append(m + d)
    edges += [0, 1, 2 ** 31 - 1, 2 ** 31 - 2]
    return np.concatenate([t, np.array(edges, dtype=np.uint64)]).astype(np.uint32)


def test_constant_is_pi_times_2_pow_minus_30():
    assert C_HALF == np.float32(np.pi * 2.0 ** -30)


def test_half_turn_reduction_bits():
    t = _samples()
    q = (t.astype(np.uint64) + (1 << 29)) >> 30
    rh = t.astype(np.int64) - (q << 30).astype(np.int64)
    x_ref = rh.astype(np.float32) * C_HALF
    s_ref = (q & 1).astype(np.uint32)
    r4 = (t << np.uint32(2)).view(np.int32)
    x_new = r4.astype(np.float32) * np.float32(C_HALF * np.float32(0.25))
    s_new = ((t + np.uint32(1 << 29)) << np.uint32(1)) >> np.uint32(31)
    assert np.array_equal(x_ref.view(np.uint32), x_new.view(np.uint32))
    assert np.array_equal(s_ref, s_new)


def test_quarter_turn_reduction_bits():
    t = _samples()
    q = (t.astype(np.uint64) + (1 << 28)) >> 29
    rh = t.astype(np.int64) - (q << 29).astype(np.int64)
    x_ref = rh.astype(np.float32) * C_QUART
    r8 = (t << np.uint32(3)).view(np.int32)
    x_new = r8.astype(np.float32) * np.float32(C_QUART * np.float32(0.125))
    assert np.array_equal(x_ref.view(np.uint32), x_new.view(np.uint32))
    assert np.all(np.abs(x_new) <= np.float32(np.pi / 4 + 1e-6))
