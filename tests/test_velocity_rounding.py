"""The division-free velocity update of the step kernels (velocity_of in
mb_kernels.cu): v = (float)(0.99 * (double)d / (double)dt), the reference
step's velocity (sim_kernel.cu:265-267), evaluated as q = RN(a * RN(1/dt))
with Ziv's rounding test and the division as fallback.  Here the method
itself, emulated in numpy float64 (IEEE round to nearest), is checked
against the division on inputs next to float rounding midpoints
(tests/golden/velocity_midpoints.npz, made by make_velocity_midpoints.py)
and on random inputs of every magnitude."""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "velocity_midpoints.npz")


def reference(d, dt):
    with np.errstate(all="ignore"):
        a = np.float64(0.99) * np.asarray(d, np.float32).astype(np.float64)
        return (a / np.float64(np.float32(dt))).astype(np.float32)


def division_free(d, dt):
    """Returns (value, fast) like the kernel: fast where the test clears."""
    with np.errstate(all="ignore"):
        return _division_free(d, dt)


def _division_free(d, dt):
    a = np.float64(0.99) * np.asarray(d, np.float32).astype(np.float64)
    ddt = np.float64(np.float32(dt))
    q = a * (np.float64(1.0) / ddt)
    bits = q.view(np.uint64)
    e = ((bits >> np.uint64(52)) & np.uint64(0x7FF)).astype(np.int64)
    low = (bits & np.uint64(0x1FFFFFFF)).astype(np.int64)
    clear = (e >= 897) & (e <= 1149) & (np.abs(low - (1 << 28)) > 4)
    zero = (bits << np.uint64(1)) == 0
    fast = clear | zero
    return np.where(fast, q.astype(np.float32), (a / ddt).astype(np.float32)), fast


def same_bits(x, y):
    return np.array_equal(np.asarray(x, np.float32).view(np.uint32), np.asarray(y, np.float32).view(np.uint32))


def test_midpoint_inputs_take_the_division():
    g = np.load(GOLDEN)
    n = 0
    for i in range(len([k for k in g.files if k.startswith("dt")])):
        dt, d = float(g[f"dt{i}"][0]), g[f"d{i}"]
        assert len(d) > 0
        z = (np.float64(0.99) * d.astype(np.float64)) / np.float64(np.float32(dt))
        low = (z.view(np.uint64) & np.uint64(0x1FFFFFFF)).astype(np.int64)
        assert (np.abs(low - (1 << 28)) <= 4).all()
        v, fast = division_free(d, dt)
        assert same_bits(v, reference(d, dt))
        assert not fast.any()
        n += len(d)
    assert n >= 40


def test_random_inputs_of_every_magnitude():
    rng = np.random.default_rng(0)
    bits = rng.integers(0, 1 << 32, 2_000_000, dtype=np.uint64).astype(np.uint32)
    d = bits.view(np.float32)
    d = d[np.isfinite(d)]
    for dt in (1e-4, 1e-3, 3.7e-4, 1e-2):
        v, fast = division_free(d, dt)
        assert same_bits(v, reference(d, dt))
        assert fast.mean() > 0.6  # the rest: outside the float range after scaling


def test_zeros_and_specials():
    d = np.array([0.0, -0.0, np.inf, -np.inf, np.nan, 1e-45, -1e-45, 3.4e38, -3.4e38,
                  1.1754944e-38, 2.0 ** -126], np.float32)
    for dt in (1e-4, 1e-3):
        v, _ = division_free(d, dt)
        r = reference(d, dt)
        assert same_bits(v[~np.isnan(r)], r[~np.isnan(r)])
        assert np.isnan(v[np.isnan(r)]).all()
        assert same_bits(v[:2], np.array([0.0, -0.0], np.float32))
