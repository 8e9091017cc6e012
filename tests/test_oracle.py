"""The CPU oracle, pinned against the reference's own outputs (tests/golden/,
generated by tests/golden/make_fixtures.py from the reference compiled from
its sources) and against the known answers of the reference's code."""
import math
import os

import numpy as np
import pytest

from oracle import core


def test_material_table_matches_reference(golden_dir):
    g = np.load(os.path.join(golden_dir, "ref_materials.npz"))
    assert int(g["composite_count"]) == 254
    ours = core.material_table()
    assert np.array_equal(ours.view(np.uint32), g["table"].view(np.uint32))


def test_decode_matches_reference(golden_dir):
    g = np.load(os.path.join(golden_dir, "ref_materials.npz"))
    ours = np.array([core.decode_id(int(e)) for e in g["encodings"]])
    assert np.array_equal(ours, g["ids"])


def test_material_encoding_kat():
    # common/tests/test_simulator.cpp:65-81: decode is the identity for air,
    # bone and adductor_muscle0, and air|bone decodes to air.
    assert core.decode_id(1 << 0) == 0
    assert core.decode_id(1 << 22) == 22
    assert core.decode_id(1 << 1) == 1
    assert core.decode_id((1 << 0) | (1 << 22)) == 0


def test_composite_id_numbering():
    L = core.lib()
    ids = {L.or_composite_id(i, j) for i in range(1, 23) for j in range(i, 23)}
    assert ids == set(range(1, 254))
    assert L.or_composite_id(0, 5) == 0
    assert L.or_composite_id(21, 22) == 253


@pytest.mark.parametrize("duration,steps", [(0.5, 5001), (1.0, 10000), (2.0, 19998), (10.0, 99937)])
def test_step_count_kat(duration, steps):
    # Simulator.cu:428-449 accumulates the remaining time in float.
    assert core.step_count(duration, 1e-4) == steps
    rem, n = np.float32(duration), 0
    dt = np.float32(1e-4)
    while rem > 0:
        rem = np.float32(rem - dt)
        n += 1
    assert n == steps


def test_clock_accumulates_in_float():
    t = np.float32(0)
    for _ in range(1234):
        t = np.float32(t + np.float32(1e-3))
    assert core.advance_clock(0.0, 1e-3, 1234) == pytest.approx(float(t), abs=0)


def test_sin_within_one_ulp_of_libm():
    rng = np.random.default_rng(3)
    xs = np.concatenate([np.linspace(-150.0, 150.0, 30001), rng.uniform(-1e4, 1e4, 20000)])
    for x in xs:
        s = core.sin(float(x))
        ref = math.sin(float(x))
        assert abs(s - ref) <= 2.3e-16, x
        assert np.float32(s) == np.float32(ref), x


def _small_batch():
    from mercury_b200 import robots
    return robots.population_batch("small", 6)


def test_fp32_tracks_fp64():
    import mercury_b200 as mb
    b = _small_batch()
    table = mb.material_table()
    p, v = b.pos.copy(), b.vel.copy()
    s = np.zeros(b.n_springs, np.float32)
    core.xpbd_run(b, p, v, s, table, 1e-3, 0.0, 500, True)
    pd, vd = b.pos.astype(np.float64), b.vel.astype(np.float64)
    sd = np.zeros(b.n_springs)
    core.xpbd_run_f64(b, pd, vd, sd, table, 1e-3, 0.0, 500, True)
    # FP32 rounding grows with the chaotic dynamics: within 5e-4 m on ~0.4 m bodies after 500 steps
    assert np.abs(p[:, :3] - pd[:, :3]).max() < 5e-4
    assert np.abs(s - sd).max() < 1e-4 * max(1.0, np.abs(sd).max())


def test_robots_are_independent():
    """Simulating robots together or one by one gives the same bits."""
    import mercury_b200 as mb
    from mercury_b200.element import pack
    from mercury_b200 import robots
    els = robots.population("uneven", 5)
    table = mb.material_table()
    b = pack(els)
    p, v, s = b.pos.copy(), b.vel.copy(), np.zeros(b.n_springs, np.float32)
    core.xpbd_run(b, p, v, s, table, 5e-3, 0.0, 200, True)
    for r, e in enumerate(els):
        bi = pack([e])
        pi, vi, si = bi.pos.copy(), bi.vel.copy(), np.zeros(bi.n_springs, np.float32)
        core.xpbd_run(bi, pi, vi, si, table, 5e-3, 0.0, 200, True)
        ms, ss = b.robot_slices(r)
        assert np.array_equal(p[ms], pi) and np.array_equal(v[ms], vi) and np.array_equal(s[ss], si)


def test_momentum_is_conserved():
    """Equal masses and +dp/-dp pairs: the mean velocity only decays by the
    0.99 damping factor, up to position rounding (which quantises velocities
    to ulp(x)/dt, so the check uses dt = 1e-3 and a 1% tolerance)."""
    import mercury_b200 as mb
    b = _small_batch()
    p, v = b.pos.copy(), b.vel.copy()
    v[:, :3] = 0.01
    s = np.zeros(b.n_springs, np.float32)
    steps = 100
    core.xpbd_run(b, p, v, s, mb.material_table(), 1e-3, 0.0, steps, False)
    for r in range(b.n_robots):
        ms, _ = b.robot_slices(r)
        mean_v = v[ms, :3].astype(np.float64).mean(axis=0)
        assert np.allclose(mean_v, 0.01 * 0.99 ** steps, rtol=1e-2)


def test_com_device_order_close_to_reference_running_mean():
    b = _small_batch()
    a = core.com_device(b, b.pos)
    r = core.com_reference(b, b.pos)
    assert np.allclose(a, r, atol=1e-6)


def _golden_cases(golden_dir):
    g = np.load(os.path.join(golden_dir, "ref_sim.npz"))
    for i in range(int(g["n_cases"])):
        yield {k: g[f"c{i}_{k}"] for k in ("flavour", "dt", "duration", "steps", "total_time", "pos", "vel", "stress")}


def test_oracle_matches_reference_cuda_fixture(golden_dir):
    """The oracle against the reference's own CUDA step (both builds), run on
    a B200 by tests/golden/make_fixtures.py: same step count and clock, and
    positions within 2e-4 x body length."""
    import mercury_b200 as mb
    from mercury_b200 import robots
    b = robots.population_batch("small", 8)
    length = mb.body_length(b)
    table = mb.material_table()
    for c in _golden_cases(golden_dir):
        dt, dur = float(c["dt"]), float(c["duration"])
        n = core.step_count(dur, dt)
        assert n == int(c["steps"])
        assert core.advance_clock(0.0, dt, n) == float(c["total_time"])
        p, v = b.pos.copy(), b.vel.copy()
        s = np.zeros(b.n_springs, np.float32)
        core.xpbd_run(b, p, v, s, table, dt, 0.0, n, True)
        for r in range(b.n_robots):
            ms, ss = b.robot_slices(r)
            dx = np.abs(p[ms, :3] - c["pos"][ms]).max() / length[r]
            assert dx < 2e-4, (c["flavour"], dt, r, dx)
        rel = np.abs(s - c["stress"]).max() / max(np.abs(c["stress"]).max(), 1e-12)
        assert rel < 1e-2, (c["flavour"], dt, rel)
