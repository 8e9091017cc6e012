"""The step kernels' division-free velocity update on the device, bit for
bit against the division (sim_kernel.cu:265-267) and the oracle, on
displacements next to float rounding midpoints and random ones: masses
without active springs at the origin move by exactly RN(v dt) in one
step, so the displacement the kernel divides is chosen through v."""
import os

import numpy as np
import pytest

import mercury_b200 as mb
from mercury_b200.materials import material_table
from oracle import core

from test_velocity_rounding import reference, same_bits

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "velocity_midpoints.npz")


def velocities_for(d, dt):
    """v with RN_f(v * dt) == d, or None when no float v gives d."""
    dt32 = np.float32(dt)
    out, keep = [], []
    for x in np.asarray(d, np.float32):
        v = np.float32(np.float64(x) / np.float64(dt32))
        hit = None
        for _ in range(8):
            p = np.float32(v * dt32)
            if p == x:
                hit = v
                break
            v = np.nextafter(v, np.float32(np.inf) if p < x else np.float32(-np.inf), dtype=np.float32)
        if hit is not None:
            out.append(hit)
            keep.append(x)
    return np.array(keep, np.float32), np.array(out, np.float32)


def run_one_step(disp, dt, streamed=False, per_robot=400):
    d, v = velocities_for(disp, dt)
    assert len(d) >= 0.8 * len(disp)
    pad = (-len(d)) % 3
    d = np.concatenate([d, np.full(pad, 0.5, np.float32)])
    v = np.concatenate([v, velocities_for(np.full(pad, 0.5, np.float32), dt)[1]])
    vel = v.reshape(-1, 3)
    els = []
    for i in range(0, len(vel), per_robot):
        m = len(vel[i:i + per_robot])
        els.append(mb.Element(np.zeros((m, 3), np.float32), np.ones(m, np.uint8), np.array([[0, 1 if m > 1 else 0]]),
                              np.ones(1, np.float32), np.zeros(1, np.uint8), vel=vel[i:i + per_robot]))
    b = mb.pack(els)
    sim = mb.Simulator(0)
    sim.setTimeStep(dt)
    if streamed:
        sim.set_launch_config(streamed=1)
    sim.set_batch(b)
    sim.run_steps(1, False)
    pos, got, _ = sim.collect_arrays()
    assert same_bits(pos[:, :3].reshape(-1), d)  # the displacement is what was asked for
    p, vv, s = b.pos.copy(), b.vel.copy(), np.zeros(b.n_springs, np.float32)
    core.xpbd_run(b, p, vv, s, material_table(), np.float32(dt), 0.0, 1, False)
    return got[:, :3].reshape(-1), vv[:, :3].reshape(-1), reference(d, dt)


@pytest.mark.parametrize("streamed", [False, True], ids=["resident", "streamed"])
def test_midpoint_displacements(streamed):
    g = np.load(GOLDEN)
    for i in range(len([k for k in g.files if k.startswith("dt")])):
        dt, disp = float(g[f"dt{i}"][0]), g[f"d{i}"]
        got, orc, ref = run_one_step(disp, dt, streamed)
        assert same_bits(got, ref)
        assert same_bits(got, orc)


def test_random_displacements():
    rng = np.random.default_rng(1)
    mag = 2.0 ** rng.uniform(-30, 0, 30000)
    disp = (mag * rng.choice([-1.0, 1.0], mag.size)).astype(np.float32)
    for dt in (1e-4, 1e-3):
        got, orc, ref = run_one_step(disp, dt)
        assert same_bits(got, ref)
        assert same_bits(got, orc)
