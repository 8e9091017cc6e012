"""The force modes of the CUDA step against the FP32 oracle, bit for bit."""
import numpy as np
import pytest

import mercury_b200 as mb
from mercury_b200 import robots
from mercury_b200 import simulator as S
from oracle import core

pytestmark = pytest.mark.gpu

ENV_KEYS = ("g", "floor_stiffness", "friction_static", "friction_kinetic", "drag", "damping")


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def gpu(mode, b, e, steps, track, dt=1e-4, cfg=None):
    sim = mb.Simulator(0)
    sim.set_materials(mb.materials.force_table())
    sim.set_mode(mode)
    sim.set_environment(**e)
    sim.setTimeStep(dt)
    if cfg:
        sim.set_launch_config(**cfg)
    sim.set_batch(b)
    sim.run_steps(steps, track)
    return sim.collect_arrays()


def oracle(mode, b, e, steps, track, dt=1e-4):
    p, v = b.pos.copy(), b.vel.copy()
    s = np.zeros(b.n_springs, np.float32)
    core.force_run(mode, b, p, v, s, mb.materials.force_table(), [e[k] for k in ENV_KEYS], dt, 0.0,
                   steps, track)
    return p, v, s


@pytest.mark.parametrize("mode,env", [(1, S.LAND), (2, S.WATER)], ids=["land", "water"])
@pytest.mark.parametrize("track", [False, True])
def test_force_bit_exact(mode, env, track):
    b = robots.population_batch("uneven", 24, mass=0.1)
    pos, vel, stress = gpu(mode, b, env, 700, track)
    p, v, s = oracle(mode, b, env, 700, track)
    assert np.array_equal(bits(pos), bits(p)) and np.array_equal(bits(vel), bits(v))
    if track:
        assert np.array_equal(bits(stress), bits(s))


def test_land_contact_and_friction_paths_exercised():
    b = robots.population_batch("small", 8, mass=0.1)
    b.vel[:, 0] = np.where(np.arange(b.n_masses) % 2, 0.3, 0.0)
    pos, vel, _ = gpu(1, b, S.LAND, 1500, False, cfg=dict(chunk=128))
    p, v, _ = oracle(1, b, S.LAND, 1500, False)
    assert np.array_equal(bits(pos), bits(p)) and np.array_equal(bits(vel), bits(v))
    assert (p[:, 2] < 0).any()  # the ground acted


def test_mode_switch_keeps_reference_step_exact():
    b = robots.population_batch("small", 4)
    sim = mb.Simulator(0)
    sim.setTimeStep(1e-3)
    sim.set_batch(b)
    sim.set_mode(1)
    sim.set_mode(0)
    sim.run_steps(100)
    pos, vel, _ = sim.collect_arrays()
    p, v = b.pos.copy(), b.vel.copy()
    core.xpbd_run(b, p, v, np.zeros(b.n_springs, np.float32), mb.material_table(), 1e-3, 0.0, 100, False)
    assert np.array_equal(bits(pos), bits(p))


@pytest.mark.parametrize("cfg", [dict(streamed=1), dict()], ids=["streamed", "split"])
def test_nn_robots_in_water_bit_exact(cfg):
    """Point-cloud robots (25-NN springs, up to ~28k springs each) in water
    with stress tracking, streamed or split over clusters (the automatic
    choice): bit-exact against the oracle."""
    b = robots.population_batch("nn", 4, mass=0.1)
    sim = mb.Simulator(0)
    sim.set_materials(mb.materials.force_table())
    sim.set_mode(2)
    sim.set_environment(**S.WATER)
    sim.setTimeStep(1e-4)
    sim.set_launch_config(**cfg)
    sim.set_batch(b)
    lc = sim.launch_config()
    assert (lc["streamed"], lc["cluster"]) == ((1, 0) if cfg else (0, 4))
    sim.run_steps(200, True)
    pos, vel, stress = sim.collect_arrays()
    p, v, s = oracle(2, b, S.WATER, 200, True)
    assert np.array_equal(bits(pos), bits(p)) and np.array_equal(bits(vel), bits(v))
    assert np.array_equal(bits(stress), bits(s))


def test_land_divergence_from_fp64():
    """Contact chaos: the CUDA land step (FP32) against the oracle's FP64
    transcription of the same law, on 32 uneven robots.  The static/kinetic
    friction switch and the penalty ground amplify rounding differences
    (about e-fold every 200 steps, 20 ms); the early part of the curve is
    bounded, the rest is printed."""
    b = robots.population_batch("uneven", 32, mass=0.1)
    sim = mb.Simulator(0)
    sim.set_materials(mb.materials.force_table())
    sim.set_mode(1)
    sim.set_environment(**S.LAND)
    sim.setTimeStep(1e-4)
    sim.set_batch(b)
    pd, vd = b.pos.astype(np.float64), b.vel.astype(np.float64)
    done, curve = 0, {}
    for n in (10, 100, 300, 1000, 3000):
        sim.run_steps(n - done, False)
        core.force_run_f64(1, b, pd, vd, mb.materials.force_table(), [S.LAND[k] for k in ENV_KEYS], 1e-4,
                           done * 1e-4, n - done)
        done = n
        pos, _, _ = sim.collect_arrays()
        curve[n] = float(np.abs(pos[:, :3] - pd[:, :3]).max())
    print("\nland, max |x_fp32 - x_fp64| (m): " + ", ".join(f"{k} steps {v:.2e}" for k, v in curve.items()))
    assert curve[10] < 1e-5 and curve[100] < 5e-4 and curve[300] < 5e-3
    assert np.isfinite(pos).all()
