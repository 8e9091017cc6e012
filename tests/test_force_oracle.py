"""The force modes of the oracle (no reference code exists for them; the
contact law is this build's, restated identically in the kernel): FP32 vs
the FP64 transcription, and physical properties."""
import numpy as np
import pytest

import mercury_b200 as mb
from mercury_b200 import robots
from mercury_b200 import simulator as S
from oracle import core

ENV_KEYS = ("g", "floor_stiffness", "friction_static", "friction_kinetic", "drag", "damping")


def env(d):
    return [d[k] for k in ENV_KEYS]


def run32(mode, b, e, steps, dt=1e-4):
    p, v = b.pos.copy(), b.vel.copy()
    s = np.zeros(b.n_springs, np.float32)
    core.force_run(mode, b, p, v, s, mb.materials.force_table(), env(e), dt, 0.0, steps, True)
    return p, v, s


def test_water_fp32_tracks_fp64():
    b = robots.population_batch("small", 6, mass=0.1)
    p, _, _ = run32(2, b, S.WATER, 1000)
    pd, vd = b.pos.astype(np.float64), b.vel.astype(np.float64)
    core.force_run_f64(2, b, pd, vd, mb.materials.force_table(), env(S.WATER), 1e-4, 0.0, 1000)
    assert np.abs(p[:, :3] - pd[:, :3]).max() < 5e-4


def test_land_contact_holds_robots_up():
    b = robots.population_batch("small", 6, mass=0.1)
    p, v, _ = run32(1, b, S.LAND, 3000)
    assert np.isfinite(p).all()
    assert p[:, 2].min() > -0.005  # penalty ground: sub-centimetre penetration
    com = core.com_device(b, p)
    assert (com[:, 2] > 0.05).all()


def test_static_friction_keeps_a_passive_block_in_place():
    grid = np.full((3, 3, 3), mb.materials.BONE, np.uint8)
    b = mb.pack([robots.voxel_robot(grid[:2, :2, :2], mass=0.1)])
    b.vel[:, 0] = 0.0
    p, _, _ = run32(1, b, S.LAND, 2000)
    # gravity only: the block settles; static friction leaves x and y alone
    assert np.abs(p[:, :2] - b.pos[:, :2]).max() < 1e-4


def test_kinetic_friction_stops_a_sliding_block():
    grid = np.full((2, 2, 2), mb.materials.BONE, np.uint8)
    b = mb.pack([robots.voxel_robot(grid, mass=0.1)])
    b.vel[:, 0] = 0.5
    b.pos[:, 2] -= 0.0001  # in contact from the start
    p, v, _ = run32(1, b, S.LAND, 4000)
    # mu_k g = 7.8 m/s^2 stops 0.5 m/s in ~0.064 s (640 steps); what is left
    # is internal spring vibration, so check the centre of mass of the
    # non-air masses
    solid = b.mass_material != 0
    assert abs(float(v[solid, 0].astype(np.float64).mean())) < 5e-3
    slid = float(np.mean(p[solid, 0] - b.pos[solid, 0]))
    assert 0.005 < slid < 0.03  # ~v^2 / (2 mu_k g) = 1.6 cm without bouncing


def test_water_drag_slows_a_coasting_robot():
    b = robots.population_batch("small", 2, mass=0.1)
    b.vel[:, :3] = 0.2
    p, v, _ = run32(2, b, S.WATER, 2000)
    v0 = np.linalg.norm(b.vel[:, :3].mean(0))
    v1 = np.linalg.norm(v[:, :3].astype(np.float64).mean(0))
    assert v1 < v0 * 0.999 ** 2000 * 1.01


@pytest.mark.parametrize("mode", [1, 2])
def test_force_modes_are_robot_independent(mode):
    els = robots.population("uneven", 4, mass=0.1)
    b = mb.pack(els)
    e = S.LAND if mode == 1 else S.WATER
    p, v, s = run32(mode, b, e, 300)
    for r, el in enumerate(els):
        bi = mb.pack([el])
        pi, vi, si = run32(mode, bi, e, 300)
        ms, ss = b.robot_slices(r)
        assert np.array_equal(p[ms], pi) and np.array_equal(s[ss], si)


def test_land_fp32_tracks_fp64_early():
    """The land law's FP32/FP64 divergence curve starts at rounding level and
    grows about e-fold every 200 steps (contact chaos); its early part is
    bounded here, on the oracle whose bits the kernel reproduces."""
    b = robots.population_batch("uneven", 16, mass=0.1)
    p, v = b.pos.copy(), b.vel.copy()
    s = np.zeros(b.n_springs, np.float32)
    pd, vd = b.pos.astype(np.float64), b.vel.astype(np.float64)
    done, curve = 0, {}
    for n in (10, 100, 300):
        core.force_run(1, b, p, v, s, mb.materials.force_table(), env(S.LAND), 1e-4,
                       core.advance_clock(0.0, 1e-4, done), n - done, False)
        core.force_run_f64(1, b, pd, vd, mb.materials.force_table(), env(S.LAND), 1e-4, done * 1e-4, n - done)
        done = n
        curve[n] = float(np.abs(p[:, :3] - pd[:, :3]).max())
    assert curve[10] < 1e-5 and curve[100] < 5e-4 and curve[300] < 5e-3, curve
