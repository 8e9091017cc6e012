"""Face drag of the water mode on the device against the FP32 oracle, bit
for bit: voxel robots with their exposed cell faces, point clouds with
their convex hulls, across launch chunks and development cycles."""
import dataclasses

import numpy as np
import pytest

import mercury_b200 as mb
from mercury_b200 import robots
from mercury_b200 import simulator as S
from oracle import core

pytestmark = pytest.mark.gpu

ENV7 = ("g", "floor_stiffness", "friction_static", "friction_kinetic", "drag", "damping", "face_drag")


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def moving(b, seed):
    """A random velocity per robot, so that every face drags."""
    rng = np.random.default_rng(seed)
    for r in range(b.n_robots):
        ms, _ = b.robot_slices(r)
        b.vel[ms, :3] = rng.normal(0.0, 0.5, 3).astype(np.float32)
    return b


def gpu(b, env, steps, track, cfg=None, dt=1e-4):
    sim = mb.Simulator(0)
    sim.set_materials(mb.materials.force_table())
    sim.set_mode(S.MODE_FORCE_WATER)
    sim.set_environment(**env)
    sim.setTimeStep(dt)
    if cfg:
        sim.set_launch_config(**cfg)
    sim.set_batch(b)
    sim.run_steps(steps, track)
    return sim


def oracle(b, env, steps, track, dt=1e-4, state=None, t0=0.0):
    p, v = (b.pos.copy(), b.vel.copy()) if state is None else (state[0].copy(), state[1].copy())
    s = np.zeros(b.n_springs, np.float32) if state is None else state[2].copy()
    core.force_run(2, b, p, v, s, mb.materials.force_table(), [env[k] for k in ENV7], dt, t0, steps, track)
    return p, v, s


def same(sim, ref, track=True):
    pos, vel, st = sim.collect_arrays()
    assert np.array_equal(bits(pos), bits(ref[0]))
    assert np.array_equal(bits(vel), bits(ref[1]))
    if track:
        assert np.array_equal(bits(st), bits(ref[2]))


@pytest.mark.parametrize("track", [False, True])
@pytest.mark.parametrize("cfg", [None, {"chunk": 97, "use_graph": 0}], ids=["graph", "chunks"])
def test_voxel_faces_bit_exact(track, cfg):
    b = moving(robots.population_batch("uneven", 24, mass=0.1, faces=True), 1)
    sim = gpu(b, S.WATER_FACES, 400, track, cfg)
    assert sim.launch_config()["cluster"] == 0 and sim.launch_config()["streamed"] == 0
    same(sim, oracle(b, S.WATER_FACES, 400, track), track)


def test_faces_and_per_mass_drag_together():
    b = moving(robots.population_batch("small", 16, mass=0.1, faces=True), 2)
    env = dict(S.WATER, face_drag=500.0)
    same(gpu(b, env, 300, True), oracle(b, env, 300, True))


def test_point_cloud_hulls_bit_exact():
    els = []
    for r in range(6):
        rng = np.random.default_rng(4000 + r)
        e = robots.nn_robot(rng, int(rng.integers(200, 401)))
        e.faces = robots.hull_faces(e.pos)
        els.append(e)
    b = moving(mb.pack(els), 3)
    sim = gpu(b, S.WATER_FACES, 300, True)
    assert sim.launch_config()["cluster"] == 0
    same(sim, oracle(b, S.WATER_FACES, 300, True))


def test_robots_with_and_without_faces_share_bins():
    els = robots.population("small", 12, mass=0.1, faces=True)
    for e in els[::2]:
        e.faces = None
    b = moving(mb.pack(els), 4)
    same(gpu(b, S.WATER_FACES, 300, True), oracle(b, S.WATER_FACES, 300, True))


def test_face_drag_off_runs_the_plain_water_step():
    b = moving(robots.population_batch("small", 8, mass=0.1, faces=True), 5)
    env = dict(S.WATER, face_drag=0.0)
    plain = dataclasses.replace(b, face_offsets=None, faces=None)
    same(gpu(b, env, 300, True), oracle(plain, env, 300, True))


def test_faces_after_development():
    b = moving(robots.population_batch("uneven", 16, mass=0.1, faces=True), 6)
    env = S.WATER_FACES
    sim = gpu(b, env, 150, True)
    ref = oracle(b, env, 150, True)
    same(sim, ref)
    assert sim.devo(16, seed=3) > 0
    pairs, mat, lbar = sim.collect_springs()
    b2 = dataclasses.replace(b, pairs=pairs, spring_material=mat, lbar=lbar)
    t = sim.getTotalTime()
    state = sim.collect_arrays()
    sim.run_steps(150, True)
    same(sim, oracle(b2, env, 150, True, state=state, t0=t))


@pytest.mark.parametrize("track", [False, True])
def test_streamed_bins_bit_exact(track):
    b = moving(robots.population_batch("uneven", 12, mass=0.1, faces=True), 7)
    sim = gpu(b, S.WATER_FACES, 300, track, {"streamed": 1, "chunk": 128})
    assert sim.launch_config()["streamed"] == 1
    same(sim, oracle(b, S.WATER_FACES, 300, track), track)


@pytest.mark.parametrize("track", [False, True])
@pytest.mark.parametrize("cfg", [None, {"chunk": 97, "use_graph": 0}], ids=["graph", "chunks"])
def test_split_point_clouds_bit_exact(track, cfg):
    """Point clouds too large for one CTA, with their convex hulls: split
    over clusters, velocities exchanged with the positions, faces across a
    cut computed in every part that holds one of their corners."""
    b = moving(mb.pack(robots.population("nn", 6, mass=0.1, faces=True)), 9)
    sim = gpu(b, S.WATER_FACES, 200, track, cfg)
    assert sim.launch_config()["cluster"] > 0
    same(sim, oracle(b, S.WATER_FACES, 200, track), track)


@pytest.mark.parametrize("cluster", [2, 4, 8])
def test_forced_split_with_faces_bit_exact(cluster):
    b = moving(robots.population_batch("uneven", 8, mass=0.1, faces=True), 10)
    sim = gpu(b, S.WATER_FACES, 200, True, {"cluster": cluster})
    assert sim.launch_config()["cluster"] == cluster
    same(sim, oracle(b, S.WATER_FACES, 200, True))


def test_face_drag_switched_on_for_a_split_population():
    b = moving(mb.pack(robots.population("nn", 2, mass=0.1, faces=True)), 8)
    sim = mb.Simulator(0)
    sim.set_materials(mb.materials.force_table())
    sim.set_mode(S.MODE_FORCE_WATER)
    sim.set_environment(**dict(S.WATER_FACES, face_drag=0.0))
    sim.setTimeStep(1e-4)
    sim.set_batch(b)
    assert sim.launch_config()["cluster"] > 0
    sim.run_steps(100, True)
    ref = oracle(b, dict(S.WATER_FACES, face_drag=0.0), 100, True)
    same(sim, ref)
    t = sim.getTotalTime()
    sim.set_environment(face_drag=S.WATER_FACES["face_drag"])
    sim.run_steps(200, True)  # re-packed with the faces in the parts, state kept
    assert sim.launch_config()["cluster"] > 0
    same(sim, oracle(b, S.WATER_FACES, 200, True, state=ref, t0=t))
