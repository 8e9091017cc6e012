"""Robots split over a thread-block cluster (one CTA per part, boundary
positions exchanged through distributed shared memory) against the CPU
oracle, bit for bit: the reference step and the force modes, stresses
tracked, clusters of 2, 4 and 8 CTAs, the automatic choice for robots too
large for one CTA, development on a split population, and the launch
configuration API."""
import dataclasses

import numpy as np
import pytest

import mercury_b200 as mb
from mercury_b200 import robots
from mercury_b200 import simulator as S
from oracle import core

pytestmark = pytest.mark.gpu

ENV_KEYS = ("g", "floor_stiffness", "friction_static", "friction_kinetic", "drag", "damping")


def bits_equal(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.uint32), np.ascontiguousarray(b).view(np.uint32))


def simulate(batch, dt, steps, track, cfg=None, mode=0):
    sim = mb.Simulator(0)
    if mode:
        sim.set_materials(mb.materials.force_table())
        sim.set_mode(mode)
        sim.set_environment(**(S.LAND if mode == S.MODE_FORCE_LAND else S.WATER))
    sim.setTimeStep(dt)
    if cfg:
        sim.set_launch_config(**cfg)
    sim.set_batch(batch)
    sim.run_steps(steps, track)
    pos, vel, stress = sim.collect_arrays()
    return sim, pos, vel, stress


def oracle(batch, dt, steps, track, mode=0):
    p, v = batch.pos.copy(), batch.vel.copy()
    s = np.zeros(batch.n_springs, np.float32)
    if mode == 0:
        core.xpbd_run(batch, p, v, s, mb.material_table(), np.float32(dt), 0.0, steps, track)
    else:
        env = S.LAND if mode == S.MODE_FORCE_LAND else S.WATER
        core.force_run(mode, batch, p, v, s, mb.materials.force_table(), [env[k] for k in ENV_KEYS],
                       np.float32(dt), 0.0, steps, track)
    return p, v, s


def check(batch, dt, steps, track, cfg=None, mode=0, cluster=None):
    sim, pos, vel, st = simulate(batch, dt, steps, track, cfg, mode)
    if cluster is not None:
        assert sim.launch_config()["cluster"] == cluster
    p, v, s = oracle(batch, dt, steps, track, mode)
    assert bits_equal(pos, p)
    assert bits_equal(vel, v)
    if track:
        assert bits_equal(st, s)
    return sim


@pytest.mark.parametrize("cluster", [2, 4, 8])
@pytest.mark.parametrize("track", [False, True])
def test_forced_split_reference_step(cluster, track):
    b = robots.population_batch("uneven", 10)
    check(b, 1e-3, 300, track, {"cluster": cluster}, cluster=cluster)


@pytest.mark.parametrize("mode", [S.MODE_FORCE_LAND, S.MODE_FORCE_WATER], ids=["land", "water"])
def test_forced_split_force_modes(mode):
    b = robots.population_batch("uneven", 8, mass=0.1)
    check(b, 1e-4, 400, True, {"cluster": 2}, mode=mode, cluster=2)


def test_large_robots_split_automatically():
    """10x10x10-cell robots do not fit one CTA: two-CTA clusters."""
    b = robots.population_batch("streamed", 3)
    check(b, 1e-4, 200, True, cluster=2)


def test_point_cloud_robots_in_water():
    """Point-cloud robots of up to 2,000 masses: four-CTA clusters."""
    b = mb.pack(robots.nn_population_device(3, mass=0.1))
    check(b, 1e-4, 150, True, mode=S.MODE_FORCE_WATER, cluster=4)


@pytest.mark.parametrize("chains", [1, 2])
def test_parts_of_one_and_two_masses_per_thread(chains):
    """A large robot beside 1,500-mass chains: one own mass per thread with
    one chain, two with two chains (fewer CTAs); bit for bit either way."""
    n = 1500
    pos = np.zeros((n, 3), np.float32)
    pos[:, 0] = 0.1 * np.arange(n)
    pos[:, 2] = 0.02 * np.sin(np.arange(n))
    pairs = np.stack([np.arange(n - 1), np.arange(1, n)], 1)
    chain = mb.Element(pos, np.full(n, 1, np.uint8), pairs, np.full(n - 1, 0.1, np.float32),
                       np.full(n - 1, 1, np.uint8))
    b = mb.pack(robots.population("streamed", 1, seed_base=4200) + [chain] * chains)
    sim = check(b, 1e-3, 150, True, cluster=2)
    assert sim.launch_config()["masses_per_thread"] == chains


def test_split_and_streamed_agree_on_large_robots():
    b = robots.population_batch("streamed", 2, seed_base=4100)
    _, p1, v1, s1 = simulate(b, 1e-4, 300, True)
    _, p2, v2, s2 = simulate(b, 1e-4, 300, True, {"streamed": 1})
    _, p3, v3, s3 = simulate(b, 1e-4, 300, True, {"cluster": 4})
    for x, y in ((p1, p2), (v1, v2), (s1, s2), (p1, p3), (v1, v3), (s1, s3)):
        assert bits_equal(x, y)


def test_split_devo_cycles():
    """Development on a split population: host re-pack, then more steps."""
    b = robots.population_batch("uneven", 6)
    sim = mb.Simulator(0)
    sim.setTimeStep(1e-3)
    sim.set_launch_config(cluster=2)
    sim.set_batch(b)
    p, v = b.pos.copy(), b.vel.copy()
    s = np.zeros(b.n_springs, np.float32)
    t = 0.0
    ob = b
    for cycle in range(2):
        sim.run_steps(100, True)
        core.xpbd_run(ob, p, v, s, mb.material_table(), np.float32(1e-3), t, 100, True)
        t = core.advance_clock(t, np.float32(1e-3), 100)
        n = sim.devo(16, seed=cycle)
        pairs, mat, lbar, recs = core.devo(ob, p, s, mb.material_table(), t, 16, cycle)
        assert n == len(recs)
        ob = dataclasses.replace(ob, pairs=pairs, spring_material=mat, lbar=lbar)
        assert sim.launch_config()["cluster"] == 2
    sim.run_steps(100, True)
    core.xpbd_run(ob, p, v, s, mb.material_table(), np.float32(1e-3), t, 100, True)
    pos, vel, st = sim.collect_arrays()
    assert bits_equal(pos, p) and bits_equal(vel, v) and bits_equal(st, s)


def test_centre_of_mass_and_flags_on_split_robots():
    b = robots.population_batch("streamed", 2)
    sim, pos, _, _ = simulate(b, 1e-4, 50, False)
    assert bits_equal(sim.CentreOfMass(), core.com_device(b, pos))
    assert not sim.robot_flags().any()


def test_cluster_config_validation():
    sim = mb.Simulator(0)
    with pytest.raises(Exception):
        sim.set_launch_config(cluster=3)
    with pytest.raises(Exception):
        sim.set_launch_config(threads=512, springs_per_thread=8, masses_per_thread=2, cluster=2)
    # never split: large robots take the streamed path
    sim.setTimeStep(1e-4)
    sim.set_launch_config(cluster=1)
    sim.set_batch(robots.population_batch("streamed", 1))
    cfg = sim.launch_config()
    assert cfg["cluster"] == 0 and cfg["streamed"] == 1


def _degenerate_elements():
    """Robots of one and two masses with no active spring (their parts of a
    cluster stay empty) beside ordinary robots."""
    one = mb.Element(np.zeros((1, 3), np.float32), np.array([1]), np.array([[0, 0]]), np.ones(1),
                     np.zeros(1, np.uint8), vel=np.array([[0.1, 0.0, 0.0]], np.float32))
    two = mb.Element(np.array([[0, 0, 0], [0.1, 0, 0]], np.float32), np.array([1, 2]), np.array([[0, 1]]),
                     np.array([0.1], np.float32), np.zeros(1, np.uint8))
    els = robots.population("uneven", 5)
    return [one, els[0], two, els[1], els[2], one, els[3], els[4]]


@pytest.mark.parametrize("cfg", [{"cluster": 8}, {"cluster": 2}], ids=["cluster8", "cluster2"])
def test_degenerate_robots_split(cfg):
    check(mb.pack(_degenerate_elements()), 1e-3, 200, True, cfg, cluster=cfg["cluster"])


def test_degenerate_robots_beside_large_ones():
    """Automatic plan: the large robots take two parts, the others one each,
    sharing clusters (with empty slots)."""
    b = mb.pack(robots.population("streamed", 2) + _degenerate_elements())
    check(b, 1e-4, 150, True, cluster=2)


def test_largest_robot_splits_over_eight():
    """4,096 masses (15x15x15 cells, 46,620 springs): eight parts."""
    rng = np.random.default_rng(3)
    e = robots.voxel_robot(robots.FOUR[rng.integers(0, 4, size=(15, 15, 15))], mass=1.0)
    check(mb.pack([e]), 1e-4, 60, True, cluster=8)


@pytest.mark.parametrize("graph", [1, 0], ids=["graph", "no_graph"])
def test_two_cluster_groups_side_by_side(graph):
    """Point clouds of one, two and four parts: four-part robots launch in
    clusters of four, the others beside them in clusters of two (a second
    stream, forked and joined around every launch of 37 steps)."""
    b = mb.pack(robots.nn_population_device(6, seed_base=2100, mass=0.1))
    pl = mb.plan(b)
    assert pl["cluster"] == 4 and pl["cluster2"] == 2 and 0 < pl["split_bins0"] < pl["bins"]
    check(b, 1e-4, 150, True, {"chunk": 37, "use_graph": graph}, mode=S.MODE_FORCE_WATER, cluster=4)


def _devo_cycles(b, cfg, k, cycles, dt=1e-3, steps=100, expect_device=True):
    sim = mb.Simulator(0)
    sim.setTimeStep(dt)
    if cfg:
        sim.set_launch_config(**cfg)
    sim.set_batch(b)
    cl = sim.launch_config()["cluster"]
    assert cl >= 2
    p, v = b.pos.copy(), b.vel.copy()
    s = np.zeros(b.n_springs, np.float32)
    t, ob = 0.0, b
    for cycle in range(cycles):
        sim.run_steps(steps, True)
        core.xpbd_run(ob, p, v, s, mb.material_table(), np.float32(dt), t, steps, True)
        t = core.advance_clock(t, np.float32(dt), steps)
        n = sim.devo(k, seed=100 + cycle)
        pairs, mat, lbar, recs = core.devo(ob, p, s, mb.material_table(), t, k, 100 + cycle)
        assert n == len(recs)
        ob = dataclasses.replace(ob, pairs=pairs, spring_material=mat, lbar=lbar)
        assert sim.launch_config()["cluster"] == cl  # still split, same clusters
        if expect_device:
            assert sim.devo_profile()["host_repacks"] == 0, sim.devo_profile()
    sim.run_steps(steps, True)
    core.xpbd_run(ob, p, v, s, mb.material_table(), np.float32(dt), t, steps, True)
    pos, vel, st = sim.collect_arrays()
    assert bits_equal(pos, p) and bits_equal(vel, v) and bits_equal(st, s)
    # the topology the device holds is the oracle's
    pr, sm, lb = sim.collect_springs()
    assert np.array_equal(pr, ob.pairs) and np.array_equal(sm, ob.spring_material) and bits_equal(lb, ob.lbar)
    return sim


@pytest.mark.parametrize("cluster", [2, 4])
def test_split_devo_on_the_device_large_robots(cluster):
    """Development of robots split over clusters re-derives every part on the
    device (the partition stays): springs that leave or join a part, new
    halo masses and their exports, rows; bit for bit the oracle through
    several development cycles, stresses tracked."""
    b = robots.population_batch("streamed", 4)
    _devo_cycles(b, {"cluster": cluster}, 96, 3)


def test_split_devo_on_the_device_shared_clusters():
    """Uneven robots in two-CTA clusters, small ones sharing a cluster, and
    point clouds split automatically (one, two or four parts)."""
    _devo_cycles(robots.population_batch("uneven", 10, seed_base=3100), {"cluster": 2}, 24, 3)
    nb = mb.pack(robots.nn_population_device(6, seed_base=2300))
    _devo_cycles(nb, None, 64, 2)


def test_split_devo_device_equals_host_repack(monkeypatch):
    b = robots.population_batch("streamed", 3, seed_base=4400)
    dev = _devo_cycles(b, {"cluster": 2}, 48, 2)
    monkeypatch.setenv("MB_DEVO_HOST_REPACK", "1")
    host = _devo_cycles(b, {"cluster": 2}, 48, 2, expect_device=False)
    for a, c in zip(dev.collect_arrays(), host.collect_arrays()):
        assert bits_equal(a, c)
