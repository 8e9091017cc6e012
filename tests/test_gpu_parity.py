"""The CUDA step against the CPU oracle, bit for bit, through the C ABI.

The kernel and the oracle fix the same summation order and use the same
correctly rounded operations, so every comparison here is exact (positions,
velocities, stresses and centres of mass as raw bits).  Full-size runs are
checked through properties that do not depend on size: determinism,
independence of the launch configuration, and momentum decay.
"""
import numpy as np
import pytest

import mercury_b200 as mb
from mercury_b200 import robots
from oracle import core

pytestmark = pytest.mark.gpu

TABLE = None


def table():
    global TABLE
    if TABLE is None:
        TABLE = mb.material_table()
    return TABLE


def bits_equal(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.uint32), np.ascontiguousarray(b).view(np.uint32))


def run_gpu(batch, dt, steps, track, sim=None, cfg=None, t0=0.0):
    sim = sim or mb.Simulator(0)
    sim.setTimeStep(dt)
    if cfg:
        sim.set_launch_config(**cfg)
    sim.set_batch(batch)
    if t0:
        mb._lib.check(mb.LIB.mb_set_total_time(sim._ctx, t0), sim._ctx)
    sim.run_steps(steps, track)
    pos, vel, stress = sim.collect_arrays()
    return sim, pos, vel, stress


def run_oracle(batch, dt, steps, track, t0=0.0):
    p, v = batch.pos.copy(), batch.vel.copy()
    s = np.zeros(batch.n_springs, np.float32)
    core.xpbd_run(batch, p, v, s, table(), dt, t0, steps, track)
    return p, v, s


def test_smoke():
    import __graft_entry__
    __graft_entry__.smoke()


@pytest.mark.parametrize("dt", [1e-4, 1e-3, 5e-3])
@pytest.mark.parametrize("track", [False, True])
def test_small_population_bit_exact(dt, track):
    b = robots.population_batch("small")
    _, pos, vel, stress = run_gpu(b, dt, 300, track)
    p, v, s = run_oracle(b, dt, 300, track)
    assert bits_equal(pos, p)
    assert bits_equal(vel, v)
    if track:
        assert bits_equal(stress, s)
    else:
        assert not stress.any()


def test_uneven_population_bit_exact():
    b = robots.population_batch("uneven", 40)
    _, pos, vel, stress = run_gpu(b, 1e-3, 250, True)
    p, v, s = run_oracle(b, 1e-3, 250, True)
    assert bits_equal(pos, p) and bits_equal(vel, v) and bits_equal(stress, s)


def test_nonzero_start_clock_and_velocity():
    b = robots.population_batch("uneven", 12, seed_base=77)
    rng = np.random.default_rng(0)
    b.vel[:, :3] = rng.normal(0, 0.05, (b.n_masses, 3)).astype(np.float32)
    _, pos, vel, stress = run_gpu(b, 2e-3, 150, True, t0=3.25)
    p, v, s = run_oracle(b, 2e-3, 150, True, t0=3.25)
    assert bits_equal(pos, p) and bits_equal(vel, v) and bits_equal(stress, s)


SHAPES = [
    dict(threads=256, springs_per_thread=8, masses_per_thread=2),
    dict(threads=512, springs_per_thread=16, masses_per_thread=4),
    dict(threads=512, springs_per_thread=8, masses_per_thread=2),
    dict(threads=1024, springs_per_thread=8, masses_per_thread=2),
    dict(threads=1024, springs_per_thread=4, masses_per_thread=1),
    dict(threads=1024, springs_per_thread=12, masses_per_thread=2),
]


@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: f"{s['threads']}x{s['springs_per_thread']}")
def test_launch_shape_does_not_change_bits(shape):
    """Every compiled shape.  Robots larger than the shape's capacity are
    split over clusters (1,024-thread shapes) or streamed: same bits."""
    b = robots.population_batch("uneven", 24, seed_base=500)
    # automatic bin count: several robots per CTA, within the shape's capacity
    _, pos, vel, stress = run_gpu(b, 1e-3, 120, True, cfg=dict(shape, chunk=37))
    p, v, s = run_oracle(b, 1e-3, 120, True)
    assert bits_equal(pos, p) and bits_equal(vel, v) and bits_equal(stress, s)


@pytest.mark.parametrize("chunk,graph", [(1, 0), (7, 1), (100, 1), (1000, 0)])
def test_chunking_and_graphs(chunk, graph):
    b = robots.population_batch("small", 10)
    _, pos, vel, _ = run_gpu(b, 1e-3, 230, False, cfg=dict(chunk=chunk, use_graph=graph))
    p, v, _ = run_oracle(b, 1e-3, 230, False)
    assert bits_equal(pos, p) and bits_equal(vel, v)


def test_graph_replay_is_repeatable():
    b = robots.population_batch("small", 16)
    sim = mb.Simulator(0)
    sim.setTimeStep(1e-3)
    outs = []
    for _ in range(3):
        sim.set_batch(b)
        sim.Reset()
        sim.Simulate(0.1)
        outs.append(sim.collect_arrays()[0].copy())
    assert bits_equal(outs[0], outs[1]) and bits_equal(outs[1], outs[2])


def test_simulate_follows_reference_clock():
    b = robots.population_batch("small", 4)
    sim = mb.Simulator(0)
    sim.setTimeStep(1e-4)
    sim.set_batch(b)
    n = sim.Simulate(0.05)
    assert n == core.step_count(0.05, 1e-4)
    assert sim.getTotalTime() == core.advance_clock(0.0, 1e-4, n)
    p, v, _ = run_oracle(b, 1e-4, n, False)
    pos, vel, _ = sim.collect_arrays()
    assert bits_equal(pos, p) and bits_equal(vel, v)


def test_centre_of_mass_bit_exact():
    b = robots.population_batch("uneven", 30)
    sim, pos, _, _ = run_gpu(b, 5e-3, 100, False)
    com = sim.CentreOfMass()
    assert bits_equal(com, core.com_device(b, pos))
    assert np.allclose(com, core.com_reference(b, pos), atol=2e-6)


def test_reference_api_round_trip():
    els = robots.population("uneven", 6)
    sim = mb.Simulator(0)
    sim.Initialize(mb.SimulatorConfig(time_step=1e-3))
    trackers = sim.SetElements(els)
    sim.Simulate(0.05, trackStresses=True)
    out = sim.Collect(trackers)
    assert len(out) == 6 and all(o.pos.shape == e.pos.shape for o, e in zip(out, els))
    b = mb.pack(els)
    p, v, s = run_oracle(b, 1e-3, core.step_count(0.05, 1e-3), True)
    for r, o in enumerate(out):
        ms, ss = b.robot_slices(r)
        assert bits_equal(o.pos, p[ms, :3]) and bits_equal(o.stress, s[ss])


def test_full_population_bit_exact_and_deterministic():
    """The full 512-robot uneven population: bit-exact against the oracle
    for 300 steps, two GPU runs bit-identical, and with a uniform initial
    velocity the mean velocity of each robot decays by 0.99 per step
    (momentum conservation of the +dp/-dp corrections)."""
    b = robots.population_batch("uneven")
    b.vel[:, :3] = 0.02
    _, p1, v1, s1 = run_gpu(b, 1e-3, 300, True)
    _, p2, v2, s2 = run_gpu(b, 1e-3, 300, True)
    assert bits_equal(p1, p2) and bits_equal(v1, v2) and bits_equal(s1, s2)
    p, v, s = run_oracle(b, 1e-3, 300, True)
    assert bits_equal(p1, p) and bits_equal(v1, v) and bits_equal(s1, s)
    for r in range(0, b.n_robots, 37):
        ms, _ = b.robot_slices(r)
        # position rounding quantises velocities to ulp(x)/dt and biases the
        # mean by up to ~6% after 300 steps; the property is checked loosely
        assert np.allclose(v1[ms, :3].astype(np.float64).mean(0), 0.02 * 0.99 ** 300, rtol=0.1)


def test_nonfinite_input_is_flagged():
    b = robots.population_batch("small", 3)
    b.pos[5, 0] = np.nan
    sim, pos, _, _ = run_gpu(b, 1e-3, 10, False)
    flags = sim.robot_flags()
    assert flags[0] & 1 and not (flags[1] & 1) and not (flags[2] & 1)


def test_invalid_topology_rejected():
    b = robots.population_batch("small", 2)
    b.pairs[3, 1] = 500  # robot has 125 masses
    with pytest.raises(mb.MercuryError) as e:
        mb.Simulator(0).set_batch(b)
    assert e.value.status == 1


def test_robot_too_large_rejected():
    grid = np.full((20, 20, 20), 22, np.uint8)
    e = robots.lattice_robot(grid)
    with pytest.raises(mb.MercuryError) as err:
        mb.Simulator(0).set_batch(mb.pack([e]))
    assert err.value.status == 3


# ---------------------------------------------------------------------------
# Streamed variant: springs, rows and per-spring scratch in global memory.

@pytest.mark.parametrize("track", [False, True])
def test_streamed_forced_bit_exact(track):
    b = robots.population_batch("uneven", 20, seed_base=321)
    _, pos, vel, stress = run_gpu(b, 1e-3, 200, track, cfg=dict(streamed=1, chunk=64))
    p, v, s = run_oracle(b, 1e-3, 200, track)
    assert bits_equal(pos, p) and bits_equal(vel, v)
    if track:
        assert bits_equal(stress, s)


@pytest.mark.parametrize("cfg", [dict(cluster=1), dict()], ids=["streamed", "split"])
def test_large_robots_bit_exact(cfg):
    """10x10x10-cell robots (1,331 masses, 14,230 springs) do not fit a
    resident bin: never split, the library streams them; by default it splits
    each over a two-CTA cluster.  Same results either way."""
    b = robots.population_batch("streamed", 6)
    sim, pos, vel, stress = run_gpu(b, 1e-4, 150, True, cfg=cfg)
    lc = sim.launch_config()
    assert (lc["streamed"], lc["cluster"]) == ((1, 0) if cfg else (0, 2))
    p, v, s = run_oracle(b, 1e-4, 150, True)
    assert bits_equal(pos, p) and bits_equal(vel, v) and bits_equal(stress, s)


@pytest.mark.parametrize("mode", [1, 2])
def test_streamed_force_modes_bit_exact(mode):
    from mercury_b200 import simulator as S
    env = S.LAND if mode == 1 else S.WATER
    b = robots.population_batch("streamed", 3, mass=0.1)
    sim = mb.Simulator(0)
    sim.set_materials(mb.materials.force_table())
    sim.set_mode(mode)
    sim.set_environment(**env)
    sim.setTimeStep(1e-4)
    sim.set_batch(b)
    sim.run_steps(300, True)
    pos, vel, stress = sim.collect_arrays()
    p, v = b.pos.copy(), b.vel.copy()
    s = np.zeros(b.n_springs, np.float32)
    keys = ("g", "floor_stiffness", "friction_static", "friction_kinetic", "drag", "damping")
    core.force_run(mode, b, p, v, s, mb.materials.force_table(), [env[k] for k in keys], 1e-4, 0.0, 300, True)
    assert bits_equal(pos, p) and bits_equal(vel, v) and bits_equal(stress, s)


@pytest.mark.parametrize("track", [False, True])
def test_rows_built_on_device_or_host_same_bits(monkeypatch, track):
    """Uploads build the incidence rows on the device (the development
    re-pack kernel); MB_HOST_ROWS=1 has the host packer build them."""
    b = robots.population_batch("uneven", 40, seed_base=77)
    _, p1, v1, s1 = run_gpu(b, 1e-3, 150, track)
    monkeypatch.setenv("MB_HOST_ROWS", "1")
    _, p2, v2, s2 = run_gpu(b, 1e-3, 150, track)
    p, v, s = run_oracle(b, 1e-3, 150, track)
    assert bits_equal(p1, p) and bits_equal(v1, v) and bits_equal(p2, p) and bits_equal(v2, v)
    if track:
        assert bits_equal(s1, s) and bits_equal(s2, s)


@pytest.mark.parametrize("name,n", [("uneven", 40), ("uneven", 512), ("small", 300)])
def test_springs_placed_on_device_as_on_host(monkeypatch, name, n):
    """With the rows built on the device the springs are placed there too
    (launch_bank_place); the slots must hold the same springs as the host
    packer's placement (MB_HOST_ROWS=1), word for word."""
    b = robots.population_batch(name, n, seed_base=5)
    sim = mb.Simulator(0)
    sim.set_batch(b)
    dev = sim.packed_springs()
    monkeypatch.setenv("MB_HOST_ROWS", "1")
    sim2 = mb.Simulator(0)
    sim2.set_batch(b)
    host = sim2.packed_springs()
    assert sim.launch_config() == sim2.launch_config()
    assert len(dev) == len(host) >= b.active_springs()
    assert np.array_equal(dev, host)
