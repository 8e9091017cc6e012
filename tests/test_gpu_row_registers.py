"""The register-row step kernel against the CPU oracle, bit for bit.

Resident bins of a 1,024-thread shape whose masses fit one per thread run a
variant of the step kernel that keeps each mass's row of incident springs in
registers (rows of at most 26 entries; wider rows are read from global
memory) and the springs in shared memory.  It performs the same operations
in the same order as the shared-memory-row kernel, so both match the oracle
exactly.
"""
import numpy as np
import pytest

import mercury_b200 as mb
from mercury_b200 import robots
from mercury_b200 import simulator as S
from oracle import core
from test_gpu_devo import OracleRun, check_same

pytestmark = pytest.mark.gpu

ENV_KEYS = ("g", "floor_stiffness", "friction_static", "friction_kinetic", "drag", "damping")
ENVS = {0: None, 1: S.LAND, 2: S.WATER}


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def run(b, mode, steps, track, dt, cfg):
    sim = mb.Simulator(0)
    if mode:
        sim.set_materials(mb.materials.force_table())
        sim.set_mode(mode)
        sim.set_environment(**ENVS[mode])
    sim.setTimeStep(dt)
    sim.set_launch_config(**cfg)
    sim.set_batch(b)
    variant = sim.step_variant()
    sim.run_steps(steps, track)
    return variant, sim.collect_arrays()


def oracle(b, mode, steps, track, dt):
    p, v = b.pos.copy(), b.vel.copy()
    s = np.zeros(b.n_springs, np.float32)
    if mode == 0:
        core.xpbd_run(b, p, v, s, mb.material_table(), dt, 0.0, steps, track)
    else:
        core.force_run(mode, b, p, v, s, mb.materials.force_table(), [ENVS[mode][k] for k in ENV_KEYS],
                       dt, 0.0, steps, track)
    return p, v, s


@pytest.mark.parametrize("mode", [0, 1, 2], ids=["reference", "land", "water"])
@pytest.mark.parametrize("track", [False, True])
@pytest.mark.parametrize("spt", [8, 10])
def test_register_rows_bit_exact(mode, track, spt):
    b = robots.population_batch("uneven", 24, seed_base=700, mass=0.1 if mode else 1.0)
    dt = 1e-3 if mode == 0 else 1e-4
    variant, (pos, vel, stress) = run(b, mode, 300, track, dt,
                                      dict(threads=1024, springs_per_thread=spt, masses_per_thread=2, bins=24,
                                           chunk=128))
    assert variant["register_rows"] == 1
    p, v, s = oracle(b, mode, 300, track, dt)
    assert np.array_equal(bits(pos), bits(p)) and np.array_equal(bits(vel), bits(v))
    if track:
        assert np.array_equal(bits(stress), bits(s))


def test_rows_grown_past_the_registers_by_development_bit_exact():
    """Development rewires springs to random pairs, so after it a mass can
    have more incident springs than the registers hold rows for: those rows
    are read from global memory, with the same bits."""
    b = robots.population_batch("small", 8, seed_base=40)
    dt = 1e-3
    sim = mb.Simulator(0)
    sim.setTimeStep(dt)
    sim.set_launch_config(threads=1024, springs_per_thread=8, masses_per_thread=2, bins=8, chunk=64)
    sim.set_batch(b)
    assert sim.step_variant()["register_rows"] == 1
    orc = OracleRun(b, mb.material_table(), dt)
    widest = 0
    for cycle in range(3):
        sim.run_steps(100, True)
        orc.steps(100)
        assert sim.devo(120, seed=cycle) == orc.devo(120, cycle)
        check_same(sim, orc)
        deg = np.zeros(b.n_masses, np.int64)
        act = orc.b.spring_material != 0
        so = np.repeat(b.mass_offsets[:-1], np.diff(b.spring_offsets))
        np.add.at(deg, (orc.b.pairs[:, 0] + so)[act], 1)
        np.add.at(deg, (orc.b.pairs[:, 1] + so)[act], 1)
        widest = max(widest, int(deg.max()))
    assert sim.devo_profile()["host_repacks"] == 0  # re-packed on the device, bins kept
    assert sim.step_variant()["register_rows"] == 1
    assert widest > 26  # some rows no longer fit the registers
    sim.run_steps(150, True)
    orc.steps(150)
    check_same(sim, orc)


def test_two_masses_per_thread_keeps_shared_memory_rows():
    """A bin of more than 1,024 masses needs two masses per thread: the
    shared-memory-row kernel runs, with the same bits."""
    b = robots.population_batch("small", 10, seed_base=700)
    variant, (pos, vel, _) = run(b, 0, 100, False, 1e-3,
                                 dict(threads=1024, springs_per_thread=12, masses_per_thread=2, bins=1, chunk=50))
    assert variant["register_rows"] == 0
    p, v, _ = oracle(b, 0, 100, False, 1e-3)
    assert np.array_equal(bits(pos), bits(p)) and np.array_equal(bits(vel), bits(v))
