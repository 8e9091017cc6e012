"""Development (mb_devo) on the device against the oracle, bit for bit:
the rewired topology after each call, and the steps that follow it on the
re-packed population (Simulate(devo_time, true); Devo() cycles as the
reference's evaluator runs them, optimize/optimizer/Evaluator)."""
import dataclasses

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


class OracleRun:
    """The same cycles on the CPU oracle."""

    def __init__(self, batch, table, dt, mode=0, env=None):
        self.b, self.table, self.dt, self.mode, self.env = batch, table, dt, mode, env
        self.p, self.v = batch.pos.copy(), batch.vel.copy()
        self.s = np.zeros(batch.n_springs, np.float32)
        self.t = 0.0

    def steps(self, n, track=True):
        if self.mode == 0:
            core.xpbd_run(self.b, self.p, self.v, self.s, self.table, self.dt, self.t, n, track)
        else:
            core.force_run(self.mode, self.b, self.p, self.v, self.s, self.table,
                           [self.env[k] for k in ENV_KEYS], self.dt, self.t, n, track)
        self.t = core.advance_clock(self.t, self.dt, n)

    def devo(self, k, seed, flags=0):
        pairs, mat, lbar, recs = core.devo(self.b, self.p, self.s, self.table, self.t, k, seed, flags)
        self.b = dataclasses.replace(self.b, pairs=pairs, spring_material=mat, lbar=lbar)
        return len(recs)


def check_same(sim, orc):
    pos, vel, stress = sim.collect_arrays()
    assert np.array_equal(bits(pos), bits(orc.p))
    assert np.array_equal(bits(vel), bits(orc.v))
    assert np.array_equal(bits(stress), bits(orc.s))
    pairs, mat, lbar = sim.collect_springs()
    assert np.array_equal(pairs, orc.b.pairs)
    assert np.array_equal(mat, orc.b.spring_material)
    assert np.array_equal(bits(lbar), bits(orc.b.lbar))


@pytest.mark.parametrize("flags", [0, mb._lib.DEVO_REFERENCE_RANKS], ids=["top", "reference_ranks"])
def test_devo_cycles_bit_exact(flags):
    b = robots.population_batch("uneven", 24)
    dt = 1e-3
    sim = mb.Simulator(0)
    sim.setTimeStep(dt)
    sim.set_batch(b)
    orc = OracleRun(b, mb.material_table(), dt)
    for cycle in range(3):
        sim.run_steps(120, True)
        orc.steps(120)
        assert np.float32(sim.getTotalTime()) == np.float32(orc.t)
        n = sim.devo(16, seed=cycle, reference_ranks=bool(flags))
        assert n == orc.devo(16, cycle, flags) and n > 0
        check_same(sim, orc)
    sim.run_steps(150, True)
    orc.steps(150)
    check_same(sim, orc)
    if not flags:  # moderate k: the device re-pack suffices every time
        assert sim.devo_profile()["host_repacks"] == 0


def test_devo_host_repack_path_bit_exact(monkeypatch):
    """The host re-pack (the device path's fallback) gives the same bits."""
    monkeypatch.setenv("MB_DEVO_HOST_REPACK", "1")
    b = robots.population_batch("uneven", 16, seed_base=321)
    sim = mb.Simulator(0)
    sim.setTimeStep(1e-3)
    sim.set_batch(b)
    orc = OracleRun(b, mb.material_table(), np.float32(1e-3))
    for cycle in range(2):
        sim.run_steps(80, True)
        orc.steps(80)
        assert sim.devo(24, seed=cycle) == orc.devo(24, cycle)
        check_same(sim, orc)
    assert sim.devo_profile()["host_repacks"] == 2
    sim.run_steps(80, True)
    orc.steps(80)
    check_same(sim, orc)


def test_devo_rewiring_every_spring_bit_exact():
    """k larger than every robot: all springs get new pairs, rows change
    completely (the device path may fall back to the host re-pack)."""
    els = [e for e in robots.population("uneven", 96) if e.n_springs <= 1024][:12]
    assert len(els) == 12
    b = mb.pack(els)
    sim = mb.Simulator(0)
    sim.setTimeStep(1e-3)
    sim.set_batch(b)
    orc = OracleRun(b, mb.material_table(), np.float32(1e-3))
    for cycle in range(3):
        sim.run_steps(60, True)
        orc.steps(60)
        assert sim.devo(1024, seed=7 + cycle) == orc.devo(1024, 7 + cycle) == b.n_springs
        check_same(sim, orc)
    sim.run_steps(60, True)
    orc.steps(60)
    check_same(sim, orc)


def test_devo_through_simulator_api():
    """Simulator.Devo uses config.replaced_springs_per_element and a seed
    counting calls from 0; Collect returns the rewired springs."""
    els = robots.population("uneven", 6)
    sim = mb.Simulator(0)
    sim.Initialize(S.SimulatorConfig(time_step=1e-3, replaced_springs_per_element=32))
    trackers = sim.SetElements(els)
    sim.Simulate(0.05, True)
    orc = OracleRun(mb.pack(els), mb.material_table(), np.float32(1e-3))
    orc.steps(core.step_count(0.05, 1e-3))
    sim.Devo()
    sim.Devo()
    orc.devo(32, 0)
    orc.devo(32, 1)
    got = sim.Collect(trackers)
    ref = mb.pack(els)
    for r, e in enumerate(got):
        ms, ss = ref.robot_slices(r)
        assert np.array_equal(e.pairs, orc.b.pairs[ss])
        assert np.array_equal(e.spring_material, orc.b.spring_material[ss])
        assert np.array_equal(bits(e.mean_length), bits(orc.b.lbar[ss]))
        assert not np.array_equal(e.pairs, els[r].pairs)


def test_devo_force_water_streamed_bit_exact():
    """Point-cloud robots in water on the streamed path, two cycles."""
    b = robots.population_batch("nn", 3, mass=0.1)
    tab = mb.materials.force_table()
    sim = mb.Simulator(0)
    sim.set_materials(tab)
    sim.set_mode(2)
    sim.set_environment(**S.WATER)
    sim.setTimeStep(1e-4)
    sim.set_launch_config(streamed=1)
    sim.set_batch(b)
    assert sim.launch_config()["streamed"] == 1
    orc = OracleRun(b, tab, np.float32(1e-4), mode=2, env=S.WATER)
    for cycle in range(2):
        sim.run_steps(100, True)
        orc.steps(100)
        assert sim.devo(64, seed=100 + cycle) == orc.devo(64, 100 + cycle)
        check_same(sim, orc)
    assert sim.launch_config()["streamed"] == 1
    sim.run_steps(100, True)
    orc.steps(100)
    check_same(sim, orc)


def test_devo_keeps_a_fitting_override_and_replans_otherwise():
    b = robots.population_batch("uneven", 20)
    sim = mb.Simulator(0)
    sim.setTimeStep(1e-3)
    sim.set_launch_config(threads=1024, springs_per_thread=8, masses_per_thread=2, bins=20)
    sim.set_batch(b)
    sim.run_steps(50, True)
    sim.devo(8, 1)
    cfg = sim.launch_config()
    assert (cfg["threads"], cfg["springs_per_thread"], cfg["bins"]) == (1024, 8, 20)
    orc = OracleRun(b, mb.material_table(), np.float32(1e-3))
    orc.steps(50)
    orc.devo(8, 1)
    check_same(sim, orc)


def test_devo_large_population_properties():
    """Full-size population: every robot loses exactly its k highest
    stresses, pairs are distinct masses, steps after it stay finite."""
    b = robots.population_batch("uneven", 512)
    sim = mb.Simulator(0)
    sim.setTimeStep(1e-4)
    sim.set_batch(b)
    sim.run_steps(500, True)
    _, _, stress = sim.collect_arrays()
    k = 128
    assert sim.devo(k, 9) == 512 * k
    pairs, mat, lbar = sim.collect_springs()
    changed = (pairs != b.pairs).any(axis=1) | (mat != b.spring_material) | (bits(lbar) != bits(b.lbar))
    for r in range(0, 512, 37):
        s0, s1 = int(b.spring_offsets[r]), int(b.spring_offsets[r + 1])
        st = stress[s0:s1]
        order = np.lexsort((np.arange(s1 - s0), -st.astype(np.float64)))
        top = set(order[:k].tolist())
        assert set(np.nonzero(changed[s0:s1])[0].tolist()) <= top
    assert (pairs[:, 0] != pairs[:, 1])[changed].all()
    sim.run_steps(1000, False)
    assert not sim.robot_flags().any()
