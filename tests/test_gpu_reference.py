"""The CUDA step against the reference's own CUDA simulator, built from the
reference's sources into oracle/_ref (IEEE and -use_fast_math flavours) and
run in this process on the same robots.

The reference sums corrections with shared-memory atomics (run-to-run
nondeterministic) and calls sinf/norm3df where this build uses its own
correctly rounded operations, so agreement is within a tolerance: positions
within 2e-4 x body length over the first 1,000 steps, stresses within 1 %
of the largest, identical step counts and clocks.
"""
import ctypes
import os
import sys

import numpy as np
import pytest

import mercury_b200 as mb
from mercury_b200 import robots
from oracle import core

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
import make_fixtures as mf  # noqa: E402

FLAVOURS = {"ieee": mf.REF, "fast": mf.REF_FM}


def _gpu(b, dt, duration, track):
    sim = mb.Simulator(0)
    sim.setTimeStep(dt)
    sim.set_batch(b)
    n = sim.Simulate(duration, track)
    pos, vel, stress = sim.collect_arrays()
    return pos, vel, stress, n, sim.getTotalTime(), sim.CentreOfMass()


def test_matches_reference_fixture(golden_dir):
    b = robots.population_batch("small", 8)
    length = mb.body_length(b)
    g = np.load(os.path.join(golden_dir, "ref_sim.npz"))
    for i in range(int(g["n_cases"])):
        dt, dur = float(g[f"c{i}_dt"]), float(g[f"c{i}_duration"])
        pos, _, stress, n, t, _ = _gpu(b, dt, dur, True)
        assert n == int(g[f"c{i}_steps"]) and t == float(g[f"c{i}_total_time"])
        for r in range(b.n_robots):
            ms, _ = b.robot_slices(r)
            assert np.abs(pos[ms, :3] - g[f"c{i}_pos"][ms]).max() < 2e-4 * length[r]
        ref_s = g[f"c{i}_stress"]
        assert np.abs(stress - ref_s).max() < 1e-2 * np.abs(ref_s).max()


@pytest.mark.parametrize("flavour", sorted(FLAVOURS))
@pytest.mark.parametrize("dt", [1e-4, 1e-3, 5e-3])
def test_matches_live_reference_uneven(flavour, dt):
    path = FLAVOURS[flavour]
    if not os.path.exists(path):
        pytest.skip("reference build absent")
    L = mf.load(path)
    b = robots.population_batch("uneven", 24, seed_base=4242)
    length = mb.body_length(b)
    dur = float(np.float32(dt) * np.float32(999.5))  # 1,000 steps
    po, vo, st, tt, steps = mf.ref_simulate(L, b, dt, dur, True)
    pos, vel, stress, n, t, com = _gpu(b, dt, dur, True)
    assert n == steps == core.step_count(dur, dt) and t == tt
    for r in range(b.n_robots):
        ms, ss = b.robot_slices(r)
        assert np.abs(pos[ms, :3] - po[ms]).max() < 2e-4 * length[r], r
        assert np.abs(stress[ss] - st[ss]).max() <= 1e-2 * max(np.abs(st[ss]).max(), 1e-9), r
    # centre of mass of the non-air masses: absolute agreement (the step
    # conserves momentum, so displacements are small and relative errors are
    # ill-conditioned)
    ref_com = core.com_reference(b, np.concatenate([po, np.ones((len(po), 1), np.float32)], 1))
    assert np.abs(com - ref_com).max() < 2e-4 * length.max()


def test_headline_population_matches_live_reference():
    """The bench's whole population (512 uneven robots, the headline
    workload's seeds) against the reference's own CUDA simulator over the
    first 1,000 steps at dt = 1e-4 (IEEE flavour): every robot within the
    stated tolerance."""
    path = FLAVOURS["ieee"]
    if not os.path.exists(path):
        pytest.skip("reference build absent")
    L = mf.load(path)
    b = robots.population_batch("uneven", seed_base=1000)
    assert b.n_robots == 512
    length = mb.body_length(b)
    dur = float(np.float32(1e-4) * np.float32(999.5))
    po, _, _, tt, steps = mf.ref_simulate(L, b, 1e-4, dur, False)
    pos, _, _, n, t, _ = _gpu(b, 1e-4, dur, False)
    assert n == steps == 1000 and t == tt
    worst = 0.0
    for r in range(b.n_robots):
        ms, _ = b.robot_slices(r)
        worst = max(worst, float(np.abs(pos[ms, :3] - po[ms]).max() / length[r]))
    print(f"\n512 robots, 1,000 steps: max |x - x_ref| / body length = {worst:.2e}")
    assert worst < 2e-4
