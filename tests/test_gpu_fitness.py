"""Fitness over a full evaluation against the reference's own Simulator.

The reference (DawsonCohen/Mercury) is compiled from its sources into
oracle/_ref (IEEE and -use_fast_math flavours) and runs here on the GPU on
the same seeded robots, built by its own VoxelRobot::Build
(oracle/population.py).  One evaluation = Simulate(1 s) from rest:
10,000 steps at dt = 1e-4 (the benchmark configurations' step), 1,000 at
1e-3 (the reference's tests, common/tests/test_simulator.cpp:32) and 200 at
5e-3 (the reference's default, common/util/config.h:19), where the XPBD
springs act.

Fitness is SoftBody::updateFitness (common/evolvables/SoftBody.cpp:124-137):
max((COMx - baseCOMx) / length, 0), the COM over non-air masses
(SoftBody.cpp:112-121) and the length from the build (SoftBody.cpp:98-110).
For this build the COM is the library's device reduction
(Simulator.CentreOfMass); for the reference, its running mean over the
collected masses (oracle.core.com_reference).

Tolerance: population relative error sum|f - f_ref| / sum|f_ref| <= 1 %
(the target fitness agreement), and the same error between two runs of the
reference itself (its shared-memory atomics make it run-to-run
nondeterministic) is printed beside it.
"""
import os

import numpy as np
import pytest

import mercury_b200 as mb
from mercury_b200 import robots
from oracle import core, population

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FLAVOURS = {"ieee": os.path.join(ROOT, "oracle", "_ref", "libmercury_ref.so"),
            "fast": os.path.join(ROOT, "oracle", "_ref", "libmercury_ref_fm.so")}
POPULATIONS = {"small": ("small", 32, 0), "uneven": ("uneven", 48, 4242)}
REL_TOL = 0.01
_LIBS = {}


def _ref(flavour):
    import ctypes
    if flavour not in _LIBS:
        L = ctypes.CDLL(FLAVOURS[flavour])
        L.ref_decode_id.argtypes = [ctypes.c_uint32]
        L.ref_decode_id(1)
        L.ref_simulate_timed.argtypes = ([ctypes.c_int] + [ctypes.c_void_p] * 8 +
                                         [ctypes.c_float, ctypes.c_float, ctypes.c_int] + [ctypes.c_void_p] * 3)
        L.ref_simulate_timed.restype = ctypes.c_int
        _LIBS[flavour] = L
    return _LIBS[flavour]


def ref_positions(flavour, b, dt, duration):
    import ctypes
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    pos3 = np.ascontiguousarray(b.pos[:, :3])
    vel3 = np.ascontiguousarray(b.vel[:, :3])
    po, vo = np.zeros_like(pos3), np.zeros_like(vel3)
    secs = np.zeros(2, np.float64)
    n = _ref(flavour).ref_simulate_timed(
        b.n_robots, P(b.mass_offsets.astype(np.int32)), P(pos3), P(vel3), P(b.mass_material),
        P(b.spring_offsets.astype(np.int32)), P(np.ascontiguousarray(b.pairs)), P(b.lbar),
        P(b.spring_material), dt, duration, 0, P(po), P(vo), P(secs))
    return np.concatenate([po, np.ones((len(po), 1), np.float32)], 1), n


def fitness_of(com, base, length):
    return np.maximum((com[:, 0] - base[:, 0]) / length, 0.0).astype(np.float32)


def rel_error(f, f_ref):
    return float(np.abs(f.astype(np.float64) - f_ref).sum() / max(np.abs(f_ref.astype(np.float64)).sum(), 1e-30))


@pytest.mark.parametrize("flavour", sorted(FLAVOURS))
@pytest.mark.parametrize("dt", [1e-4, 1e-3, 5e-3])
@pytest.mark.parametrize("pop", sorted(POPULATIONS))
def test_fitness_matches_reference_over_full_evaluation(pop, dt, flavour):
    if not os.path.exists(FLAVOURS[flavour]):
        pytest.skip("reference build absent")
    name, n, seed = POPULATIONS[pop]
    rb = population.population_batch(name, n, seed)
    b = robots.population_batch(name, n, seed)
    duration = 1.0
    base = rb.base_com  # the reference's own SoftBody::mBaseCOM after the build

    p1, n1 = ref_positions(flavour, rb, dt, duration)
    p2, _ = ref_positions(flavour, rb, dt, duration)
    f_ref = fitness_of(core.com_reference(rb, p1), base, rb.length)
    f_ref2 = fitness_of(core.com_reference(rb, p2), base, rb.length)

    sim = mb.Simulator(0)
    sim.setTimeStep(dt)
    sim.set_batch(b)
    steps = sim.Simulate(duration)
    assert steps == n1 == core.step_count(duration, dt)
    f = fitness_of(sim.CentreOfMass(), base, rb.length)

    err, spread = rel_error(f, f_ref), rel_error(f_ref2, f_ref)
    moving = int(np.count_nonzero(f_ref > 0))
    print(f"\nfitness {pop} dt={dt:g} {flavour}: {steps} steps, mean fitness {f_ref.mean():.3e}, "
          f"{moving}/{n} robots > 0; relative error vs reference {err:.2e}, "
          f"reference run-to-run {spread:.2e}; max |df| {np.abs(f - f_ref).max():.2e}")
    assert f_ref.sum() > 0, "no robot moved forward: the comparison would be empty"
    assert err <= REL_TOL, (err, spread)
