"""Surrogate-screened evolution on the device: the evaluator's fitness is
the oracle's to the bit, and a trained surrogate screens better than random
screening of the same size (what the network gains over the method without
it)."""
import numpy as np
import pytest

import mercury_b200 as mb
from mercury_b200 import evolve, robots
from mercury_b200 import simulator as S
from mercury_b200.surrogate import Surrogate, to_cells
from oracle import core

pytestmark = pytest.mark.gpu

ENV_KEYS = ("g", "floor_stiffness", "friction_static", "friction_kinetic", "drag", "damping")


def test_evaluator_fitness_matches_oracle():
    rng = np.random.default_rng(3)
    g = evolve.random_genomes(rng, 24)
    ev = evolve.Evaluator(0, duration=0.03)
    f = ev(g)
    b = mb.pack([robots.voxel_robot(c, evolve.CELL, evolve.MASS) for c in to_cells(g)])
    n = core.step_count(0.03, evolve.DT)
    p, v = b.pos.copy(), b.vel.copy()
    core.force_run(1, b, p, v, np.zeros(b.n_springs, np.float32), mb.materials.force_table(),
                   [S.LAND[k] for k in ENV_KEYS], evolve.DT, 0.0, n, False)
    d = core.com_device(b, p).astype(np.float64) - core.com_device(b, b.pos)
    fo = np.hypot(d[:, 0], d[:, 1]).astype(np.float32)
    assert np.array_equal(f.view(np.uint32), fo.view(np.uint32))
    assert ev.last_steps == n


def test_screening_beats_random_screening():
    ev = evolve.Evaluator(0)
    sg = Surrogate(0, max_batch=1024, seed=0)
    scr = evolve.ScreenedEvolution(ev, sg, seed=1, children=2048)
    warm = scr.warmup(4 * 4096, epochs=30)
    assert warm["robots"] == 16384
    g = scr.generation(truth=True)
    new = 2048 - g["known"]  # copies of simulated genomes are not screened
    assert g["simulated"] == round(0.25 * new) + round(0.05 * new)
    assert g["random_screen_recall"] == pytest.approx(g["simulated"] / new)
    assert g["top10_recall_new"] > g["random_screen_recall"] + 0.2, g
    assert g["spearman"] > 0.3, g
