"""Host logic of the surrogate-screened evolution (mercury_b200/evolve.py)."""
import numpy as np
import pytest

from mercury_b200 import evolve


def test_orientations_form_the_square_symmetry_group():
    P = evolve.ORIENTATIONS
    assert P.shape == (8, 216)
    assert len({tuple(p) for p in P}) == 8
    for p in P:
        assert sorted(p) == list(range(216))
        # z layers stay put
        assert (p // 36 == np.arange(216) // 36).all()
    comp = {tuple(a[b]) for a in P for b in P}
    assert comp == {tuple(p) for p in P}


def test_children_stay_in_range_and_mix_parents():
    rng = np.random.default_rng(0)
    parents = evolve.random_genomes(rng, 64)
    fit = rng.random(64).astype(np.float32)
    kids = evolve.make_children(rng, parents, fit, 4096)
    assert kids.shape == (4096, 216) and kids.dtype == np.uint8 and kids.max() <= 4
    # children differ from every parent by little, and the best parents have
    # the most children (rank selection)
    d = (kids[:, None, :] != parents[None, :, :]).sum(2).min(1)
    assert np.median(d) < 40
    best = np.argmax(fit)
    near = (kids != parents[best]).sum(1) < 10
    assert near.sum() > 4096 / 64


def test_pool_keeps_the_best():
    pool = evolve.Pool(size=4)
    g = np.arange(10, dtype=np.uint8)[:, None].repeat(216, 1)
    pool.add(g, np.arange(10, dtype=np.float32))
    assert list(pool.fitness) == [9, 8, 7, 6]
    assert (pool.genomes[0] == 9).all()


def test_quality_metrics():
    truth = np.arange(100, dtype=np.float32)
    q = evolve.quality(truth.copy(), truth, np.arange(90, 100), 0.25)
    assert q["spearman"] == pytest.approx(1.0) and q["top10_recall"] == 1.0 and q["top10_recall_top10"] == 1.0
    q = evolve.quality(-truth, truth, np.arange(0, 10), 0.25)
    assert q["top10_recall"] == 0.0 and q["random_screen_recall"] == 0.1
