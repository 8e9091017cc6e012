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
    # recall of the score's top fraction: the true top 10 (indices 90-99)
    # sit at score ranks 0-4 (95-99) and 26, 28, ..., 34 (90-94, between
    # indices 20-24), so the top 5 % holds half of them, the top 30 % seven
    score = -np.arange(100, dtype=np.float64)
    score[95:] = 10.0 + np.arange(5)
    score[90:95] = -20.5 - np.arange(5)
    q = evolve.quality(truth, truth, np.arange(90, 100), 0.25, score, fractions=(0.05, 0.3, 0.35))
    assert q["top10_recall_at"] == {"0.05": 0.5, "0.3": 0.7, "0.35": 1.0}


class _FakeEvaluator:
    """Fitness = share of muscle voxels (classes 3, 4): a stand-in for the
    simulator in host-logic tests."""

    def __init__(self):
        self.calls = []

    def __call__(self, g):
        self.calls.append(np.array(g, copy=True))
        return ((g >= 3).mean(1)).astype(np.float32)


class _FakeSurrogate:
    def __init__(self):
        self.steps = 0

    def predict(self, g):
        return ((g >= 3).mean(1) - 0.4).astype(np.float32)

    def train_step(self, g, t, lr):
        self.steps += 1
        return 0.0


def test_warmup_draws_random_batches_then_children_of_the_pool():
    ev = _FakeEvaluator()
    scr = evolve.ScreenedEvolution(ev, _FakeSurrogate(), seed=0, children=256, batch=64)
    w = scr.warmup(5 * 256, batch=256, epochs=1.0, random_batches=2)
    assert w["robots"] == 1280 and w["random_batches"] == 2 and len(ev.calls) == 5
    # children of an elite pool of muscle-rich genomes are muscle-richer than
    # random genomes (random: 0.35 on average)
    rand_share = np.mean([(c >= 3).mean() for c in ev.calls[:2]])
    kid_share = np.mean([(c >= 3).mean() for c in ev.calls[2:]])
    assert abs(rand_share - 0.35) < 0.02 and kid_share > rand_share + 0.05
    # all random when asked
    ev2 = _FakeEvaluator()
    evolve.ScreenedEvolution(ev2, _FakeSurrogate(), seed=0, children=256, batch=64).warmup(
        3 * 256, batch=256, epochs=1.0, random_batches=None)
    assert all(abs((c >= 3).mean() - 0.35) < 0.03 for c in ev2.calls)


def test_race_gives_each_method_the_same_budget():
    class Steady:
        def __init__(self, dt, gain):
            self.dt, self.gain, self.best = dt, gain, 0.0

        def generation(self):
            self.best += self.gain
            return {"wall_s": self.dt, "best": self.best}

    curves = evolve.race({"fast": Steady(0.25, 0.1), "slow": Steady(1.0, 0.3)}, 2.0)
    assert [t for t, _ in curves["fast"]] == [0.25, 0.5, 0.75, 1.0, 1.25, 1.5, 1.75, 2.0]
    assert [t for t, _ in curves["slow"]] == [1.0, 2.0]
    assert evolve.best_at(curves["fast"], 2.0) == pytest.approx(0.8)
    assert evolve.best_at(curves["slow"], 2.0) == pytest.approx(0.6)
    assert evolve.best_at(curves["slow"], 0.5) == float("-inf")
