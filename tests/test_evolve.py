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


def test_pool_holds_distinct_genomes():
    pool = evolve.Pool(size=3)
    g = np.arange(4, dtype=np.uint8)[:, None].repeat(216, 1)
    pool.add(np.concatenate([g, g]), np.array([1, 5, 3, 2, 1, 5, 3, 2], np.float32))
    assert list(pool.fitness) == [5, 3, 2]
    assert [int(x[0]) for x in pool.genomes] == [1, 2, 3]


def test_memo_finds_copies():
    m = evolve.Memo()
    g = np.random.default_rng(0).integers(0, 5, (5, 216)).astype(np.uint8)
    m.add(g[:3], np.array([0.1, 0.2, 0.3], np.float32))
    known, f = m.lookup(np.concatenate([g[2:], g[:1]]))
    assert list(known) == [True, False, False, True]
    assert f[0] == np.float32(0.3) and f[3] == np.float32(0.1) and np.isnan(f[1:3]).all()


def test_quality_counts_known_children_as_evaluated():
    truth = np.arange(100, dtype=np.float32)
    known = np.zeros(100, bool)
    known[95:] = True  # half of the best 10 known, never screened
    pred = truth.copy()
    pred[known] = np.nan
    q = evolve.quality(pred, truth, np.arange(90, 95), 0.25, pred, fractions=(0.1,), known=known)
    # the best 10 % of the 95 new children: indices 86-94 (9 of them)
    assert q["top10_recall"] == 1.0 and q["known_share"] == 0.05 and q["known_in_top10"] == 0.5
    assert q["top10_recall_new"] == pytest.approx(5 / 9)
    assert q["top10_recall_at"] == {"0.1": 1.0}
    assert q["random_screen_recall"] == pytest.approx(5 / 95)


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


def test_plain_and_screened_simulate_only_new_children():
    ev = _FakeEvaluator()
    scr = evolve.ScreenedEvolution(ev, _FakeSurrogate(), seed=0, children=256, batch=64, screen=0.25)
    scr.warmup(2 * 256, batch=256, epochs=1.0, random_batches=1)
    n0 = len(ev.calls)
    before = set(scr.memo.d)
    g = scr.generation(truth=True)
    new = 256 - g["known"]
    assert g["known"] > 0 and g["simulated"] == round(0.25 * new) + round(0.05 * new)
    # every simulated genome was new, and the truth pass simulated only new children
    assert not any(row.tobytes() in before for c in ev.calls[n0:] for row in c)
    assert len(ev.calls[n0]) == g["simulated"] and len(ev.calls[n0 + 1]) == new
    plain = evolve.PlainEvolution(ev, seed=1, children=256, pool=scr.pool, memo=scr.memo)
    k = len(ev.calls)
    p = plain.generation()
    assert p["simulated"] == len(ev.calls[k]) == 256 - p["known"] and p["known"] > 0
