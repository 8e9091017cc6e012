"""Surrogate-screened evolution of voxel robots (the learned part of the
batched simulator), beside plain evolution that simulates every candidate.

Genomes are 6x6x6 voxel grids of 5 classes (air .3, bone .175, tissue .175,
muscle a .175, muscle b .175 when drawn at random).  A genome's fitness is the
horizontal displacement of its robot's centre of mass (non-air masses) after
1 s on land -- force mode, dt = 1e-4, 0.1 kg masses, 0.1 m cells, the robot
built on the device (Simulator.set_voxel_population) and stepped from t = 0.

One generation, as the reference optimiser's child step does it
(optimize/optimizer/optimizer_impl.h:113-276, steady state with elitism): 4096
children of parents drawn by rank from the elite pool, crossover with
probability 0.7 (a random axis-aligned cut between two parents), mutation
with probability 0.6 (one voxel plus each other with probability 2/216
redrawn); the children are
evaluated, and the pool keeps the best simulated genomes.

Warm-up: 53,248 simulated robots -- three batches of 4096 random genomes,
then batches of children of the elite pool so far (plain evolution), so that
the surrogate trains on the distribution it will screen -- then 60 epochs
with a cosine learning rate.

Both methods keep the fitness of every genome they have simulated (the
simulator is deterministic to the bit, so a copy needs no simulation): a
child identical to a simulated genome -- a fifth to a quarter of the
children, the unchanged copies of a parent and the crossovers of a parent
with itself -- takes its known fitness.  The elite pool holds distinct
genomes.

Screened: the surrogate predicts the new children (the mean over the 8
horizontal orientations of each, plus `kappa` times their spread: children
the orientations disagree on are the least certain), its top `screen`
fraction plus a random `audit` fraction of the rest are simulated, and the
surrogate trains on the new (genome, fitness) pairs; the others are
discarded unsimulated.  A child differs from its (simulated) parents in a
few voxels, so each prediction is corrected by the surrogate's error on the
parents, weighted by the share of voxels from each (lineage correction).
Training draws every sample in a random orientation; per generation, a few
steps whose batches are half from the newest generation.
Plain: every new child is simulated.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np

from . import materials
from . import simulator as S
from .surrogate import Surrogate, to_cells

P_CLASS = np.array([0.3, 0.175, 0.175, 0.175, 0.175])
CELL, MASS, DT, DURATION = 0.1, 0.1, 1e-4, 1.0


def _orientations() -> np.ndarray:
    """The 8 symmetries of the horizontal square (mirror x, mirror y, swap x
    and y) as voxel permutations: oriented[v] = genome[perm[v]].  Gravity
    fixes z; a mirrored or turned robot moves as far (simulated: Spearman
    0.99 between the fitness of a child and of its mirror image)."""
    v = np.arange(216)
    x, y, z = v % 6, (v // 6) % 6, v // 36
    out = []
    for mx in (0, 1):
        for my in (0, 1):
            for sw in (0, 1):
                xx, yy = (5 - x if mx else x), (5 - y if my else y)
                if sw:
                    xx, yy = yy, xx
                out.append(xx + 6 * yy + 36 * z)
    return np.array(out)


ORIENTATIONS = _orientations()


def random_genomes(rng: np.random.Generator, n: int) -> np.ndarray:
    return rng.choice(5, size=(n, 216), p=P_CLASS).astype(np.uint8)


class Evaluator:
    """Simulates genomes on one GPU; one Simulator per batch size (rounded
    up to a multiple of `bucket` with copies of the first genome, whose
    results are dropped) so that each keeps its packing plan.  With `autotune`, the launch configuration
    of each batch size is tuned on its first call (measured on 6x6x6 genomes:
    no faster than the automatic plan, and seconds of tuning per size)."""

    def __init__(self, device: int = 0, duration: float = DURATION, autotune: bool = False, bucket: int = 256):
        self.device = device
        self.bucket = bucket
        self.duration = duration
        self.autotune = autotune
        self._sims: dict[int, S.Simulator] = {}
        self._tuned: dict[int, dict] = {}
        self.simulated = 0

    def _sim(self, n: int) -> S.Simulator:
        sim = self._sims.get(n)
        if sim is None:
            sim = S.Simulator(self.device)
            sim.set_materials(materials.force_table())
            sim.set_mode(S.MODE_FORCE_LAND)
            sim.set_environment(**S.LAND)
            sim.setTimeStep(DT)
            self._sims[n] = sim
        return sim

    def __call__(self, genomes: np.ndarray) -> np.ndarray:
        n = len(genomes)
        if n == 0:
            return np.zeros(0, np.float32)
        size = -(-n // self.bucket) * self.bucket
        if size > n:
            genomes = np.concatenate([genomes, np.repeat(genomes[:1], size - n, axis=0)])
        sim = self._sim(size)
        cells = to_cells(genomes)
        if self.autotune and n not in self._tuned:
            # launch configuration for this batch size, tuned once on these
            # genomes (the packing plan is per batch size and grid)
            from . import autotune
            sim.set_voxel_population(cells, CELL, MASS)
            up = lambda: sim.set_voxel_population(cells, CELL, MASS)  # noqa: E731
            self._tuned[n] = autotune.tune(sim, sim.batch, steps=300, upload=up, use_cache=False)["config"]
        sim.set_voxel_population(cells, CELL, MASS)
        sim.Reset()
        com0 = sim.CentreOfMass()
        steps = sim.Simulate(self.duration)
        com1 = sim.CentreOfMass()
        d = com1.astype(np.float64) - com0
        fit = np.hypot(d[:, 0], d[:, 1])
        fit[~np.isfinite(fit)] = 0.0
        self.simulated += n
        self.last_steps = steps
        return fit[:n].astype(np.float32)


def make_children(rng: np.random.Generator, parents: np.ndarray, fitness: np.ndarray, n: int,
                  p_cross: float = 0.7, p_mut: float = 0.6, lineage: bool = False):
    """Children of rank-selected parents: axis-aligned cut crossover, then
    redraws of about 1 + Poisson(2) voxels.  With `lineage`, also returns
    each child's parents (indices into `parents`) and the share of its
    voxels taken from the second one."""
    order = np.argsort(-fitness, kind="stable")
    P = len(parents)
    w = 1.0 / (1.0 + np.arange(P))  # rank weights
    w /= w.sum()
    ia = order[rng.choice(P, size=n, p=w)]
    ib = order[rng.choice(P, size=n, p=w)]
    a, b = parents[ia], parents[ib]
    kids = a.copy()
    share_b = np.zeros(n)
    cross = rng.random(n) < p_cross
    if cross.any():
        coord = np.stack(np.meshgrid(np.arange(6), np.arange(6), np.arange(6), indexing="ij"), -1)
        coord = coord.reshape(216, 3)[:, ::-1]  # voxel v = x + 6y + 36z -> (x, y, z)
        axis = rng.integers(0, 3, n)
        cut = rng.integers(1, 6, n)
        side = coord[:, axis].T  # (n, 216): each child's coordinate along its cut axis
        take_b = (side >= cut[:, None]) & cross[:, None]
        kids[take_b] = b[take_b]
        share_b = take_b.mean(1)
    mut = rng.random(n) < p_mut
    m = int(mut.sum())
    if m:
        # one voxel surely, every other with probability 2/216: about
        # 1 + Poisson(2) redraws per mutated child
        mask = rng.random((m, 216)) < 2.0 / 216.0
        mask[np.arange(m), rng.integers(0, 216, m)] = True
        rows = kids[mut]
        rows[mask] = rng.choice(5, size=int(mask.sum()), p=P_CLASS)
        kids[mut] = rows
    if lineage:
        return kids, ia, ib, share_b
    return kids


@dataclass
class Pool:
    """Elite pool: the best distinct simulated genomes."""
    size: int = 256
    genomes: np.ndarray = field(default_factory=lambda: np.zeros((0, 216), np.uint8))
    fitness: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float32))

    def add(self, g: np.ndarray, f: np.ndarray) -> None:
        G = np.concatenate([self.genomes, np.asarray(g, np.uint8)])
        F = np.concatenate([self.fitness, np.asarray(f, np.float32)])
        order = np.argsort(-F, kind="stable")
        keep, seen = [], set()
        for i in order:  # best first; a genome already kept is a copy
            k = G[i].tobytes()
            if k in seen:
                continue
            seen.add(k)
            keep.append(i)
            if len(keep) == self.size:
                break
        self.genomes, self.fitness = G[keep], F[keep]


class Memo:
    """Fitness of every simulated genome, by genome bytes."""

    def __init__(self):
        self.d: dict[bytes, float] = {}

    def add(self, g: np.ndarray, f: np.ndarray) -> None:
        for row, v in zip(np.asarray(g, np.uint8), f):
            self.d[row.tobytes()] = float(v)

    def lookup(self, g: np.ndarray):
        """(known mask, fitness with NaN where unknown)."""
        f = np.array([self.d.get(row.tobytes(), np.nan) for row in np.asarray(g, np.uint8)], np.float32)
        return ~np.isnan(f), f

    def __len__(self):
        return len(self.d)


class Dataset:
    def __init__(self):
        self.g: list[np.ndarray] = []
        self.f: list[np.ndarray] = []
        self._cat = None

    def add(self, g, f):
        self.g.append(np.asarray(g, np.uint8))
        self.f.append(np.asarray(f, np.float32))
        self._cat = None

    def arrays(self):
        if self._cat is None:
            self._cat = (np.concatenate(self.g), np.concatenate(self.f))
        return self._cat

    def __len__(self):
        return sum(len(x) for x in self.f)


class ScreenedEvolution:
    """Screening with the surrogate.  Training draws every sample in a random
    orientation (the fitness does not change); predictions average the 8
    orientations."""

    def __init__(self, evaluator: Evaluator, surrogate, seed: int = 0, children: int = 4096,
                 screen: float = 0.25, audit: float = 0.05, batch: int = 256, lr: float = 1e-3,
                 steps_per_generation: int = 60, finetune_lr: float = 3e-4, lineage_correction: bool = True,
                 kappa: float = 1.0):
        """`surrogate`: one Surrogate or a list of them (an ensemble: each
        member trains on its own minibatches, predictions are averaged)."""
        self.ev = evaluator
        self.members = list(surrogate) if isinstance(surrogate, (list, tuple)) else [surrogate]
        self.sg = self.members[0]
        self.rng = np.random.default_rng(seed)
        self.children, self.screen, self.audit = children, screen, audit
        self.batch, self.lr, self.steps, self.finetune_lr = batch, lr, steps_per_generation, finetune_lr
        self.lineage_correction = lineage_correction
        self.kappa = kappa  # screening bonus per unit of spread over the orientations
        self.data = Dataset()
        self.pool = Pool()
        self.memo = Memo()
        self.mu, self.sd = 0.0, 1.0
        self.trained_steps = 0

    def predict(self, genomes: np.ndarray, spread: bool = False):
        """Mean prediction over the 8 orientations (and the members); with
        `spread`, also the standard deviation over them."""
        g = np.asarray(genomes, np.uint8)
        views = [np.ascontiguousarray(g[:, p]) for p in ORIENTATIONS]
        preds = np.array([sg.predict(v) for sg in self.members for v in views])
        return (preds.mean(0), preds.std(0)) if spread else preds.mean(0)

    def _norm(self):
        _, f = self.data.arrays()
        self.mu, self.sd = float(f.mean()), float(f.std() + 1e-9)

    def train(self, steps: int, lr: float, recent: tuple | None = None, cosine: bool = False) -> float:
        g, f = self.data.arrays()
        loss = 0.0
        for i in range(steps):
            step_lr = lr * 0.5 * (1.0 + np.cos(np.pi * i / steps)) if cosine else lr
            for sg in self.members:
                idx = self.rng.integers(0, len(f), self.batch)
                gb, fb = g[idx], f[idx]
                if recent is not None:  # half of every batch from the newest generation
                    r = self.rng.integers(0, len(recent[1]), self.batch // 2)
                    gb = np.concatenate([gb[: self.batch - len(r)], recent[0][r]])
                    fb = np.concatenate([fb[: self.batch - len(r)], recent[1][r]])
                gb = np.take_along_axis(gb, ORIENTATIONS[self.rng.integers(0, 8, len(gb))], axis=1)
                loss = sg.train_step(gb, (fb - self.mu) / self.sd, step_lr)
            self.trained_steps += 1
        return loss

    def warmup(self, n: int, batch: int = 4096, epochs: float = 60.0, random_batches: int | None = 3) -> dict:
        """Simulates n robots in batches and trains on them.  The first
        `random_batches` batches are random genomes; the others are children
        of the elite pool so far (plain evolution: every child simulated),
        so that the surrogate learns the distribution it will screen --
        children a few voxels away from good parents.  None: every batch
        random."""
        t0 = time.perf_counter()
        for k, i in enumerate(range(0, n, batch)):
            m = min(batch, n - i)
            if random_batches is None or k < random_batches or len(self.pool.fitness) == 0:
                g = random_genomes(self.rng, m)
            else:
                g = make_children(self.rng, self.pool.genomes, self.pool.fitness, m)
            f = self.ev(g)
            self.data.add(g, f)
            self.pool.add(g, f)
            self.memo.add(g, f)
        t1 = time.perf_counter()
        self._norm()
        loss = self.train(int(epochs * n / self.batch), self.lr, cosine=True)
        return {"robots": n, "random_batches": random_batches, "simulate_s": t1 - t0,
                "train_s": time.perf_counter() - t1, "loss": loss, "train_steps": self.trained_steps}

    def select(self, pred: np.ndarray) -> np.ndarray:
        n = len(pred)
        k = int(round(self.screen * n))
        order = np.argsort(-pred, kind="stable")
        top, rest = order[:k], order[k:]
        audit = self.rng.choice(rest, size=int(round(self.audit * n)), replace=False)
        return np.concatenate([top, audit])

    def generation(self, truth: bool = False) -> dict:
        t0 = time.perf_counter()
        kids, ia, ib, sb = make_children(self.rng, self.pool.genomes, self.pool.fitness, self.children,
                                         lineage=True)
        known, fk = self.memo.lookup(kids)
        nov = np.nonzero(~known)[0]
        t1 = time.perf_counter()
        pred = np.full(len(kids), np.nan)
        score = np.full(len(kids), np.nan)
        sel = nov[:0]
        if len(nov):
            p, spread = self.predict(kids[nov], spread=True)
            if self.lineage_correction:
                # a child is a near copy of simulated parents: carry over the
                # surrogate's error on them
                res = self.pool.fitness - self.predict(self.pool.genomes) * self.sd - self.mu
                p = p * self.sd + self.mu + (1.0 - sb[nov]) * res[ia[nov]] + sb[nov] * res[ib[nov]]
            pred[nov] = p
            # children the orientations disagree on get a bonus (their fitness
            # is the least certain), in fitness units
            score[nov] = p + self.kappa * self.sd * spread
            sel = nov[self.select(score[nov])]
        t2 = time.perf_counter()
        f = self.ev(kids[sel])
        t3 = time.perf_counter()
        self.data.add(kids[sel], f)
        self.memo.add(kids[sel], f)
        self.pool.add(kids[sel], f)
        if len(sel):
            self.train(self.steps, self.finetune_lr, recent=(kids[sel], f))
        t4 = time.perf_counter()
        out = {"wall_s": t4 - t0, "children_s": t1 - t0, "screen_s": t2 - t1, "simulate_s": t3 - t2,
               "train_s": t4 - t3, "simulated": len(sel), "known": int(known.sum()),
               "best": float(self.pool.fitness[0])}
        if truth:  # ground truth for every new child, outside the timed region
            ft = fk.copy()
            ft[nov] = self.ev(kids[nov])
            out.update(quality(pred, ft, sel, self.screen, score, known=known))
        return out


class PlainEvolution:
    """Every new child simulated (copies of simulated genomes take their
    known fitness)."""

    def __init__(self, evaluator: Evaluator, seed: int = 0, children: int = 4096, pool: Pool | None = None,
                 memo: Memo | None = None):
        self.ev = evaluator
        self.rng = np.random.default_rng(seed)
        self.children = children
        self.pool = pool or Pool()
        self.memo = memo or Memo()

    def generation(self) -> dict:
        t0 = time.perf_counter()
        kids = make_children(self.rng, self.pool.genomes, self.pool.fitness, self.children)
        known, f = self.memo.lookup(kids)
        nov = np.nonzero(~known)[0]
        t1 = time.perf_counter()
        f[nov] = self.ev(kids[nov])
        t2 = time.perf_counter()
        self.memo.add(kids[nov], f[nov])
        self.pool.add(kids, f)
        return {"wall_s": time.perf_counter() - t0, "children_s": t1 - t0, "simulate_s": t2 - t1,
                "simulated": len(nov), "known": int(known.sum()), "best": float(self.pool.fitness[0])}


def race(methods: dict, seconds: float) -> dict:
    """Runs each method's generations (objects with .generation() returning
    wall_s and best) for the same wall-time budget, one method after the
    other, and returns per method the (elapsed seconds, best fitness) after
    each generation -- best fitness against wall time at an equal budget."""
    out = {}
    for name, m in methods.items():
        t, curve = 0.0, []
        while t < seconds:
            g = m.generation()
            t += g["wall_s"]
            curve.append((round(t, 4), g["best"]))
        out[name] = curve
    return out


def best_at(curve: list, seconds: float) -> float:
    """Best fitness reached within `seconds` on a race curve."""
    best = [b for t, b in curve if t <= seconds]
    return max(best) if best else float("-inf")


def quality(pred: np.ndarray, truth: np.ndarray, selected: np.ndarray, screen: float,
            score: np.ndarray | None = None, fractions=(0.2, 0.25, 0.3, 0.35, 0.4, 0.5),
            known: np.ndarray | None = None) -> dict:
    """Quality of a screen over the children of one generation.  `known`
    marks children whose fitness was known without simulation (copies of
    simulated genomes); the others are new, and only they are predicted,
    ranked and screened.

    - top10_recall: the share of the truly best 10% of all children whose
      fitness the generation obtained -- known, or simulated because the
      screen (surrogate top `screen` + audit) selected them;
    - top10_recall_new: the share of the truly best 10% of the new children
      that the screen selected (the surrogate's own part);
    - top10_recall_top10: the share of that best 10% inside the surrogate's
      own top 10% of the new children;
    - random_screen_recall: what random screening of the same size would
      give on the new children;
    - spearman: rank correlation of predictions and simulated fitness over
      the new children;
    - with the screening `score`: top10_recall_at, the recall on the new
      children of the score's top fraction alone (no audit) for each of
      `fractions`."""
    from scipy.stats import spearmanr
    n = len(truth)
    known = np.zeros(n, bool) if known is None else np.asarray(known, bool)
    new = np.nonzero(~known)[0]
    m = len(new)
    sel = set(np.asarray(selected).tolist())
    top = np.argsort(-truth, kind="stable")[: n // 10]
    top_new = new[np.argsort(-truth[new], kind="stable")[: m // 10]]
    own = new[np.argsort(-pred[new], kind="stable")[: m // 10]]
    tn = set(top_new.tolist())

    def rec(s):
        return len(tn & s) / len(tn) if tn else 1.0
    out = {
        "spearman": float(spearmanr(pred[new], truth[new]).correlation) if m > 1 else float("nan"),
        "top10_recall": float(np.mean([(i in sel) or known[i] for i in top])) if len(top) else 1.0,
        "top10_recall_new": rec(sel),
        "top10_recall_top10": rec(set(own.tolist())),
        "random_screen_recall": len(sel) / m if m else 1.0,
        "known_share": float(known.mean()) if n else 0.0,
        "known_in_top10": float(np.mean(known[top])) if len(top) else 0.0,
    }
    if score is not None:
        ranked = new[np.argsort(-score[new], kind="stable")]
        out["top10_recall_at"] = {str(fr): rec(set(ranked[: int(round(fr * m))].tolist())) for fr in fractions}
    return out
