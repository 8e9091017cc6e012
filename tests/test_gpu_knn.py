"""k-nearest-neighbour springs built on the GPU (mb_knn_springs) against the
host builder of the point-cloud robots, bit for bit: pairs, order, mean
lengths, materials -- including point sets full of equal distances."""
import numpy as np
import pytest

from mercury_b200 import robots
from mercury_b200.materials import composite_id

pytestmark = pytest.mark.gpu


def host_springs(p, mats, k):
    n = len(p)
    d2 = ((p[:, None, :] - p[None, :, :]) ** 2).sum(-1)
    np.fill_diagonal(d2, np.inf)
    nb = np.argsort(d2, axis=1, kind="stable")[:, :k]
    i = np.repeat(np.arange(n), k)
    j = nb.reshape(-1)
    pairs = np.unique(np.stack([np.minimum(i, j), np.maximum(i, j)], 1), axis=0)
    diff = p[pairs[:, 0]] - p[pairs[:, 1]]
    lbar = np.sqrt((diff * diff).sum(1)).astype(np.float32)
    smat = np.array([composite_id(int(mats[u]), int(mats[v])) for u, v in pairs], np.uint8)
    return pairs.astype(np.uint16), smat, lbar


def test_nn_population_matches_host_builder():
    host = robots.population("nn", 6, mass=0.1)
    dev = robots.nn_population_device(6, mass=0.1)
    for h, d in zip(host, dev):
        assert np.array_equal(h.pos.view(np.uint32), d.pos.view(np.uint32))
        assert np.array_equal(h.pairs, d.pairs)
        assert np.array_equal(h.spring_material, d.spring_material)
        assert np.array_equal(h.mean_length.view(np.uint32), d.mean_length.view(np.uint32))


@pytest.mark.parametrize("k", [1, 6, 25, 32])
def test_ties_and_k(k):
    # a lattice: many equal distances, ties broken by the lower index
    g = np.stack(np.meshgrid(np.arange(7), np.arange(6), np.arange(5), indexing="ij"), -1).reshape(-1, 3)
    p = (g * 0.1).astype(np.float32)
    rng = np.random.default_rng(k)
    mats = robots.FOUR[rng.integers(0, 4, len(p))]
    q = rng.uniform(0, 1, (300, 3)).astype(np.float32)
    mq = robots.FOUR[rng.integers(0, 4, len(q))]
    so, pairs, smat, lbar = robots.knn_springs([p, q], [mats, mq], k)
    for r, (pts, mm) in enumerate(((p, mats), (q, mq))):
        hp, hm, hl = host_springs(pts, mm, k)
        s = slice(int(so[r]), int(so[r + 1]))
        assert np.array_equal(pairs[s], hp)
        assert np.array_equal(smat[s], hm)
        assert np.array_equal(lbar[s].view(np.uint32), hl.view(np.uint32))


def test_many_small_clouds():
    rng = np.random.default_rng(9)
    pts = [rng.normal(size=(int(rng.integers(30, 200)), 3)).astype(np.float32) for _ in range(40)]
    mats = [robots.FOUR[rng.integers(0, 4, len(p))] for p in pts]
    so, pairs, smat, lbar = robots.knn_springs(pts, mats, 25)
    for r in range(40):
        hp, hm, hl = host_springs(pts[r], mats[r], 25)
        s = slice(int(so[r]), int(so[r + 1]))
        assert np.array_equal(pairs[s], hp) and np.array_equal(lbar[s].view(np.uint32), hl.view(np.uint32))
