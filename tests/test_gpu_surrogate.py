"""The surrogate's CUDA kernels (BF16 tensor-core GEMMs, FP32 accumulation)
against the CPU oracle with the same BF16 rounding points: predictions,
loss and every parameter gradient; determinism; and that training on the
device fits a learnable target."""
import numpy as np
import pytest

from mercury_b200.surrogate import Surrogate, to_cells
from oracle import surrogate as so

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def test_predictions_match_oracle():
    rng = np.random.default_rng(0)
    flat = so.init_params(5)
    s = Surrogate(0, max_batch=64)
    s.set_params(flat)
    assert np.array_equal(s.get_params(), flat)
    genomes = rng.integers(0, 5, (100, 216)).astype(np.uint8)  # two chunks
    y = s.predict(genomes)
    yo, _ = so.Net(flat).forward(genomes)
    assert rel(y, yo) < 1e-2
    assert np.abs(y - yo).max() <= 2e-2 * np.abs(yo).max()


@pytest.mark.parametrize("n", [1, 100, 700])
def test_tcgen05_forward_matches_mma_sync(n):
    """The forward on tcgen05 (TMEM accumulators) against the mma.sync
    kernel and the oracle, with partial tiles (M not a multiple of 128)."""
    rng = np.random.default_rng(10 + n)
    flat = so.init_params(8)
    s = Surrogate(0, max_batch=256)
    s.set_params(flat)
    genomes = rng.integers(0, 5, (n, 216)).astype(np.uint8)
    s.use_tcgen05(True)
    y_tc = s.predict(genomes)
    s.use_tcgen05(False)
    y_ms = s.predict(genomes)
    yo, _ = so.Net(flat).forward(genomes)
    scale = np.abs(yo).max()
    assert np.abs(y_tc - y_ms).max() <= 2e-2 * scale
    assert np.abs(y_tc - yo).max() <= 2e-2 * scale
    assert rel(y_tc, yo) < 1e-2


def test_gradients_match_oracle():
    rng = np.random.default_rng(1)
    flat = so.init_params(6)
    s = Surrogate(0, max_batch=96)
    s.set_params(flat)
    genomes = rng.integers(0, 5, (96, 216)).astype(np.uint8)
    targets = rng.normal(size=96).astype(np.float32)
    loss, g = s.gradients(genomes, targets)
    lo, _, go = so.Net(flat).loss_and_grads(genomes, targets)
    assert abs(loss - lo) <= 1e-2 * lo
    gf = so.unflatten(g)
    for name in so.NAMES:
        a, b = gf[name].astype(np.float64), np.asarray(go[name], np.float64).reshape(-1)
        if name == "W1":  # padding channels carry no gradient
            assert not a.reshape(32, 27, 8)[:, :, 5:].any()
        assert rel(a, b) < 3e-2, name
        assert a @ b / (np.linalg.norm(a) * np.linalg.norm(b) + 1e-30) > 0.999, name


@pytest.mark.parametrize("n", [1, 77, 256])
def test_tcgen05_backward_matches_mma_sync(n):
    """The input gradients of the 32 -> 32 convolutions on tcgen05 (the
    forward convolution kernel with the mirrored, transposed weights and a
    ReLU-mask epilogue) against the mma.sync implicit GEMMs and the oracle:
    every parameter gradient, partial tiles included."""
    rng = np.random.default_rng(20 + n)
    flat = so.init_params(9)
    s = Surrogate(0, max_batch=256)
    s.set_params(flat)
    genomes = rng.integers(0, 5, (n, 216)).astype(np.uint8)
    targets = rng.normal(size=n).astype(np.float32)
    s.use_tcgen05(True)
    l_tc, g_tc = s.gradients(genomes, targets)
    s.use_tcgen05(False)
    l_ms, g_ms = s.gradients(genomes, targets)
    lo, _, go = so.Net(flat).loss_and_grads(genomes, targets)
    a, b = so.unflatten(g_tc), so.unflatten(g_ms)
    for name in so.NAMES:
        x, y = a[name].astype(np.float64), b[name].astype(np.float64)
        z = np.asarray(go[name], np.float64).reshape(-1)
        assert rel(x, y) < 3e-2, name
        assert rel(x, z) < 3e-2, name
        assert x @ z / (np.linalg.norm(x) * np.linalg.norm(z) + 1e-30) > 0.999, name


def test_gradients_are_deterministic():
    rng = np.random.default_rng(2)
    s = Surrogate(0, max_batch=128, seed=3)
    genomes = rng.integers(0, 5, (128, 216)).astype(np.uint8)
    targets = rng.normal(size=128).astype(np.float32)
    l1, g1 = s.gradients(genomes, targets)
    l2, g2 = s.gradients(genomes, targets)
    assert l1 == l2 and np.array_equal(g1.view(np.uint32), g2.view(np.uint32))
    p1 = s.predict(genomes)
    assert np.array_equal(p1.view(np.uint32), s.predict(genomes).view(np.uint32))


def test_training_fits_a_voxel_statistic():
    """A target the network can represent: the bone fraction of the lower
    half weighted by height, plus the muscle balance.  Adam on the device
    must bring the held-out rank correlation above 0.9."""
    rng = np.random.default_rng(4)

    def target(g):
        z = np.arange(216) // 36
        bone = ((g == 1) * (z < 3) * (3 - z)).sum(1) / 54.0
        mus = ((g == 3).sum(1) - (g == 4).sum(1)) / 216.0
        return (bone + 2 * mus).astype(np.float32)

    train = rng.integers(0, 5, (6000, 216)).astype(np.uint8)
    test = rng.integers(0, 5, (1000, 216)).astype(np.uint8)
    yt, ye = target(train), target(test)
    mu, sd = yt.mean(), yt.std()
    s = Surrogate(0, max_batch=256, seed=7)
    first = None
    for step in range(600):
        idx = rng.integers(0, len(train), 128)
        loss = s.train_step(train[idx], (yt[idx] - mu) / sd, lr=1e-3)
        first = loss if first is None else first
    assert loss < 0.3 * first
    from scipy.stats import spearmanr
    rho = spearmanr(s.predict(test), ye).correlation
    assert rho > 0.9, rho


def test_to_cells_layout():
    g = np.zeros((1, 216), np.uint8)
    g[0, 1 + 6 * 2 + 36 * 3] = 1  # x=1, y=2, z=3 is bone
    c = to_cells(g)
    from mercury_b200.materials import BONE
    assert c.shape == (1, 6, 6, 6) and c[0, 1, 2, 3] == BONE and (c != 0).sum() == 1
