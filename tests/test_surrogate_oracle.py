"""The surrogate's CPU oracle (oracle/surrogate.py): its backward against
finite differences in float64, its BF16 rounding against torch, and its
layout against the library's."""
import numpy as np
import pytest

from oracle import surrogate as so


def test_layout_matches_library():
    from mercury_b200.surrogate import Surrogate
    assert list(Surrogate.layout()) == so.layout()


def test_bf16_rounding_matches_torch():
    import torch
    rng = np.random.default_rng(0)
    a = (rng.normal(0, 1, 10000) * 10.0 ** rng.integers(-8, 8, 10000)).astype(np.float32)
    a[:4] = [0.0, -0.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8]  # ties to even
    ref = torch.from_numpy(a).to(torch.bfloat16).to(torch.float32).numpy()
    assert np.array_equal(so.bf16(a).view(np.uint32), ref.view(np.uint32))


def test_im2col_adjoint():
    rng = np.random.default_rng(1)
    a = rng.normal(size=(2, 6, 6, 6, 8))
    d = rng.normal(size=(2 * 216, 27 * 8))
    assert np.isclose((so.im2col(a) * d).sum(), (a * so.col2im(d, 8)).sum())


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(2)
    flat = so.init_params(3).astype(np.float64)
    genomes = rng.integers(0, 5, (3, 216))
    targets = rng.normal(size=3)
    net = so.Net(flat, exact=True)
    loss, _, g = net.loss_and_grads(genomes, targets)
    gflat = so.flatten(g, np.float64)
    off = so.layout()
    h = 1e-6
    for i, name in enumerate(so.NAMES):
        idx = rng.choice(so.SIZES[i], size=min(4, so.SIZES[i]), replace=False)
        if name == "W1":
            idx = [k for k in range(so.SIZES[i]) if k % 8 < 5][:4]
        for k in idx:
            p = flat.copy()
            p[off[i] + k] += h
            lp = so.Net(p, exact=True).loss_and_grads(genomes, targets)[0]
            p[off[i] + k] -= 2 * h
            lm = so.Net(p, exact=True).loss_and_grads(genomes, targets)[0]
            fd = (lp - lm) / (2 * h)
            assert abs(fd - gflat[off[i] + k]) <= 1e-5 * max(1.0, abs(fd)), (name, k, fd, gflat[off[i] + k])
