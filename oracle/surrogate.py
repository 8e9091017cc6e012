"""CPU ORACLE of the fitness surrogate -- test infrastructure, never shipped.

A numpy restatement of the network the library's surrogate kernels compute
(mercury_b200/csrc/mb_surrogate.cu): forward, mean-squared-error loss and
backward, with the same BF16 rounding points (weights, activations after
ReLU, the gradients fed to GEMMs) and FP32 elsewhere, so the CUDA results
agree with it up to the order of FP32 accumulation.  `exact=True` drops every
rounding and works in float64, for finite-difference checks of the backward
itself.  The surrogate has no counterpart in the reference.

Layout: genomes (n, 216) of classes 0..4, voxel v = x + 6y + 36z; tensors
channels-last (n, 6, 6, 6, C) indexed [n, z, y, x, c]; conv weights
[out][27 * in] with k = offset * in + c and offset = (dx+1) + 3(dy+1) + 9(dz+1);
W4 [128][6912] over voxel * 32 + channel.
"""
from __future__ import annotations

import numpy as np

SIZES = [32 * 27 * 8, 32, 32 * 27 * 32, 32, 32 * 27 * 32, 32, 128 * 6912, 128, 128 * 128, 128, 128, 1]
NAMES = ["W1", "b1", "W2", "b2", "W3", "b3", "W4", "b4", "W5", "b5", "W6", "b6"]


def layout():
    off, o = [], 0
    for s in SIZES:
        off.append(o)
        o += (s + 7) // 8 * 8
    off.append(o)
    return off


def unflatten(flat):
    off = layout()
    return {n: flat[off[i]:off[i] + SIZES[i]] for i, n in enumerate(NAMES)}


def flatten(params, dtype=np.float32):
    off = layout()
    out = np.zeros(off[-1], dtype)
    for i, n in enumerate(NAMES):
        out[off[i]:off[i] + SIZES[i]] = np.asarray(params[n]).reshape(-1)
    return out


def bf16(a):
    """Round-to-nearest-even to bfloat16, returned as float32."""
    a = np.ascontiguousarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32)


def offsets():
    return [((o % 3) - 1, ((o // 3) % 3) - 1, (o // 9) - 1) for o in range(27)]


def im2col(a):
    """(n, 6, 6, 6, C) -> (n * 216, 27 * C), zero outside the grid."""
    n, C = a.shape[0], a.shape[-1]
    p = np.zeros((n, 8, 8, 8, C), a.dtype)
    p[:, 1:7, 1:7, 1:7] = a
    cols = [p[:, 1 + dz:7 + dz, 1 + dy:7 + dy, 1 + dx:7 + dx] for dx, dy, dz in offsets()]
    return np.stack(cols, axis=4).reshape(n * 216, 27 * C)


def col2im(dcol, C):
    """Adjoint of im2col: (n * 216, 27 * C) -> (n, 6, 6, 6, C)."""
    n = dcol.shape[0] // 216
    d = dcol.reshape(n, 6, 6, 6, 27, C)
    p = np.zeros((n, 8, 8, 8, C), dcol.dtype)
    for o, (dx, dy, dz) in enumerate(offsets()):
        p[:, 1 + dz:7 + dz, 1 + dy:7 + dy, 1 + dx:7 + dx] += d[:, :, :, :, o]
    return p[:, 1:7, 1:7, 1:7]


def onehot(genomes):
    g = np.asarray(genomes, np.int64).reshape(-1, 6, 6, 6)
    x = np.zeros(g.shape + (8,), np.float32)
    for c in range(5):
        x[..., c] = g == c
    return x


class Net:
    def __init__(self, flat, exact=False):
        self.exact = exact
        self.dt = np.float64 if exact else np.float32
        p = unflatten(np.asarray(flat, np.float64 if exact else np.float32))
        r = (lambda a: a.astype(np.float64)) if exact else bf16
        self.W = {k: r(p[k]).astype(self.dt) for k in ("W1", "W2", "W3", "W4", "W5", "W6")}
        self.b = {k: p[k].astype(self.dt) for k in ("b1", "b2", "b3", "b4", "b5", "b6")}

    def _r(self, a):
        return a.astype(np.float64) if self.exact else bf16(a)

    def forward(self, genomes):
        n = len(genomes)
        W, b = self.W, self.b
        x0 = onehot(genomes).astype(self.dt)
        cache = {"x0": x0}
        a = x0
        for i, (w, bb, cin) in enumerate((("W1", "b1", 8), ("W2", "b2", 32), ("W3", "b3", 32)), 1):
            col = im2col(a)
            z = col @ W[w].reshape(32, 27 * cin).T + b[bb]
            a = self._r(np.maximum(z, 0)).reshape(n, 6, 6, 6, 32).astype(self.dt)
            cache[f"col{i}"], cache[f"a{i}"] = col, a
        a3 = a.reshape(n, 6912)
        h1 = self._r(np.maximum(a3 @ W["W4"].reshape(128, 6912).T + b["b4"], 0)).astype(self.dt)
        h2 = self._r(np.maximum(h1 @ W["W5"].reshape(128, 128).T + b["b5"], 0)).astype(self.dt)
        y = h2 @ W["W6"] + b["b6"][0]
        cache.update(a3f=a3, h1=h1, h2=h2)
        return y, cache

    def loss_and_grads(self, genomes, targets):
        n = len(genomes)
        W = self.W
        y, c = self.forward(genomes)
        t = np.asarray(targets, self.dt)
        e = y - t
        loss = float(np.mean(e * e))
        dy = 2.0 * e / n
        g = {"W6": dy @ c["h2"], "b6": np.array([dy.sum()])}
        dz2 = self._r(np.outer(dy, W["W6"]) * (c["h2"] > 0)).astype(self.dt)
        g["W5"] = dz2.T @ c["h1"]
        g["b5"] = dz2.sum(0)
        dz1 = self._r((dz2 @ W["W5"].reshape(128, 128)) * (c["h1"] > 0)).astype(self.dt)
        g["W4"] = dz1.T @ c["a3f"]
        g["b4"] = dz1.sum(0)
        dz = self._r((dz1 @ W["W4"].reshape(128, 6912)) * (c["a3f"] > 0)).astype(self.dt)
        dz = dz.reshape(n * 216, 32)
        for i, cin in ((3, 32), (2, 32), (1, 8)):
            g[f"W{i}"] = dz.T @ c[f"col{i}"]
            g[f"b{i}"] = dz.sum(0)
            if i > 1:
                da = col2im(dz @ W[f"W{i}"].reshape(32, 27 * cin), cin)
                prev = c[f"a{i - 1}"]
                dz = self._r(da * (prev > 0)).astype(self.dt).reshape(n * 216, cin)
        return loss, y, g


def init_params(seed: int = 0):
    """A random parameter set (He-normal weights, small random biases) for
    tests; padding channels of W1 zero."""
    rng = np.random.default_rng(seed)
    p = {}
    fan = {"W1": 27 * 5, "W2": 27 * 32, "W3": 27 * 32, "W4": 6912, "W5": 128, "W6": 128}
    for i, n in enumerate(NAMES):
        if n in fan:
            p[n] = rng.normal(0, np.sqrt(2.0 / fan[n]), SIZES[i]).astype(np.float32)
        else:
            p[n] = rng.normal(0, 0.05, SIZES[i]).astype(np.float32)
    w1 = p["W1"].reshape(32, 27, 8)
    w1[:, :, 5:] = 0
    return flatten(p)
