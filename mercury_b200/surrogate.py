"""Fitness surrogate: a 3-D convolutional network over 6x6x6 voxel genomes,
trained on the device by the library's BF16 tensor-core kernels
(mb_surrogate_*, mercury_b200/csrc/mb_surrogate.cu).

Genomes are (n, 216) arrays of classes 0 air, 1 bone, 2 tissue, 3 muscle a,
4 muscle b, voxel v = x + 6y + 36z.  to_cells() turns them into the cell
grids the simulator builds robots from (robots.FIVE material ids).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .robots import FIVE

N_VOX = 216


def to_cells(genomes: np.ndarray) -> np.ndarray:
    """(n, 216) classes -> (n, 6, 6, 6) material ids indexed [robot, x, y, z]."""
    g = np.asarray(genomes, np.uint8).reshape(-1, 6, 6, 6)  # [n, z, y, x]
    return FIVE[g].transpose(0, 3, 2, 1)


class Surrogate:
    def __init__(self, device: int = 0, max_batch: int = 1024, seed: int = 0):
        s = ctypes.c_void_p()
        st = _lib.LIB.mb_surrogate_create(device, max_batch, seed, ctypes.byref(s))
        if st != _lib.MB_OK:
            raise _lib.MercuryError(st, "mb_surrogate_create failed")
        self._s = s
        self.max_batch = max_batch
        self.n_params = int(_lib.LIB.mb_surrogate_param_count())

    def __del__(self):
        s = getattr(self, "_s", None)
        lib = getattr(_lib, "LIB", None)
        if s and lib is not None:
            lib.mb_surrogate_destroy(s)
            self._s = None

    def _check(self, st):
        if st != _lib.MB_OK:
            raise _lib.MercuryError(st, _lib.LIB.mb_surrogate_last_error(self._s).decode())

    @staticmethod
    def layout() -> np.ndarray:
        off = np.zeros(13, np.uint32)
        _lib.LIB.mb_surrogate_layout(_lib.ptr(off))
        return off

    def get_params(self) -> np.ndarray:
        p = np.empty(self.n_params, np.float32)
        self._check(_lib.LIB.mb_surrogate_get_params(self._s, _lib.ptr(p)))
        return p

    def set_params(self, params: np.ndarray) -> None:
        p = np.ascontiguousarray(params, np.float32)
        assert p.size == self.n_params
        self._check(_lib.LIB.mb_surrogate_set_params(self._s, _lib.ptr(p)))

    @staticmethod
    def _g(genomes):
        g = np.ascontiguousarray(genomes, np.uint8)
        assert g.ndim == 2 and g.shape[1] == N_VOX
        return g

    def predict(self, genomes: np.ndarray) -> np.ndarray:
        g = self._g(genomes)
        out = np.empty(len(g), np.float32)
        self._check(_lib.LIB.mb_surrogate_predict(self._s, _lib.ptr(g), len(g), _lib.ptr(out)))
        return out

    def gradients(self, genomes: np.ndarray, targets: np.ndarray):
        g = self._g(genomes)
        t = np.ascontiguousarray(targets, np.float32)
        grads = np.empty(self.n_params, np.float32)
        loss = np.zeros(1, np.float32)
        self._check(_lib.LIB.mb_surrogate_gradients(self._s, _lib.ptr(g), _lib.ptr(t), len(g), _lib.ptr(grads),
                                                    _lib.ptr(loss)))
        return float(loss[0]), grads

    def use_tcgen05(self, on: bool = True) -> None:
        """Forward products on tcgen05 (default) or on the mma.sync kernel."""
        self._check(_lib.LIB.mb_surrogate_use_tcgen05(self._s, int(bool(on))))

    def set_weight_decay(self, wd: float) -> None:
        """Decoupled weight decay of the Adam steps (AdamW)."""
        self._check(_lib.LIB.mb_surrogate_set_weight_decay(self._s, float(wd)))

    def train_step(self, genomes: np.ndarray, targets: np.ndarray, lr: float = 1e-3) -> float:
        g = self._g(genomes)
        t = np.ascontiguousarray(targets, np.float32)
        loss = np.zeros(1, np.float32)
        self._check(_lib.LIB.mb_surrogate_train_step(self._s, _lib.ptr(g), _lib.ptr(t), len(g), float(lr),
                                                     _lib.ptr(loss)))
        return float(loss[0])
