"""Generates velocity_midpoints.npz: float32 displacements d for which the
reference step's velocity (float)(0.99 * (double)d / (double)dt)
(sim_kernel.cu:265-267) lands within 4 double units in the last place of a
float rounding midpoint -- the inputs on which a division-free evaluation
must fall back to the division.  Exhaustive over the significands of the
binades 2^-20 .. 2^1, both signs, for a few time steps.

    python tests/golden/make_velocity_midpoints.py
"""
import os

import numpy as np

DTS = (1e-3, 1e-2)
EXPONENTS = range(-20, 2)
TOL = 4


def near_midpoints(dt: np.float32) -> np.ndarray:
    out = []
    m = np.arange(1 << 23, dtype=np.uint32)
    for e in EXPONENTS:
        f = ((np.uint32(e + 127) << np.uint32(23)) | m).view(np.float32)
        for sgn in (np.float32(1), np.float32(-1)):
            ff = (f * sgn).astype(np.float32)
            z = (np.float64(0.99) * ff.astype(np.float64)) / np.float64(dt)
            low = (z.view(np.uint64) & np.uint64(0x1FFFFFFF)).astype(np.int64)
            out.append(ff[np.abs(low - (1 << 28)) <= TOL])
    return np.concatenate(out)


def main():
    arrays = {}
    for i, dt in enumerate(DTS):
        arrays[f"dt{i}"] = np.array([dt], np.float32)
        arrays[f"d{i}"] = near_midpoints(np.float32(dt))
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "velocity_midpoints.npz")
    np.savez_compressed(path, **arrays)
    print(path, {k: v.shape for k, v in arrays.items()})


if __name__ == "__main__":
    main()
