"""One run of each topology kernel, for profilers.

    python -m mercury_b200.profile_builders

  1. Devo on 512 default voxel robots (1,728 masses, 18,788 springs; 128
     springs per robot) after 100 stress-tracked steps: devo_kernel,
     apply_kernel (2 launches), rebuild_kernel;
  2. 4096 random 6x6x6 voxel genomes built on the device, twice (the first
     call plans the packing): build_kernel, compact_kernel, rebuild_kernel;
  3. k = 25 nearest-neighbour springs of 64 point-cloud robots (500-2000
     masses): select_kernel, mark_kernel, count_kernel, emit_kernel.
Prints the host wall time of each.  With ncu, select kernels with -k, e.g.
-k regex:"devo_kernel|rebuild_kernel|build_kernel|select_kernel".
"""
from __future__ import annotations

import time

import numpy as np

import mercury_b200 as mb
from mercury_b200 import evolve, robots
from mercury_b200.surrogate import to_cells


def main():
    grid = np.full((12, 12, 12), 22, np.uint8)
    grid[11, :, :] = grid[:, 11, :] = grid[:, :, 11] = 0
    b = mb.pack([robots.lattice_robot(grid, 1.0)] * 512)
    sim = mb.Simulator(0)
    sim.setTimeStep(1e-4)
    sim.set_batch(b)
    sim.run_steps(100, True)
    sim.synchronize()
    t0 = time.perf_counter()
    sim.devo(128, 0)
    print(f"devo: {(time.perf_counter() - t0) * 1e3:.2f} ms, phases {sim.devo_profile()}")

    cells = to_cells(evolve.random_genomes(np.random.default_rng(1), 4096))
    vs = mb.Simulator(0)
    vs.set_voxel_population(cells, 0.1, 0.1)
    t0 = time.perf_counter()
    vs.set_voxel_population(cells, 0.1, 0.1)
    print(f"voxel build of 4096: {(time.perf_counter() - t0) * 1e3:.2f} ms")

    pts, mats = [], []
    for r in range(64):
        g = np.random.default_rng(2000 + r)
        p, m = robots.nn_points(g, int(g.integers(500, 2001)))
        pts.append(p)
        mats.append(m)
    t0 = time.perf_counter()
    so, _, _, _ = robots.knn_springs(pts, mats)
    print(f"knn springs of 64 robots: {(time.perf_counter() - t0) * 1e3:.2f} ms, {int(so[-1])} springs")


if __name__ == "__main__":
    main()
