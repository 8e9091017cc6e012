"""The library's lattice builder (mb_voxel_build) against the reference's
VoxelRobot::Build outputs (tests/golden/ref_voxel_robots.npz)."""
import os

import numpy as np
import pytest

import mercury_b200 as mb
from mercury_b200 import robots


def test_voxel_build_matches_reference(golden_dir):
    g = np.load(os.path.join(golden_dir, "ref_voxel_robots.npz"))
    mo, so, go = g["mass_offsets"], g["spring_offsets"], g["grid_offsets"]
    for k in range(len(g["dims"])):
        nx, ny, nz = (int(v) for v in g["dims"][k])
        grid = g["grid"][go[k]:go[k + 1]].reshape(nz, ny, nx).transpose(2, 1, 0)
        e = robots.lattice_robot(grid, float(g["h"][k]))
        ms, ss = slice(mo[k], mo[k + 1]), slice(so[k], so[k + 1])
        assert np.array_equal(e.pos.view(np.uint32), g["pos"][ms].view(np.uint32)), k
        assert np.array_equal(e.mass_material, g["mass_material"][ms]), k
        assert np.array_equal(e.pairs, g["pairs"][ss]), k
        assert np.array_equal(e.mean_length.view(np.uint32), g["lbar"][ss].view(np.uint32)), k
        assert np.array_equal(e.spring_material, g["spring_material"][ss]), k


def test_baseline_com_and_length_match_reference(golden_dir):
    from oracle import core
    g = np.load(os.path.join(golden_dir, "ref_voxel_robots.npz"))
    mo, so = g["mass_offsets"], g["spring_offsets"]
    els = [mb.Element(g["pos"][mo[k]:mo[k + 1]], g["mass_material"][mo[k]:mo[k + 1]],
                      g["pairs"][so[k]:so[k + 1]], g["lbar"][so[k]:so[k + 1]],
                      g["spring_material"][so[k]:so[k + 1]]) for k in range(len(g["dims"]))]
    b = mb.pack(els)
    assert np.array_equal(core.com_reference(b, b.pos).view(np.uint32), g["com"].view(np.uint32))
    assert np.array_equal(mb.body_length(b), g["length"])


@pytest.mark.parametrize("side,springs", [(4, 468), (5, 1036), (6, 1940), (7, 3258), (8, 5068),
                                          (9, 7448), (10, 10476), (11, 14230)])
def test_full_lattice_spring_counts(side, springs):
    grid = np.full((side, side, side), 22, np.uint8)
    grid[side - 1, :, :] = grid[:, side - 1, :] = grid[:, :, side - 1] = 0
    e = robots.lattice_robot(grid)
    assert e.n_masses == side ** 3 and e.n_springs == springs
    assert np.count_nonzero(e.spring_material == 0) == 0


def test_default_reference_robot():
    # VoxelRobot::Initialize (VoxelRobot.cpp:352-381): 12^3 points, bone
    # inside, air on the upper faces: 1728 masses, 18,788 springs.
    grid = np.full((12, 12, 12), 22, np.uint8)
    grid[11, :, :] = grid[:, 11, :] = grid[:, :, 11] = 0
    e = robots.lattice_robot(grid, 1.0)
    assert (e.n_masses, e.n_springs) == (1728, 18788)


def test_population_shapes():
    small = robots.population("small")
    assert len(small) == 32 and all(e.n_masses == 125 for e in small)
    uneven = robots.population("uneven", 64)
    sides = {round(e.n_masses ** (1 / 3)) - 1 for e in uneven}
    assert sides <= set(range(3, 9)) and len(sides) >= 4
    assert all(e.n_springs <= 7448 for e in uneven)


def test_builder_rejects_bad_input():
    with pytest.raises(mb.MercuryError):
        robots.lattice_robot(np.full((2, 2, 2), 99, np.uint8))


def test_nn_robots_shape():
    """Point-cloud robots: masses in the ellipsoid, lowest on z = 0, 25-NN
    springs deduplicated (each pair once, lower index first), mean length =
    initial distance, composite material of the two masses."""
    from mercury_b200.materials import composite_id
    for e in robots.population("nn", 3, mass=0.1):
        assert 500 <= e.n_masses <= 2000
        p = e.pos.astype(np.float64)
        assert p[:, 2].min() == 0.0
        assert ((p[:, 0] / 0.3) ** 2 + (p[:, 1] / 0.2) ** 2 <= 1.0 + 1e-5).all()
        assert (e.pairs[:, 0] < e.pairs[:, 1]).all()
        assert len({tuple(x) for x in e.pairs}) == e.n_springs
        assert e.n_springs >= 25 * e.n_masses // 2
        d = np.linalg.norm(e.pos[e.pairs[:, 0]] - e.pos[e.pairs[:, 1]], axis=1)
        assert np.allclose(d, e.mean_length, rtol=1e-6)
        exp = [composite_id(int(e.mass_material[u]), int(e.mass_material[v])) for u, v in e.pairs[:50]]
        assert list(e.spring_material[:50]) == exp
        assert len(np.unique(e.mass_material)) >= 2
        assert np.all(e.mass == np.float32(0.1))
