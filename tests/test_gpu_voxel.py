"""Voxel robots built on the device (mb_set_voxel_population) against the
host builder (mb_voxel_build, pinned to the reference's VoxelRobot::Build)
followed by mb_set_elements: same materials after the strip, same springs,
and the same bits after stepping."""
import numpy as np
import pytest

import mercury_b200 as mb
from mercury_b200 import robots
from mercury_b200 import simulator as S
from mercury_b200.materials import BONE, TISSUE, ADDUCTOR_MUSCLE0
from oracle import core

pytestmark = pytest.mark.gpu

ENV_KEYS = ("g", "floor_stiffness", "friction_static", "friction_kinetic", "drag", "damping")


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def genomes(n, side=6, seed=5):
    rng = np.random.default_rng(seed)
    cells = np.stack([robots.random_cells(side, rng) for _ in range(n)])
    cells[0] = 0                                   # all air
    cells[1] = 0
    cells[1][2, 3, 1] = BONE                       # one voxel
    cells[2] = 0
    cells[2][0, 0, 0] = BONE
    cells[2][3:, 3:, 3:] = TISSUE                  # two pieces: the larger stays
    cells[3] = BONE                                # full
    cells[4] = 0
    cells[4][0:2, 0:2, 0] = TISSUE
    cells[4][4:6, 4:6, 5] = ADDUCTOR_MUSCLE0       # two equal pieces: the first stays
    return cells


def host_batch(cells, h, mass):
    return mb.pack([robots.voxel_robot(c, h, mass) for c in cells])


def make_sim(mode):
    sim = mb.Simulator(0)
    if mode:
        sim.set_materials(mb.materials.force_table())
        sim.set_mode(mode)
        sim.set_environment(**S.LAND)
    return sim


@pytest.mark.parametrize("mode", [0, 1], ids=["xpbd", "land"])
def test_device_build_matches_host_build(mode):
    cells = genomes(40)
    h, mass = 0.1, (0.1 if mode else 1.0)
    ref = host_batch(cells, h, mass)
    a, b = make_sim(mode), make_sim(mode)
    for sim in (a, b):
        sim.setTimeStep(1e-4 if mode else 1e-3)
    a.set_voxel_population(cells, h, mass)
    b.set_batch(ref)
    pa, ma, la = a.collect_springs()
    assert np.array_equal(pa, ref.pairs)
    assert np.array_equal(ma, ref.spring_material)
    assert np.array_equal(bits(la), bits(ref.lbar))
    assert np.array_equal(a.batch.mass_material, ref.mass_material)
    for sim in (a, b):
        sim.run_steps(400, True)
    xa, va, sa = a.collect_arrays()
    xb, vb, sb = b.collect_arrays()
    assert np.array_equal(bits(xa), bits(xb)) and np.array_equal(bits(va), bits(vb))
    assert np.array_equal(bits(sa), bits(sb))
    # and the oracle
    p, v = ref.pos.copy(), ref.vel.copy()
    s = np.zeros(ref.n_springs, np.float32)
    if mode:
        core.force_run(mode, ref, p, v, s, mb.materials.force_table(), [S.LAND[k] for k in ENV_KEYS], 1e-4,
                       0.0, 400, True)
    else:
        core.xpbd_run(ref, p, v, s, mb.material_table(), 1e-3, 0.0, 400, True)
    assert np.array_equal(bits(xa), bits(p)) and np.array_equal(bits(sa), bits(s))
    com = a.CentreOfMass()
    assert np.array_equal(bits(com), bits(core.com_device(ref, p)))


def test_repeated_uploads_reuse_the_template():
    sim = make_sim(1)
    sim.setTimeStep(1e-4)
    for seed in (11, 12, 13):
        cells = genomes(24, seed=seed)
        sim.set_voxel_population(cells, 0.1, 0.1)
        sim.run_steps(200, False)
        ref = host_batch(cells, 0.1, 0.1)
        p, v = ref.pos.copy(), ref.vel.copy()
        core.force_run(1, ref, p, v, np.zeros(ref.n_springs, np.float32), mb.materials.force_table(),
                       [S.LAND[k] for k in ENV_KEYS], 1e-4, core.advance_clock(0.0, 1e-4, 200 * (seed - 11)),
                       200, False)
        x, _, _ = sim.collect_arrays()
        assert np.array_equal(bits(x), bits(p))


def test_other_grid_shapes_and_devo_after_device_build():
    cells = np.stack([robots.random_cells(4, np.random.default_rng(i)) for i in range(16)])
    cells = np.concatenate([cells, cells[:, :3]], axis=1)  # 7 x 4 x 4 cells
    ref = host_batch(cells, 0.1, 1.0)
    sim = mb.Simulator(0)
    sim.setTimeStep(1e-3)
    sim.set_voxel_population(cells, 0.1, 1.0)
    sim.run_steps(100, True)
    n = sim.devo(8, 3)
    p, v = ref.pos.copy(), ref.vel.copy()
    s = np.zeros(ref.n_springs, np.float32)
    core.xpbd_run(ref, p, v, s, mb.material_table(), 1e-3, 0.0, 100, True)
    pairs, mat, lbar, recs = core.devo(ref, p, s, mb.material_table(), core.advance_clock(0.0, 1e-3, 100), 8, 3)
    assert n == len(recs)
    gp, gm, gl = sim.collect_springs()
    assert np.array_equal(gp, pairs) and np.array_equal(gm, mat) and np.array_equal(bits(gl), bits(lbar))


def test_bad_material_is_rejected():
    cells = genomes(8)
    cells[6, 0, 0, 0] = 40
    sim = mb.Simulator(0)
    with pytest.raises(mb.MercuryError):
        sim.set_voxel_population(cells, 0.1, 1.0)
