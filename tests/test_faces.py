"""Face drag of the water mode on the CPU: the surface builders, the face
law of the oracle against a float64 restatement of the reference's formula
(sim_kernel.cu:96-121), and the packer's handling of faces."""
import numpy as np
import pytest

import mercury_b200 as mb
from mercury_b200 import robots
from mercury_b200 import simulator as S
from oracle import core

ENV7 = ("g", "floor_stiffness", "friction_static", "friction_kinetic", "drag", "damping", "face_drag")


def _edges(tri):
    e = np.concatenate([tri[:, [0, 1]], tri[:, [1, 2]], tri[:, [2, 0]]]).astype(np.int64)
    e.sort(axis=1)
    _, counts = np.unique(e, axis=0, return_counts=True)
    return counts


def test_voxel_faces_of_a_full_cube():
    s = 3
    tri = robots.voxel_faces(np.full((s, s, s), robots.BONE, np.uint8))
    assert tri.shape == (6 * s * s * 2, 3)
    # corners on the cube's boundary, every edge in exactly two triangles
    n = s + 1
    idx = tri.astype(np.int64).reshape(-1)
    x, y, z = idx % n, (idx // n) % n, idx // (n * n)
    assert np.all((x == 0) | (x == s) | (y == 0) | (y == s) | (z == 0) | (z == s))
    assert np.all(_edges(tri) == 2)


def test_voxel_faces_close_every_random_robot():
    for r in range(8):
        rng = np.random.default_rng(100 + r)
        cells = robots.random_cells(4, rng)
        tri = robots.voxel_faces(cells)
        occ = cells != robots.AIR
        # one square (two triangles) per occupied-cell face with an empty neighbour
        pad = np.pad(occ, 1)
        exposed = sum(int((occ & ~np.roll(pad, d, a)[1:-1, 1:-1, 1:-1]).sum())
                      for a in range(3) for d in (1, -1))
        assert len(tri) == 2 * exposed
        assert np.all(_edges(tri) % 2 == 0)  # closed (edges of touching cubes: four)
        assert len(np.unique(tri, axis=0)) == len(tri)
        assert np.all((tri[:, 0] != tri[:, 1]) & (tri[:, 1] != tri[:, 2]) & (tri[:, 0] != tri[:, 2]))


def test_hull_faces_are_a_closed_surface():
    rng = np.random.default_rng(7)
    e = robots.nn_robot(rng, 400)
    tri = robots.hull_faces(e.pos)
    assert np.all(_edges(tri) == 2)
    v = len(np.unique(tri))
    edges = len(_edges(tri))
    assert v - edges + len(tri) == 2  # Euler characteristic of a sphere


def _face_law_f64(x, v, rho):
    """-rho/2 A ((v.n) v + 0.2 |v|^2 n) / 3 with n turned towards v
    (sim_kernel.cu:104-112), in float64."""
    x = x.astype(np.float64)
    vm = v.astype(np.float64).mean(0)
    N = np.cross(x[1] - x[0], x[2] - x[0])
    A = np.linalg.norm(N)
    n = N / (A + 1e-12)
    if not np.dot(n, vm) > 0:
        n = -n
    return -0.5 * rho * A * (np.dot(vm, n) * vm + 0.2 * np.dot(vm, vm) * n) / 3.0


def test_face_law_matches_the_reference_formula():
    rng = np.random.default_rng(3)
    rho = 1000.0
    coef = np.float32(-rho / 6.0)
    for _ in range(500):
        x = rng.normal(0, 0.1, (3, 3)).astype(np.float32)
        v = rng.normal(0, 1.0, (3, 3)).astype(np.float32)
        f = core.face_force(x, v, coef)
        ref = _face_law_f64(x, v, rho)
        assert np.linalg.norm(f - ref) <= 1e-5 * np.linalg.norm(ref) + 1e-30
        # drag opposes the mean motion
        assert np.dot(f.astype(np.float64), v.astype(np.float64).mean(0)) <= 0.0
        # the orientation does not matter (up to the order of the velocity sum)
        g = core.face_force(x[[0, 2, 1]], v[[0, 2, 1]], coef)
        assert np.allclose(f, g, rtol=1e-5, atol=1e-6 * np.abs(f).max())
    assert not np.any(core.face_force(rng.normal(0, 0.1, (3, 3)), np.zeros((3, 3)), coef))


def _cube(vel):
    cells = np.full((2, 2, 2), robots.BONE, np.uint8)
    e = robots.voxel_robot(cells, mass=0.1)
    e.faces = robots.voxel_faces(cells)
    e.vel[:] = vel
    return mb.pack([e])


def _run_water(b, env, steps=1000):
    p, v = b.pos.copy(), b.vel.copy()
    s = np.zeros(b.n_springs, np.float32)
    core.force_run(2, b, p, v, s, mb.materials.force_table(), [env[k] for k in ENV7], np.float32(1e-4),
                   0.0, steps, True)
    return p, v, s


def test_face_drag_slows_a_cube_along_its_motion():
    # a direction oblique to every face: for a face parallel to the motion
    # (v.n = 0) the law's normal, and so its lift, has no preferred side
    v0 = np.array([0.3, 0.2, 1.0], np.float32)
    b = _cube(v0)
    _, v_free, _ = _run_water(b, dict(S.WATER_FACES, face_drag=0.0))
    _, v_drag, _ = _run_water(b, S.WATER_FACES)
    m_free, m_drag = v_free[:, :3].mean(0), v_drag[:, :3].mean(0)
    assert np.linalg.norm(m_drag) < 0.5 * np.linalg.norm(m_free)
    cos = np.dot(m_drag, v0) / (np.linalg.norm(m_drag) * np.linalg.norm(v0))
    assert cos > 0.95


def test_zero_face_drag_changes_nothing():
    b = _cube([0.3, -0.2, 1.0])
    env = dict(S.WATER, face_drag=0.0)
    p0, v0, s0 = _run_water(mb.Batch(**{k: getattr(b, k) for k in (
        "mass_offsets", "pos", "vel", "mass_material", "spring_offsets", "pairs", "spring_material", "lbar")}),
        env)
    p1, v1, s1 = _run_water(b, env)
    for a, c in ((p0, p1), (v0, v1), (s0, s1)):
        assert np.array_equal(a.view(np.uint32), c.view(np.uint32))


def test_plan_counts_the_faces_shared_memory():
    b = robots.population_batch("uneven", 64, faces=True)
    b0 = robots.population_batch("uneven", 64)
    p, p0 = mb.plan(b), mb.plan(b0)
    assert p["active_springs"] == p0["active_springs"] and p["streamed"] == p0["streamed"] == 0
    assert p["max_smem_bytes"] > p0["max_smem_bytes"]
    assert p["max_smem_bytes"] <= 232448


def test_bad_faces_are_rejected():
    e = robots.voxel_robot(np.full((2, 2, 2), robots.BONE, np.uint8))
    e.faces = np.array([[0, 1, 27]], np.uint16)  # 27 masses: corner out of range
    with pytest.raises(mb._lib.MercuryError) as ex:
        mb.plan(mb.pack([e]))
    assert ex.value.status == 1  # MB_ERR_ARGUMENT
    # more than 255 faces on one mass
    e.faces = np.array([[0, 1 + (i % 26), 1 + ((i + 1) % 26)] for i in range(256)], np.uint16)
    with pytest.raises(mb._lib.MercuryError) as ex:
        mb.plan(mb.pack([e]))
    assert ex.value.status == 3  # MB_ERR_CAPACITY
    # faces with two equal corners are skipped, not rejected
    e.faces = np.array([[0, 0, 1], [2, 3, 3]], np.uint16)
    mb.plan(mb.pack([e]))
