"""Seeded synthetic robot populations.

Voxel robots are built by the library's lattice builder (mb_voxel_build, the
topology of the reference's VoxelRobot::Build, VoxelRobot.cpp:310-331).  A
robot of `side` cells per axis has (side+1)^3 grid points; grid point p
carries the material of the cell whose lowest corner is p, so points on the
upper faces carry air (as VoxelRobot::Initialize does, VoxelRobot.cpp:375-378).

Populations (cell size 0.1 m, one seed per robot = 1000*population + robot,
numpy PCG64):
  small      32 robots of 4x4x4 cells, cells iid {air .3, bone .175,
             tissue .175, muscle_a .175, muscle_b .175}
  uneven     512 robots, side uniform in 3..8, same materials
  streamed   64 robots of 10x10x10 cells, all occupied, iid over
             {bone, tissue, muscle_a, muscle_b}
  nn         256 point-cloud robots (nn_robot): 500..2000 masses uniform in
             an ellipsoid with semi-axes 0.3/0.2/0.15 m, 25-nearest-neighbour
             springs (deduplicated), materials from a random tanh MLP
             3 -> 25 -> 25 -> 4 over the position (argmax over bone, tissue,
             muscle_a, muscle_b)
Surfaces (faces=True): voxel robots get the exposed faces of their occupied
cells, two triangles per square (voxel_faces); point clouds get their
convex hull (hull_faces), standing in for the alpha-shape surface the
reference's NNRobot builds with CGAL (NNRobot.cpp:236-311, delaunay.cpp).
For the reference step, muscle_a is adductor_muscle0 (phase 0) and muscle_b
abductor_muscle0 (phase pi), material.h:112, 122.  The force-based
configurations give every mass 0.1 kg (population(..., mass=0.1)) and use
materials.force_table().
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .element import Element, pack
from .materials import ABDUCTOR_MUSCLE0, ADDUCTOR_MUSCLE0, AIR, BONE, TISSUE

CELL = 0.1
FIVE = np.array([AIR, BONE, TISSUE, ADDUCTOR_MUSCLE0, ABDUCTOR_MUSCLE0], np.uint8)
FIVE_P = np.array([0.3, 0.175, 0.175, 0.175, 0.175])
FOUR = np.array([BONE, TISSUE, ADDUCTOR_MUSCLE0, ABDUCTOR_MUSCLE0], np.uint8)


def voxel_robot(cells: np.ndarray, h: float = CELL, mass: float = 1.0) -> Element:
    """Robot from a grid of cells (base material ids indexed [x, y, z]); an
    extra air layer of grid points closes the upper faces."""
    cells = np.asarray(cells, np.uint8)
    sx, sy, sz = cells.shape
    nx, ny, nz = sx + 1, sy + 1, sz + 1
    grid = np.zeros((nx, ny, nz), np.uint8)
    grid[:sx, :sy, :sz] = cells
    return lattice_robot(grid, h, mass)


def lattice_robot(grid: np.ndarray, h: float = CELL, mass: float = 1.0) -> Element:
    """Robot from a grid of points indexed [x, y, z] (mb_voxel_build)."""
    grid = np.asarray(grid, np.uint8)
    nx, ny, nz = grid.shape
    mats = np.ascontiguousarray(grid.transpose(2, 1, 0).reshape(-1))  # x fastest
    n = nx * ny * nz
    pos = np.zeros(3 * n, np.float32)
    mm = np.zeros(n, np.uint8)
    pairs = np.zeros(2 * 13 * n, np.uint16)
    lbar = np.zeros(13 * n, np.float32)
    sm = np.zeros(13 * n, np.uint8)
    nm, ns = ctypes.c_int(), ctypes.c_int()
    st = _lib.LIB.mb_voxel_build(nx, ny, nz, h, _lib.ptr(mats), ctypes.byref(nm), ctypes.byref(ns),
                                 _lib.ptr(pos), _lib.ptr(mm), _lib.ptr(pairs), _lib.ptr(lbar),
                                 _lib.ptr(sm))
    _lib.check(st)
    s = ns.value
    return Element(pos.reshape(n, 3), mm, pairs[: 2 * s].reshape(s, 2), lbar[:s], sm[:s],
                   mass=np.full(n, mass, np.float32))


def voxel_faces(cells: np.ndarray) -> np.ndarray:
    """Surface of a voxel robot (voxel_robot(cells)): every face of an
    occupied (non-air) cell whose neighbour across it is air or outside the
    grid, as two triangles (p00, p10, p11), (p00, p11, p01) of its corner
    grid points.  Order: axis x, y, z; the lower side, then the upper; cells
    in [x, y, z] order.  Returns (F, 3) uint16 grid-point indices (x
    fastest)."""
    occ = np.asarray(cells) != AIR
    sx, sy, sz = occ.shape
    nx, ny = sx + 1, sy + 1
    pad = np.pad(occ, 1)
    out = []
    for axis in range(3):
        u, v = [a for a in range(3) if a != axis]
        eu, ev = np.eye(3, dtype=np.int64)[u], np.eye(3, dtype=np.int64)[v]
        for side in (0, 1):
            sl = [slice(1, 1 + sx), slice(1, 1 + sy), slice(1, 1 + sz)]
            d = 1 if side else -1
            sl[axis] = slice(1 + d, 1 + d + occ.shape[axis])
            cell = np.argwhere(occ & ~pad[tuple(sl)])
            base = cell.copy()
            base[:, axis] += side
            corners = [base, base + eu, base + eu + ev, base + ev]
            p00, p10, p11, p01 = [c[:, 0] + nx * (c[:, 1] + ny * c[:, 2]) for c in corners]
            tri = np.stack([np.stack([p00, p10, p11], 1), np.stack([p00, p11, p01], 1)], 1).reshape(-1, 3)
            out.append(tri)
    return np.concatenate(out).astype(np.uint16) if out else np.zeros((0, 3), np.uint16)


def hull_faces(points: np.ndarray) -> np.ndarray:
    """Convex hull triangles of a point cloud (qhull through scipy), each
    with ascending corners, sorted.  Returns (F, 3) uint16."""
    from scipy.spatial import ConvexHull
    t = np.sort(ConvexHull(np.asarray(points, np.float64)).simplices, axis=1)
    t = t[np.lexsort((t[:, 2], t[:, 1], t[:, 0]))]
    return t.astype(np.uint16)


def random_cells(side: int, rng: np.random.Generator, choices=FIVE, p=FIVE_P) -> np.ndarray:
    return choices[rng.choice(len(choices), size=(side, side, side), p=p)]


def nn_points(rng: np.random.Generator, n_masses: int, axes=(0.3, 0.2, 0.15), hidden=(25, 25)):
    """Masses of a point-cloud robot: uniform in an ellipsoid, lowest on
    z = 0 (float32 positions); materials from a random-init tanh MLP over
    (x, y, z) in ellipsoid units, argmax over bone, tissue, muscle_a,
    muscle_b (unit-variance weights, small biases)."""
    pts = []
    a = np.asarray(axes, np.float64)
    while sum(len(p) for p in pts) < n_masses:
        c = rng.uniform(-1.0, 1.0, size=(2 * n_masses, 3))
        pts.append(c[(c * c).sum(1) <= 1.0] * a)
    p = np.concatenate(pts)[:n_masses]
    p[:, 2] -= p[:, 2].min()  # lowest mass on z = 0
    p = p.astype(np.float32)
    x = (p - p.mean(0)).astype(np.float64) / a
    for h in (*hidden, 4):
        w = rng.normal(0.0, 1.0 / np.sqrt(x.shape[1]), size=(x.shape[1], h)) * 2.0
        bias = rng.normal(0.0, 0.1, size=h)
        x = x @ w + bias
        if h != 4:
            x = np.tanh(x)
    return p, FOUR[np.argmax(x, axis=1)]


def nn_robot(rng: np.random.Generator, n_masses: int, k: int = 25, axes=(0.3, 0.2, 0.15),
             hidden=(25, 25), mass: float = 0.1) -> Element:
    """Point-cloud robot (nn_points) with k-nearest-neighbour springs, built
    on the host: each unordered pair once, the lower index first, in
    lexicographic order, the initial distance as mean length and the
    composite material of the two masses."""
    from .materials import composite_id
    p, mats = nn_points(rng, n_masses, axes, hidden)
    # k nearest neighbours of every mass (float32 distances, ties by index)
    d2 = ((p[:, None, :] - p[None, :, :]) ** 2).sum(-1)
    np.fill_diagonal(d2, np.inf)
    nb = np.argsort(d2, axis=1, kind="stable")[:, :k]
    i = np.repeat(np.arange(n_masses), k)
    j = nb.reshape(-1)
    pairs = np.unique(np.stack([np.minimum(i, j), np.maximum(i, j)], 1), axis=0)
    diff = p[pairs[:, 0]] - p[pairs[:, 1]]
    lbar = np.sqrt((diff * diff).sum(1)).astype(np.float32)
    smat = np.array([composite_id(int(mats[u]), int(mats[v])) for u, v in pairs], np.uint8)
    return Element(p, mats, pairs.astype(np.uint16), lbar, smat, mass=np.full(n_masses, mass, np.float32))


def knn_springs(points: list, materials: list, k: int = 25, device: int = 0):
    """The springs nn_robot builds, for many robots at once on the GPU
    (mb_knn_springs).  Returns (spring_offsets, pairs, spring_material,
    lbar) over the robots in order."""
    R = len(points)
    mo = np.zeros(R + 1, np.int64)
    mo[1:] = np.cumsum([len(p) for p in points])
    pos = np.ascontiguousarray(np.concatenate(points), np.float32)
    mm = np.ascontiguousarray(np.concatenate(materials), np.uint8)
    so = np.zeros(R + 1, np.int64)
    # one call: a mass has at most k springs of its own, so M * k bounds the
    # count (the arrays are not touched beyond what the call writes)
    cap = int(mo[-1]) * k
    pairs = np.empty((cap, 2), np.uint16)
    smat = np.empty(cap, np.uint8)
    lbar = np.empty(cap, np.float32)
    _lib.check(_lib.LIB.mb_knn_springs(device, R, _lib.ptr(mo), _lib.ptr(pos), _lib.ptr(mm), k, _lib.ptr(so),
                                       _lib.ptr(pairs), _lib.ptr(smat), _lib.ptr(lbar), cap))
    S = int(so[-1])
    return so, pairs[:S], smat[:S], lbar[:S]


def nn_population_device(n_robots: int = 256, seed_base: int = 2000, mass: float = 0.1, k: int = 25,
                         device: int = 0) -> list[Element]:
    """population("nn", ...) with the springs built on the GPU."""
    pts, mats = [], []
    for r in range(n_robots):
        rng = np.random.default_rng(seed_base + r)
        p, m = nn_points(rng, int(rng.integers(500, 2001)))
        pts.append(p)
        mats.append(m)
    so, pairs, smat, lbar = knn_springs(pts, mats, k, device)
    return [Element(pts[r], mats[r], pairs[so[r]:so[r + 1]], lbar[so[r]:so[r + 1]], smat[so[r]:so[r + 1]],
                    mass=np.full(len(pts[r]), mass, np.float32)) for r in range(n_robots)]


def population(name: str, n_robots: int | None = None, seed_base: int | None = None,
               mass: float = 1.0, faces: bool = False) -> list[Element]:
    """One of the named synthetic populations (see module docstring); with
    faces=True every robot carries its surface triangles."""
    spec = {
        "small": (0, 32),
        "uneven": (1, 512),
        "nn": (2, 256),
        "streamed": (4, 64),
    }
    if name not in spec:
        raise ValueError(f"unknown population {name!r}")
    base, default_n = spec[name]
    n = default_n if n_robots is None else n_robots
    seed0 = 1000 * base if seed_base is None else seed_base
    out = []
    for r in range(n):
        rng = np.random.default_rng(seed0 + r)
        if name == "nn":
            e = nn_robot(rng, int(rng.integers(500, 2001)), mass=mass)
            if faces:
                e.faces = hull_faces(e.pos)
            out.append(e)
            continue
        if name == "small":
            cells = random_cells(4, rng)
        elif name == "uneven":
            side = int(rng.integers(3, 9))
            cells = random_cells(side, rng)
        else:
            cells = FOUR[rng.integers(0, 4, size=(10, 10, 10))]
        e = voxel_robot(cells, mass=mass)
        if faces:
            e.faces = voxel_faces(cells)
        out.append(e)
    return out


def population_batch(name: str, n_robots: int | None = None, seed_base: int | None = None,
                     mass: float = 1.0, faces: bool = False):
    return pack(population(name, n_robots, seed_base, mass, faces))
