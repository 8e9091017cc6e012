"""Seeded voxel-robot populations built by the reference's own VoxelRobot::Build.

Test infrastructure, like the rest of oracle/: bench.py's reference arm and
the tests use it so that the reference side of a comparison runs no code of
the product (mercury_b200/).  Robots are built by the reference's lattice
builder (common/evolvables/VoxelRobot.cpp:310-331), compiled from its sources
into oracle/_ref/libmercury_ref.so by oracle/Makefile and reached through
oracle/ref_harness.cpp (ref_voxel_build).

The draws are the same as the product's generator (mercury_b200/robots.py),
seed for seed, so both sides simulate the same robots; tests/test_population.py
checks that the two populations are identical bit for bit.

  small     32 robots of 4x4x4 cells, cells iid {air .3, bone .175, tissue .175,
            muscle_a .175, muscle_b .175}            seed 0    + robot
  uneven    512 robots, side uniform in 3..8, same materials  seed 1000 + robot
  streamed  64 robots of 10x10x10 cells, all occupied, iid over
            {bone, tissue, muscle_a, muscle_b}      seed 4000 + robot

A robot of `side` cells has (side+1)^3 grid points; grid point p carries the
material of the cell whose lowest corner is p, and the points on the upper
faces are air (VoxelRobot::Initialize, VoxelRobot.cpp:375-378).  Cell size
0.1 m.  Material ids are the reference's (material.h:111-133): air 0,
adductor_muscle0 1 (muscle_a, phase 0), abductor_muscle0 11 (muscle_b,
phase pi), tissue 21, bone 22.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(_HERE, "_ref", "libmercury_ref.so")

CELL = 0.1
AIR, ADDUCTOR_MUSCLE0, ABDUCTOR_MUSCLE0, TISSUE, BONE = 0, 1, 11, 21, 22
FIVE = np.array([AIR, BONE, TISSUE, ADDUCTOR_MUSCLE0, ABDUCTOR_MUSCLE0], np.uint8)
FIVE_P = np.array([0.3, 0.175, 0.175, 0.175, 0.175])
FOUR = np.array([BONE, TISSUE, ADDUCTOR_MUSCLE0, ABDUCTOR_MUSCLE0], np.uint8)
SPEC = {"small": (0, 32), "uneven": (1, 512), "streamed": (4, 64)}

_lib = None


def ref_lib() -> ctypes.CDLL:
    """The reference build (IEEE flavour); raises if it was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(REF_LIB):
            raise FileNotFoundError(f"{REF_LIB} missing: the reference is built by `make -C oracle ref`")
        L = ctypes.CDLL(REF_LIB)
        L.ref_decode_id.argtypes = [ctypes.c_uint32]
        L.ref_decode_id.restype = ctypes.c_int
        L.ref_voxel_build.argtypes = [ctypes.c_int] * 3 + [ctypes.c_float] + [ctypes.c_void_p] * 10
        L.ref_voxel_build.restype = ctypes.c_int
        L.ref_decode_id(1)  # materials::decode's table first, as Simulator::SetElements does
        _lib = L
    return _lib


@dataclass
class RefBatch:
    """A population in flat arrays (the attribute names oracle.core reads)."""
    mass_offsets: np.ndarray    # int64 (R+1,)
    pos: np.ndarray             # float32 (M, 4): x, y, z, mass
    vel: np.ndarray             # float32 (M, 4)
    mass_material: np.ndarray   # uint8 (M,)
    spring_offsets: np.ndarray  # int64 (R+1,)
    pairs: np.ndarray           # uint16 (S, 2)
    spring_material: np.ndarray # uint8 (S,)
    lbar: np.ndarray            # float32 (S,)
    base_com: np.ndarray        # float32 (R, 3): SoftBody::mBaseCOM after the build
    length: np.ndarray          # float32 (R,): SoftBody::mLength after the build

    @property
    def n_robots(self) -> int:
        return len(self.mass_offsets) - 1

    @property
    def n_masses(self) -> int:
        return int(self.mass_offsets[-1])

    @property
    def n_springs(self) -> int:
        return int(self.spring_offsets[-1])

    def active_springs(self) -> int:
        return int(np.count_nonzero(self.spring_material))

    def robot_slices(self, r: int):
        return (slice(int(self.mass_offsets[r]), int(self.mass_offsets[r + 1])),
                slice(int(self.spring_offsets[r]), int(self.spring_offsets[r + 1])))


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def build_cells(cells: np.ndarray, h: float = CELL):
    """VoxelRobot::Build of a cell grid (indexed [x, y, z]) with an air layer
    of grid points closing its upper faces."""
    cells = np.asarray(cells, np.uint8)
    sx, sy, sz = cells.shape
    nx, ny, nz = sx + 1, sy + 1, sz + 1
    grid = np.zeros((nx, ny, nz), np.uint8)
    grid[:sx, :sy, :sz] = cells
    mats = np.ascontiguousarray(grid.transpose(2, 1, 0).reshape(-1))  # x fastest
    n = nx * ny * nz
    pos = np.zeros(3 * n, np.float32)
    mm = np.zeros(n, np.uint8)
    pairs = np.zeros(2 * 13 * n, np.uint16)
    lbar = np.zeros(13 * n, np.float32)
    sm = np.zeros(13 * n, np.uint8)
    com = np.zeros(3, np.float32)
    length = np.zeros(1, np.float32)
    nm = np.zeros(1, np.int32)
    ns = np.zeros(1, np.int32)
    rc = ref_lib().ref_voxel_build(nx, ny, nz, h, _p(mats), _p(nm), _p(ns), _p(pos), _p(mm), _p(pairs),
                                   _p(lbar), _p(sm), _p(com), _p(length))
    if rc != 0:
        raise RuntimeError(f"ref_voxel_build failed ({rc})")
    s = int(ns[0])
    return (pos.reshape(n, 3), mm, pairs[: 2 * s].reshape(s, 2), lbar[:s], sm[:s], com, float(length[0]))


def cells_of(name: str, seed: int) -> np.ndarray:
    """The cell grid of one robot: the same draws as mercury_b200/robots.py."""
    rng = np.random.default_rng(seed)
    if name == "small":
        return FIVE[rng.choice(5, size=(4, 4, 4), p=FIVE_P)]
    if name == "uneven":
        side = int(rng.integers(3, 9))
        return FIVE[rng.choice(5, size=(side, side, side), p=FIVE_P)]
    if name == "streamed":
        return FOUR[rng.integers(0, 4, size=(10, 10, 10))]
    raise ValueError(f"unknown population {name!r}")


def population_batch(name: str, n_robots: int | None = None, seed_base: int | None = None,
                     mass: float = 1.0) -> RefBatch:
    """A named population, built robot by robot by the reference."""
    base, default_n = SPEC[name]
    n = default_n if n_robots is None else n_robots
    seed0 = 1000 * base if seed_base is None else seed_base
    robots = [build_cells(cells_of(name, seed0 + r)) for r in range(n)]
    nm = np.array([len(r[0]) for r in robots], np.int64)
    ns = np.array([len(r[2]) for r in robots], np.int64)
    mo = np.concatenate([[0], np.cumsum(nm)]).astype(np.int64)
    so = np.concatenate([[0], np.cumsum(ns)]).astype(np.int64)
    pos = np.zeros((int(mo[-1]), 4), np.float32)
    pos[:, 3] = mass
    vel = np.zeros_like(pos)
    pos[:, :3] = np.concatenate([r[0] for r in robots])
    return RefBatch(mo, pos, vel, np.concatenate([r[1] for r in robots]), so,
                    np.ascontiguousarray(np.concatenate([r[2] for r in robots])),
                    np.concatenate([r[4] for r in robots]), np.concatenate([r[3] for r in robots]),
                    np.stack([r[5] for r in robots]), np.array([r[6] for r in robots], np.float32))
