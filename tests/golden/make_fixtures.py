"""Generates the golden fixtures of tests/golden/ from the reference itself.

The reference (DawsonCohen/Mercury) is compiled from its own sources by
oracle/Makefile into oracle/_ref/libmercury_ref.so (IEEE flavour) and
libmercury_ref_fm.so (-use_fast_math flavour); this script only calls it
through oracle/ref_harness.cpp.

    python tests/golden/make_fixtures.py host   # no GPU needed
        ref_materials.npz     composite material table (material.h, via
                              materials::id_lookup) and materials::decode ids
                              of 2,300 encodings
        ref_voxel_robots.npz  VoxelRobot::Build output for 24 seeded grids
    python tests/golden/make_fixtures.py gpu    # on a GPU
        ref_sim.npz           Simulator::Simulate + Collect of the reference
                              CUDA step on seeded populations (both flavours)
"""
from __future__ import annotations

import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.path.join(ROOT, "oracle", "_ref", "libmercury_ref.so")
REF_FM = os.path.join(ROOT, "oracle", "_ref", "libmercury_ref_fm.so")


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def load(path=REF):
    L = ctypes.CDLL(path)
    L.ref_decode_id.argtypes = [ctypes.c_uint32]
    L.ref_decode_id.restype = ctypes.c_int
    L.ref_composite_count.restype = ctypes.c_int
    L.ref_voxel_build.argtypes = [ctypes.c_int] * 3 + [ctypes.c_float] + [ctypes.c_void_p] * 10
    L.ref_simulate.argtypes = [ctypes.c_int] + [ctypes.c_void_p] * 8 + [ctypes.c_float, ctypes.c_float,
                                                                      ctypes.c_int] + [ctypes.c_void_p] * 4
    L.ref_simulate.restype = ctypes.c_int
    # materials::decode's static table must be built before id_lookup's (the
    # harness calls both); do it first, as Simulator::SetElements does.
    L.ref_decode_id(1)
    return L


def voxel_build(L, nx, ny, nz, h, mats):
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
    L.ref_voxel_build(nx, ny, nz, h, _p(mats), _p(nm), _p(ns), _p(pos), _p(mm), _p(pairs), _p(lbar),
                      _p(sm), _p(com), _p(length))
    s = int(ns[0])
    return dict(pos=pos.reshape(n, 3), mass_material=mm, pairs=pairs[: 2 * s].reshape(s, 2),
                lbar=lbar[:s], spring_material=sm[:s], com=com, length=float(length[0]))


def host_fixtures():
    L = load()
    count = L.ref_composite_count()
    table = np.zeros((count, 4), np.float32)
    L.ref_material_table(_p(table))
    rng = np.random.default_rng(2024)
    encs = ([1 << i for i in range(23)] + [(1 << i) | (1 << j) for i in range(23) for j in range(i + 1, 23)]
            + [int(x) for x in rng.integers(0, 1 << 23, 2000)] + [0])
    encs = np.array(encs, np.uint32)
    ids = np.array([L.ref_decode_id(int(e)) for e in encs], np.int32)
    np.savez_compressed(os.path.join(HERE, "ref_materials.npz"), table=table, encodings=encs, ids=ids,
                        composite_count=count)

    five = np.array([0, 22, 21, 1, 11], np.uint8)
    p5 = [0.3, 0.175, 0.175, 0.175, 0.175]
    robots = []
    for k in range(24):
        r = np.random.default_rng(5000 + k)
        nx, ny, nz = (int(v) for v in r.integers(2, 10, 3)) if k % 4 == 3 else (int(r.integers(2, 10)),) * 3
        if k % 3 == 0:
            mats = r.integers(0, 23, nx * ny * nz).astype(np.uint8)
        else:
            mats = five[r.choice(5, nx * ny * nz, p=p5)]
        idx = np.arange(nx * ny * nz)
        ix, iy, iz = idx % nx, (idx // nx) % ny, idx // (nx * ny)
        if k % 2 == 0:
            mats[(ix == nx - 1) | (iy == ny - 1) | (iz == nz - 1)] = 0
        h = [0.1, 1.0, 0.25][k % 3]
        out = voxel_build(L, nx, ny, nz, h, mats)
        out.update(dims=np.array([nx, ny, nz], np.int32), h=h, grid=mats)
        robots.append(out)
    flat = {}
    for key in ("pos", "mass_material", "pairs", "lbar", "spring_material", "grid"):
        flat[key] = np.concatenate([r[key] for r in robots])
    flat["mass_offsets"] = np.concatenate([[0], np.cumsum([len(r["mass_material"]) for r in robots])])
    flat["spring_offsets"] = np.concatenate([[0], np.cumsum([len(r["lbar"]) for r in robots])])
    flat["grid_offsets"] = np.concatenate([[0], np.cumsum([len(r["grid"]) for r in robots])])
    flat["dims"] = np.stack([r["dims"] for r in robots])
    flat["h"] = np.array([r["h"] for r in robots], np.float32)
    flat["com"] = np.stack([r["com"] for r in robots])
    flat["length"] = np.array([r["length"] for r in robots], np.float32)
    np.savez_compressed(os.path.join(HERE, "ref_voxel_robots.npz"), **flat)
    print("wrote ref_materials.npz, ref_voxel_robots.npz")


def ref_simulate(L, batch, dt, duration, track):
    R = batch.n_robots
    mo = batch.mass_offsets.astype(np.int32)
    so = batch.spring_offsets.astype(np.int32)
    pos3 = np.ascontiguousarray(batch.pos[:, :3])
    vel3 = np.ascontiguousarray(batch.vel[:, :3])
    po = np.zeros_like(pos3)
    vo = np.zeros_like(vel3)
    st = np.zeros(batch.n_springs, np.float32)
    tt = np.zeros(1, np.float32)
    steps = L.ref_simulate(R, _p(mo), _p(pos3), _p(vel3), _p(batch.mass_material), _p(so),
                           _p(np.ascontiguousarray(batch.pairs)), _p(batch.lbar), _p(batch.spring_material),
                           dt, duration, int(track), _p(po), _p(vo), _p(st), _p(tt))
    return po, vo, st, float(tt[0]), steps


def gpu_fixtures(out_dir):
    sys.path.insert(0, ROOT)
    from mercury_b200 import robots
    cases = []
    batch = robots.population_batch("small", 8)
    for flavour, path in (("ieee", REF), ("fast", REF_FM)):
        L = load(path)
        for dt, duration in ((1e-3, 0.1), (5e-3, 0.5), (1e-4, 0.1)):
            po, vo, st, tt, steps = ref_simulate(L, batch, dt, duration, True)
            cases.append(dict(flavour=flavour, dt=dt, duration=duration, pos=po, vel=vo, stress=st,
                              total_time=tt, steps=steps))
    data = {"n_cases": len(cases)}
    for i, c in enumerate(cases):
        for k, v in c.items():
            data[f"c{i}_{k}"] = np.asarray(v)
    os.makedirs(out_dir, exist_ok=True)
    np.savez_compressed(os.path.join(out_dir, "ref_sim.npz"), **data)
    print("wrote", os.path.join(out_dir, "ref_sim.npz"))


if __name__ == "__main__":
    mode = sys.argv[1] if len(sys.argv) > 1 else "host"
    if mode == "host":
        host_fixtures()
    else:
        gpu_fixtures(sys.argv[2] if len(sys.argv) > 2 else HERE)
