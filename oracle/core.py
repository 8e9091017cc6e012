"""Python wrapper of the CPU oracle liboracle.so (mercury_oracle.c).

Test infrastructure: the checker for the CUDA kernels, never the product.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liboracle.so")

_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} missing; run `make -C oracle oracle`")
        L = ctypes.CDLL(LIB_PATH)
        P, U32, I32, F32, F64 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int, ctypes.c_float, ctypes.c_double
        L.or_material_table.argtypes = [P]
        L.or_material_table.restype = None
        L.or_decode_id.argtypes = [U32]
        L.or_decode_id.restype = I32
        L.or_composite_id.argtypes = [I32, I32]
        L.or_composite_id.restype = I32
        L.or_step_count.argtypes = [F32, F32]
        L.or_step_count.restype = U32
        L.or_advance_clock.argtypes = [F32, F32, U32]
        L.or_advance_clock.restype = F32
        L.or_sin.argtypes = [F64]
        L.or_sin.restype = F64
        L.or_xpbd_run.argtypes = [I32, P, P, P, P, P, P, P, P, P, F32, F32, U32, I32, I32]
        L.or_xpbd_run.restype = I32
        L.or_xpbd_run_f64.argtypes = [I32, P, P, P, P, P, P, P, P, P, F64, F64, U32, I32]
        L.or_xpbd_run_f64.restype = I32
        L.or_com_device.argtypes = [I32, P, P, P, P]
        L.or_com_device.restype = None
        L.or_com_reference.argtypes = [I32, P, P, P, P]
        L.or_com_reference.restype = None
        L.or_force_run.argtypes = [I32, I32, P, P, P, P, P, P, P, P, P, P, F32, F32, U32, I32, I32, P, P]
        L.or_force_run.restype = I32
        L.or_face_force.argtypes = [P, P, P, P, P, P, F32, P]
        L.or_face_force.restype = None
        L.or_face_forces.argtypes = [I32, P, P, I32, P, F32, P]
        L.or_face_forces.restype = None
        L.or_force_run_f64.argtypes = [I32, I32, P, P, P, P, P, P, P, P, P, F64, F64, U32]
        L.or_force_run_f64.restype = I32
        U64 = ctypes.c_uint64
        L.or_devo.argtypes = [I32, P, P, P, P, P, P, P, P, P, F32, U32, U64, U32, P]
        L.or_devo.restype = ctypes.c_long
        L.or_devo_pair.argtypes = [U64, U32, U32, U32, P, P]
        L.or_devo_pair.restype = None
        L.or_stress_key.argtypes = [F32]
        L.or_stress_key.restype = U32
        L.or_max_threads.argtypes = []
        L.or_max_threads.restype = I32
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data


def material_table() -> np.ndarray:
    t = np.zeros((254, 4), np.float32)
    lib().or_material_table(_p(t))
    return t


def decode_id(enc: int) -> int:
    return lib().or_decode_id(enc)


def step_count(duration: float, dt: float) -> int:
    return lib().or_step_count(duration, dt)


def advance_clock(t0: float, dt: float, steps: int) -> float:
    return lib().or_advance_clock(t0, dt, steps)


def sin(x: float) -> float:
    return lib().or_sin(x)


def max_threads() -> int:
    return lib().or_max_threads()


def xpbd_run(batch, pos, vel, stress, table, dt, t0, steps, track, threads=0):
    """Runs the FP32 restatement in place on pos/vel ((M,4) float32) and
    stress ((S,) float32)."""
    assert pos.dtype == np.float32 and pos.flags.c_contiguous
    assert vel.dtype == np.float32 and vel.flags.c_contiguous
    table = np.ascontiguousarray(table, np.float32)
    rc = lib().or_xpbd_run(batch.n_robots, _p(batch.mass_offsets), _p(pos), _p(vel),
                           _p(batch.spring_offsets), _p(batch.pairs), _p(batch.spring_material),
                           _p(batch.lbar), _p(stress), _p(table), dt, t0, steps,
                           int(bool(track)), threads)
    assert rc == 0


def xpbd_run_f64(batch, pos, vel, stress, table, dt, t0, steps, track):
    assert pos.dtype == np.float64 and vel.dtype == np.float64
    lbar = np.ascontiguousarray(batch.lbar, np.float64)
    table = np.ascontiguousarray(table, np.float32)
    rc = lib().or_xpbd_run_f64(batch.n_robots, _p(batch.mass_offsets), _p(pos), _p(vel),
                               _p(batch.spring_offsets), _p(batch.pairs), _p(batch.spring_material),
                               _p(lbar), _p(stress), _p(table), dt, t0, steps, int(bool(track)))
    assert rc == 0


def com_device(batch, pos) -> np.ndarray:
    com = np.zeros((batch.n_robots, 3), np.float32)
    lib().or_com_device(batch.n_robots, _p(batch.mass_offsets), _p(np.ascontiguousarray(pos, np.float32)),
                        _p(batch.mass_material), _p(com))
    return com


def com_reference(batch, pos) -> np.ndarray:
    com = np.zeros((batch.n_robots, 3), np.float32)
    lib().or_com_reference(batch.n_robots, _p(batch.mass_offsets), _p(np.ascontiguousarray(pos, np.float32)),
                           _p(batch.mass_material), _p(com))
    return com


def force_run(mode, batch, pos, vel, stress, table, env, dt, t0, steps, track, threads=0):
    """Force modes (1 land, 2 water), FP32, in place.  env = (g, floor
    stiffness, mu_s, mu_k, drag, damping[, face_drag]); the batch's faces
    (if any) drag in water when face_drag is given."""
    assert pos.dtype == np.float32 and vel.dtype == np.float32
    table = np.ascontiguousarray(table, np.float32)
    envf = np.ascontiguousarray(env, np.float32)
    fo = getattr(batch, "face_offsets", None)
    faces = len(envf) > 6 and fo is not None and int(fo[-1]) > 0
    rc = lib().or_force_run(mode, batch.n_robots, _p(batch.mass_offsets), _p(pos), _p(vel),
                            _p(batch.spring_offsets), _p(batch.pairs), _p(batch.spring_material),
                            _p(batch.lbar), _p(stress), _p(table), _p(envf), dt, t0, steps,
                            int(bool(track)), threads,
                            _p(fo) if faces else None, _p(batch.faces) if faces else None)
    assert rc == 0


def face_force(x, v, coef):
    """Share per corner of the face drag of one triangle: x, v (3, 3) float32
    corner positions and velocities, coef = -rho/6 (float32)."""
    x = np.ascontiguousarray(x, np.float32).reshape(3, 3)
    v = np.ascontiguousarray(v, np.float32).reshape(3, 3)
    out = np.zeros(3, np.float32)
    lib().or_face_force(_p(x[0]), _p(x[1]), _p(x[2]), _p(v[0]), _p(v[1]), _p(v[2]), np.float32(coef), _p(out))
    return out


def face_forces(pos4, vel4, faces, coef):
    """Per-mass sums of the face shares of one robot (faces ascending):
    pos4, vel4 (M, 4) float32, faces (F, 3) uint16.  Returns (M, 3)."""
    pos4 = np.ascontiguousarray(pos4, np.float32)
    vel4 = np.ascontiguousarray(vel4, np.float32)
    faces = np.ascontiguousarray(faces, np.uint16)
    out = np.zeros((len(pos4), 3), np.float32)
    lib().or_face_forces(len(pos4), _p(pos4), _p(vel4), len(faces), _p(faces), np.float32(coef), _p(out))
    return out


def force_run_f64(mode, batch, pos, vel, table, env, dt, t0, steps):
    assert pos.dtype == np.float64 and vel.dtype == np.float64
    lbar = np.ascontiguousarray(batch.lbar, np.float64)
    rc = lib().or_force_run_f64(mode, batch.n_robots, _p(batch.mass_offsets), _p(pos), _p(vel),
                                _p(batch.spring_offsets), _p(batch.pairs), _p(batch.spring_material),
                                _p(lbar), _p(np.ascontiguousarray(table, np.float32)),
                                _p(np.ascontiguousarray(env, np.float64)), dt, t0, steps)
    assert rc == 0


DEVO_REFERENCE_RANKS = 1


def devo(batch, pos, stress, table, t, k, seed, flags=0):
    """Development step on a copy of the batch's topology.  Returns
    (pairs, spring_material, lbar, records) with records an (n, 4) uint32
    array: global spring, a | b << 16, material, mean-length bits."""
    pairs = np.ascontiguousarray(batch.pairs, np.uint16).copy()
    mat = np.ascontiguousarray(batch.spring_material, np.uint8).copy()
    lbar = np.ascontiguousarray(batch.lbar, np.float32).copy()
    out = np.zeros((max(batch.n_robots * k, 1), 4), np.uint32)
    n = lib().or_devo(batch.n_robots, _p(batch.mass_offsets), _p(np.ascontiguousarray(pos, np.float32)),
                      _p(batch.mass_material), _p(batch.spring_offsets), _p(pairs), _p(mat), _p(lbar),
                      _p(np.ascontiguousarray(stress, np.float32)), _p(np.ascontiguousarray(table, np.float32)),
                      t, k, seed, flags, _p(out))
    return pairs, mat, lbar, out[:n]


def devo_pair(seed: int, robot: int, j: int, m: int):
    a, b = ctypes.c_uint32(), ctypes.c_uint32()
    lib().or_devo_pair(seed, robot, j, m, ctypes.byref(a), ctypes.byref(b))
    return a.value, b.value


def stress_key(s: float) -> int:
    return lib().or_stress_key(s)
