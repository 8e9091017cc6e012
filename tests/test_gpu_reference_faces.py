"""The face law of the oracle against the reference's own face-drag kernel
(surfaceDragForce, common/simulator/sim_kernel.cu:66-139), compiled from
the reference's source into oracle/_ref/libmercury_ref_faces.so
(oracle/Makefile) and run on the GPU.  The reference accumulates the shares
with shared-memory atomics (order unspecified) and rounds differently
(divisions where this law multiplies by rounded reciprocals), so the
comparison is to 1e-4 of the largest force."""
import ctypes
import os

import numpy as np
import pytest

from mercury_b200 import robots
from oracle import core

pytestmark = pytest.mark.gpu

LIB = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                   "libmercury_ref_faces.so")
RHO = 1.0e6  # large, so that F dominates x + v in newPos = x + v dt + F dt^2 (dt = 1)


def reference_face_forces(pos4, vel4, faces):
    lib = ctypes.CDLL(LIB)
    P = ctypes.c_void_p
    lib.ref_surface_drag.argtypes = [ctypes.c_int, P, P, ctypes.c_int, P, ctypes.c_float, ctypes.c_float, P]
    lib.ref_surface_drag.restype = ctypes.c_int
    pos4 = np.ascontiguousarray(pos4, np.float32)
    vel4 = np.ascontiguousarray(vel4, np.float32)
    faces = np.ascontiguousarray(faces, np.uint16)
    assert faces.max() < len(pos4)  # the reference kernel does not check its corners
    new = np.zeros_like(pos4)
    rc = lib.ref_surface_drag(len(pos4), pos4.ctypes.data, vel4.ctypes.data, len(faces), faces.ctypes.data,
                              RHO, 1.0, new.ctypes.data)
    assert rc == 0
    return new[:, :3].astype(np.float64) - pos4[:, :3] - vel4[:, :3]


def cases():
    rng = np.random.default_rng(11)
    cells = robots.random_cells(4, rng)
    e = robots.voxel_robot(cells)
    yield "voxel", e.pos, robots.voxel_faces(cells), rng
    p = robots.nn_robot(rng, 300).pos
    yield "hull", p, robots.hull_faces(p), rng


@pytest.mark.parametrize("velocity", ["uniform", "random"])
def test_face_law_matches_the_reference_kernel(velocity):
    if not os.path.exists(LIB):
        pytest.skip("oracle/_ref/libmercury_ref_faces.so not built")
    for name, pos, faces, rng in cases():
        n = len(pos)
        pos4 = np.zeros((n, 4), np.float32)
        pos4[:, :3] = pos
        vel4 = np.zeros((n, 4), np.float32)
        vel4[:, :3] = ([0.3, -0.2, 0.9] if velocity == "uniform" else rng.normal(0, 1.0, (n, 3)))
        ref = reference_face_forces(pos4, vel4, faces)
        ours = core.face_forces(pos4, vel4, faces, np.float32(-RHO / 6.0)).astype(np.float64)
        scale = np.abs(ref).max()
        assert scale > 0
        assert np.abs(ours - ref).max() <= 1e-4 * scale, name
        # per mass and component: relative to the force itself, with a floor
        # of 1e-5 of the largest force for sums that cancel -- a wrong sign or
        # a missing share on a mass with a small force fails here
        err = np.abs(ours - ref)
        bound = 1e-5 * np.abs(ref) + 1e-5 * scale
        assert (err <= bound).all(), (name, float((err / bound).max()))
