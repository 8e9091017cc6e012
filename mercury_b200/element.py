"""The reference's Element data model (common/simulator/element.h, mass.h,
spring.h) as numpy arrays, and the packing of a list of Elements into the
flat arrays of the C ABI.

Element.masses: pos (M, 3) float32, vel (M, 3) float32, material (M,) base
id, mass (M,) float32 (reference default 1.0, mass.h:17).
Element.springs: pairs (S, 2) uint16 robot-local mass indices, mean_length
(S,) float32, material (S,) composite id; rest_length mirrors mean_length as
the reference initialises it (VoxelRobot.cpp:149).
Element.faces: (F, 3) uint16 robot-local corners of the surface triangles
(Face, face.h:6-10), or None; they act only through the face drag of the
water mode.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class Element:
    pos: np.ndarray
    mass_material: np.ndarray
    pairs: np.ndarray
    mean_length: np.ndarray
    spring_material: np.ndarray
    vel: np.ndarray | None = None
    mass: np.ndarray | None = None
    stress: np.ndarray | None = None
    sim_time: float = 0.0
    total_sim_time: float = 0.0
    faces: np.ndarray | None = None

    def __post_init__(self):
        self.pos = np.ascontiguousarray(self.pos, np.float32).reshape(-1, 3)
        m = self.pos.shape[0]
        self.mass_material = np.ascontiguousarray(self.mass_material, np.uint8).reshape(m)
        self.pairs = np.ascontiguousarray(self.pairs, np.uint16).reshape(-1, 2)
        s = self.pairs.shape[0]
        self.mean_length = np.ascontiguousarray(self.mean_length, np.float32).reshape(s)
        self.spring_material = np.ascontiguousarray(self.spring_material, np.uint8).reshape(s)
        self.vel = (np.zeros((m, 3), np.float32) if self.vel is None
                    else np.ascontiguousarray(self.vel, np.float32).reshape(m, 3))
        self.mass = (np.ones(m, np.float32) if self.mass is None
                     else np.ascontiguousarray(self.mass, np.float32).reshape(m))
        if self.faces is not None:
            self.faces = np.ascontiguousarray(self.faces, np.uint16).reshape(-1, 3)

    @property
    def n_masses(self) -> int:
        return self.pos.shape[0]

    @property
    def n_springs(self) -> int:
        return self.pairs.shape[0]

    def copy(self) -> "Element":
        return Element(self.pos.copy(), self.mass_material.copy(), self.pairs.copy(),
                       self.mean_length.copy(), self.spring_material.copy(),
                       self.vel.copy(), self.mass.copy(),
                       None if self.stress is None else self.stress.copy(),
                       self.sim_time, self.total_sim_time,
                       None if self.faces is None else self.faces.copy())


@dataclass
class Batch:
    """A population in the flat layout of mb_batch_desc."""
    mass_offsets: np.ndarray   # int64 (R+1,)
    pos: np.ndarray            # float32 (M, 4): x, y, z, mass
    vel: np.ndarray            # float32 (M, 4)
    mass_material: np.ndarray  # uint8 (M,)
    spring_offsets: np.ndarray # int64 (R+1,)
    pairs: np.ndarray          # uint16 (S, 2)
    spring_material: np.ndarray# uint8 (S,)
    lbar: np.ndarray           # float32 (S,)
    extra: dict = field(default_factory=dict)
    face_offsets: np.ndarray | None = None  # int64 (R+1,), or None: no faces
    faces: np.ndarray | None = None         # uint16 (F, 3) robot-local corners

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
        """Springs that act: non-air material (sim_kernel.cu:211)."""
        return int(np.count_nonzero(self.spring_material))

    def robot_slices(self, r: int):
        return (slice(int(self.mass_offsets[r]), int(self.mass_offsets[r + 1])),
                slice(int(self.spring_offsets[r]), int(self.spring_offsets[r + 1])))


def pack(elements: list[Element]) -> Batch:
    """Concatenates Elements into the C-ABI layout."""
    nm = np.array([e.n_masses for e in elements], np.int64)
    ns = np.array([e.n_springs for e in elements], np.int64)
    mo = np.concatenate([[0], np.cumsum(nm)]).astype(np.int64)
    so = np.concatenate([[0], np.cumsum(ns)]).astype(np.int64)
    M, S = int(mo[-1]), int(so[-1])
    pos = np.zeros((M, 4), np.float32)
    vel = np.zeros((M, 4), np.float32)
    mm = np.zeros(M, np.uint8)
    pairs = np.zeros((S, 2), np.uint16)
    sm = np.zeros(S, np.uint8)
    lb = np.zeros(S, np.float32)
    for r, e in enumerate(elements):
        a, b = mo[r], mo[r + 1]
        pos[a:b, :3] = e.pos
        pos[a:b, 3] = e.mass
        vel[a:b, :3] = e.vel
        mm[a:b] = e.mass_material
        c, d = so[r], so[r + 1]
        pairs[c:d] = e.pairs
        sm[c:d] = e.spring_material
        lb[c:d] = e.mean_length
    if all(e.faces is None for e in elements):
        return Batch(mo, pos, vel, mm, so, pairs, sm, lb)
    nf = np.array([0 if e.faces is None else len(e.faces) for e in elements], np.int64)
    fo = np.concatenate([[0], np.cumsum(nf)]).astype(np.int64)
    faces = np.zeros((int(fo[-1]), 3), np.uint16)
    for r, e in enumerate(elements):
        if e.faces is not None:
            faces[fo[r]:fo[r + 1]] = e.faces
    return Batch(mo, pos, vel, mm, so, pairs, sm, lb, face_offsets=fo, faces=faces)


def unpack(batch: Batch, pos: np.ndarray, vel: np.ndarray, stress: np.ndarray | None,
           template: list[Element]) -> list[Element]:
    """Splits device results back into Elements shaped like `template`."""
    out = []
    for r, e in enumerate(template):
        ms, ss = batch.robot_slices(r)
        x = e.copy()
        x.pos = pos[ms, :3].copy()
        x.vel = vel[ms, :3].copy()
        # topology from the batch: development may have rewired springs, a
        # device build decides the materials
        x.mass_material = batch.mass_material[ms].copy()
        x.pairs = batch.pairs[ss].copy()
        x.spring_material = batch.spring_material[ss].copy()
        x.mean_length = batch.lbar[ss].copy()
        if stress is not None:
            x.stress = stress[ss].copy()
        out.append(x)
    return out
