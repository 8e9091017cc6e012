"""Material tables of the reference (common/simulator/material.h).

Base materials: id 0 is air, 1-10 adductor muscles, 11-20 abductor muscles,
21 tissue, 22 bone (material.h:79-107, 111-133).  A spring carries a
composite id: a base id, or for two different base materials the id
assigned by material.h:192-213, with every field the double-precision mean of
the two (material.h:215-227).  The table is laid out as the reference uploads
it (Simulator.cu:286-292): float4 {k, dL0, omega, phi} per composite id.
"""
from __future__ import annotations

import math

import numpy as np

COMPOSITE_COUNT = 254
AIR, TISSUE, BONE = 0, 21, 22
ADDUCTOR_MUSCLE0, ABDUCTOR_MUSCLE0 = 1, 11

# Named materials of the synthetic populations and the base ids they use.
NAMED = {
    "air": AIR,
    "bone": BONE,
    "tissue": TISSUE,
    "muscle_a": ADDUCTOR_MUSCLE0,  # phase 0
    "muscle_b": ABDUCTOR_MUSCLE0,  # phase pi
}


def _base(i: int) -> tuple[float, float, float, float]:
    """k, dL0, omega, phi of base material i as the reference's constexpr
    initialisers evaluate them (double expressions narrowed to float)."""
    omega = 1.0 * (2.0 * math.pi)  # OMEGA: (float)1.0f * (2.0f*M_PI), a double
    amp = float(np.float32(0.14))
    if i == 0:
        return (0.0, 0.0, 0.0, 0.0)
    if 1 <= i <= 20:
        j, abd = (i - 1) % 10, i >= 11
        if j <= 7:
            return (50.0, amp, omega, ((8 if abd else 0) + j) * math.pi / 8.0)
        if j == 8:
            return (50.0, amp, omega * 2, math.pi if abd else 0.0)
        return (50.0, amp, omega / 2, math.pi if abd else 0.0)
    if i == 21:
        return (40.0, 0.0, omega, 0.0)
    return (100.0, 0.0, omega, 0.0)


def composite_id(m1: int, m2: int) -> int:
    """Composite id of two base materials (material.h:192-213)."""
    if m1 == 0 or m2 == 0:
        return 0
    i, j = min(m1, m2) - 1, max(m1, m2) - 1
    if i == j:
        return i + 1
    return 23 + i * 21 - i * (i - 1) // 2 + (j - i - 1)


def material_table() -> np.ndarray:
    """(254, 4) float32 table indexed by composite id."""
    t = np.zeros((COMPOSITE_COUNT, 4), np.float32)
    for i in range(23):
        t[i] = np.array(_base(i), np.float64).astype(np.float32)
    for i in range(1, 23):
        a = np.array(_base(i), np.float64).astype(np.float32).astype(np.float64)
        for j in range(i + 1, 23):
            b = np.array(_base(j), np.float64).astype(np.float32).astype(np.float64)
            t[composite_id(i, j)] = ((a + b) / 2.0).astype(np.float32)
    return t


# Materials of the force-based benchmark configurations: stiffness bone
# 1e5, tissue 1e4, muscles 1e4 N/m; muscle rest length L0 (1 + 0.14 sin(2 pi
# 2 Hz t + phi)) with phi = 0 (muscle_a) and pi (muscle_b).  Composite
# springs average their two materials as the reference does
# (material.h:215-227); base materials the configurations do not use keep
# the reference's values.
FORCE_BASE = {
    BONE: (1.0e5, 0.0, 2.0 * math.pi * 2.0, 0.0),
    TISSUE: (1.0e4, 0.0, 2.0 * math.pi * 2.0, 0.0),
    ADDUCTOR_MUSCLE0: (1.0e4, 0.14, 2.0 * math.pi * 2.0, 0.0),
    ABDUCTOR_MUSCLE0: (1.0e4, 0.14, 2.0 * math.pi * 2.0, math.pi),
}


def force_table() -> np.ndarray:
    """(254, 4) float32 table of the force-based configurations."""
    def base(i):
        return FORCE_BASE.get(i, _base(i))
    t = np.zeros((COMPOSITE_COUNT, 4), np.float32)
    for i in range(23):
        t[i] = np.array(base(i), np.float64).astype(np.float32)
    for i in range(1, 23):
        a = np.array(base(i), np.float64).astype(np.float32).astype(np.float64)
        for j in range(i + 1, 23):
            b = np.array(base(j), np.float64).astype(np.float32).astype(np.float64)
            t[composite_id(i, j)] = ((a + b) / 2.0).astype(np.float32)
    return t
