"""mercury_b200: B200-native batched soft-body simulation step.

The product is the C-ABI shared library libmercury_b200.so (CUDA kernels for
sm_100a + host C++), declared in include/mercury_b200.h.  This package is its
Python host side: a mirror of the reference's Simulator API, the Element data
model, material tables and seeded robot populations.
"""
from ._lib import LIB, MercuryError  # noqa: F401  (fails loudly if the library is missing)
from .element import Batch, Element, pack, unpack  # noqa: F401
from .materials import COMPOSITE_COUNT, material_table  # noqa: F401
from .simulator import ElementTracker, Simulator, SimulatorConfig, body_length, fitness, plan  # noqa: F401

__version__ = LIB.mb_version().decode()
