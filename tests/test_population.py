"""The oracle's populations (built by the reference's own VoxelRobot::Build,
oracle/population.py) are the product's populations (mercury_b200/robots.py)
bit for bit, so bench.py's reference arm and the product simulate the same
robots without the reference arm loading the product."""
import os

import numpy as np
import pytest

import mercury_b200 as mb
from mercury_b200 import robots
from oracle import core, population

pytestmark = pytest.mark.skipif(not os.path.exists(population.REF_LIB), reason="reference build absent")


@pytest.mark.parametrize("name,n", [("small", 32), ("uneven", 48), ("streamed", 3)])
def test_same_robots_as_product(name, n):
    a = population.population_batch(name, n)
    b = robots.population_batch(name, n)
    for k in ("mass_offsets", "pos", "vel", "mass_material", "spring_offsets", "pairs", "spring_material", "lbar"):
        x, y = getattr(a, k), getattr(b, k)
        assert x.dtype == y.dtype and x.shape == y.shape, k
        assert np.array_equal(x.view(np.uint8), y.view(np.uint8)), k
    assert np.array_equal(a.length, mb.body_length(b))


def test_oracle_table_is_product_table():
    assert np.array_equal(core.material_table().view(np.uint32), mb.material_table().view(np.uint32))
