"""The host-side packer and launch planner (mb_plan_population), without a
GPU: balance of the bins, the streamed cutover, capacity errors."""
import numpy as np
import pytest

import mercury_b200 as mb
from mercury_b200 import robots


def test_uneven_population_fills_whole_waves_evenly():
    b = robots.population_batch("uneven")
    st = mb.plan(b)
    assert st["streamed"] == 0 and st["bins"] % 148 == 0
    assert st["active_springs"] == b.active_springs() and st["masses"] == b.n_masses
    assert st["max_bin_springs"] <= 1.1 * st["min_bin_springs"]
    assert st["max_smem_bytes"] <= 232448
    assert st["incidence_entries"] - st["incidence_padding"] == 2 * st["active_springs"]
    assert st["aligned_slices"] > 5 * st["rank_slices"]


def test_large_robots_are_streamed():
    st = mb.plan(robots.population_batch("streamed", 8))
    assert st["streamed"] == 1 and st["bins"] == 8 and st["threads"] == 1024


def test_forced_shape_and_bins():
    b = robots.population_batch("small")
    st = mb.plan(b, threads=512, springs_per_thread=8, masses_per_thread=2, bins=8)
    assert (st["threads"], st["springs_per_thread"], st["bins"], st["streamed"]) == (512, 8, 8, 0)
    # a bin count too small for the shape's capacity falls back to streaming
    assert mb.plan(b, threads=512, springs_per_thread=8, masses_per_thread=2, bins=2)["streamed"] == 1


def test_bins_follow_the_sm_count():
    b = robots.population_batch("uneven")
    assert mb.plan(b, num_sms=296)["bins"] == 296  # one bin per SM when robots allow
    assert mb.plan(b, num_sms=74)["bins"] % 74 == 0  # whole waves


def test_oversized_robot_is_rejected():
    grid = np.full((20, 20, 20), 22, np.uint8)
    with pytest.raises(mb.MercuryError) as e:
        mb.plan(mb.pack([robots.lattice_robot(grid)]))
    assert e.value.status == 3


def test_bad_topology_is_rejected():
    b = robots.population_batch("small", 2)
    b.pairs[0, 0] = 999
    with pytest.raises(mb.MercuryError) as e:
        mb.plan(b)
    assert e.value.status == 1
