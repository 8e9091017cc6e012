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
    # several waves: one CTA per group of bins, and the groups are what must be even
    if st["ctas"] < st["bins"]:
        assert st["ctas"] == 148 and st["max_cta_springs"] <= 1.05 * st["min_cta_springs"]
    else:
        assert st["max_bin_springs"] <= 1.1 * st["min_bin_springs"]
    assert st["max_smem_bytes"] <= 232448
    assert st["incidence_entries"] - st["incidence_padding"] == 2 * st["active_springs"]
    assert st["aligned_slices"] > 5 * st["rank_slices"]


def test_automatic_plan_leaves_room_for_register_rows():
    """Bins of a 1,024-thread shape hold at most 1,024 masses, with room for
    the register-row kernel's 8 bytes of shared memory per spring."""
    b = robots.population_batch("uneven")
    st = mb.plan(b)
    assert st["threads"] == 1024 and st["masses"] / st["bins"] <= 1024
    assert st["max_smem_bytes"] + 8 * st["max_bin_springs"] + 8 <= 232448


def test_large_robots_are_split_over_clusters():
    b = robots.population_batch("streamed", 8)
    st = mb.plan(b)  # 10x10x10 cells: two parts of at most 8,192 springs
    assert (st["cluster"], st["bins"], st["streamed"], st["threads"]) == (2, 16, 0, 1024)
    assert st["max_bin_springs"] <= 8192 and st["max_smem_bytes"] <= 232448
    # a part holds every spring touching it: the cut's springs are in both
    assert st["active_springs"] == b.active_springs()
    st4 = mb.plan(b, cluster=4)
    assert (st4["cluster"], st4["bins"]) == (4, 32)
    assert st4["max_bin_springs"] < st["max_bin_springs"]


def _chain(n):
    """A robot of n masses in a line, one spring between neighbours."""
    pos = np.zeros((n, 3), np.float32)
    pos[:, 0] = 0.1 * np.arange(n)
    pairs = np.stack([np.arange(n - 1), np.arange(1, n)], 1)
    return mb.Element(pos, np.full(n, 1, np.uint8), pairs, np.full(n - 1, 0.1, np.float32),
                      np.full(n - 1, 1, np.uint8))


def test_split_parts_take_one_mass_per_thread_unless_that_costs_ctas():
    """Parts of split robots run one own mass per thread, except when two per
    thread would place the population in fewer CTAs: 1,500-mass chains fit a
    CTA whole at two masses per thread but need two parts at one."""
    big = robots.population("streamed", 1)[0]
    st = mb.plan(mb.pack([big, big]))
    assert (st["masses_per_thread"], st["bins"], st["cluster"]) == (1, 4, 2)
    st = mb.plan(mb.pack([big, _chain(1500)]))  # four bins either way
    assert (st["masses_per_thread"], st["bins"]) == (1, 4)
    st = mb.plan(mb.pack([big, _chain(1500), _chain(1500)]))  # four bins, not six
    assert (st["masses_per_thread"], st["bins"], st["cluster"]) == (2, 4, 2)


def test_large_robots_are_streamed_when_never_split():
    st = mb.plan(robots.population_batch("streamed", 8), cluster=1)
    assert st["streamed"] == 1 and st["bins"] == 8 and st["threads"] == 1024 and st["cluster"] == 0


def test_point_cloud_robots_need_four_part_clusters():
    b = robots.population_batch("nn", 6)
    assert mb.plan(b)["cluster"] == 4
    with pytest.raises(mb._lib.MercuryError):
        mb.plan(b, cluster=2)
    with pytest.raises(mb._lib.MercuryError):
        mb.plan(b, cluster=3)


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
    with pytest.raises(mb._lib.MercuryError) as e:
        mb.plan(mb.pack([robots.lattice_robot(grid)]))
    assert e.value.status == 3


def test_bad_topology_is_rejected():
    b = robots.population_batch("small", 2)
    b.pairs[0, 0] = 999
    with pytest.raises(mb._lib.MercuryError) as e:
        mb.plan(b)
    assert e.value.status == 1


def test_split_robots_take_their_fewest_parts_and_share_clusters():
    """Automatic split: each robot is cut into as few parts as fit, and
    robots with fewer parts than the cluster size share a cluster."""
    b = robots.population_batch("nn", 24)
    auto, uniform = mb.plan(b), mb.plan(b, cluster=4)
    assert auto["cluster"] == uniform["cluster"] == 4
    assert auto["bins"] < uniform["bins"] == 96 and uniform["cluster2"] == 0
    # robots of more than two parts in clusters of four from bin 0; the rest
    # in two-CTA clusters from split_bins0 on
    assert auto["cluster2"] == 2 and auto["split_bins0"] % 4 == 0
    assert 0 < auto["split_bins0"] < auto["bins"] and (auto["bins"] - auto["split_bins0"]) % 2 == 0
    assert auto["active_springs"] == uniform["active_springs"] == b.active_springs()
    assert auto["max_smem_bytes"] <= 232448
