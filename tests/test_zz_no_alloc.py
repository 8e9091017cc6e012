"""The entry point that allocates nothing (mb_simulate_robot_noalloc).

It is for callers that cannot call cudaMalloc, such as an engine that owns
all device memory through its own pool: they hand over device arrays, and
the library works inside a fixed scratch array that is part of its image.
This test allocates the robot's arrays itself (with torch), then calls the
entry point through the C ABI twice in a row -- on two different robots, the
second one smaller and with stress tracking, so stale scratch contents of
the first call would show -- and checks every result against the batched
entry point (mb_set_elements + mb_run_steps + mb_collect) bit for bit, the
tolerance of the other GPU parity tests.

The file is named so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

import mercury_b200 as mb
from mercury_b200 import _lib, robots

pytestmark = pytest.mark.gpu


def _fn():
    f = mb.LIB.mb_simulate_robot_noalloc
    P, U32, F32 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_float
    f.argtypes = [P, P, U32, P, P, U32, P, P, P, P, F32, F32, U32, ctypes.c_int, ctypes.POINTER(F32)]
    f.restype = ctypes.c_int
    return f


def _batched(batch, dt, t0, steps, track):
    sim = mb.Simulator(0)
    sim.setTimeStep(dt)
    sim.set_batch(batch)
    _lib.check(mb.LIB.mb_set_total_time(sim._ctx, t0), sim._ctx)
    sim.run_steps(steps, track)
    pos, vel, stress = sim.collect_arrays()
    return pos, vel, stress, sim.getTotalTime()


def _noalloc(torch, batch, table_dev, dt, t0, steps, track):
    dev = torch.device("cuda", 0)
    pos = torch.from_numpy(batch.pos.copy()).to(dev)
    vel = torch.from_numpy(batch.vel.copy()).to(dev)
    pairs = torch.from_numpy(batch.pairs.view(np.int16).copy()).to(dev)
    mat = torch.from_numpy(batch.spring_material.copy()).to(dev)
    lbar = torch.from_numpy(batch.lbar.copy()).to(dev)
    stress = torch.zeros(batch.n_springs, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    t_end = ctypes.c_float()
    st = _fn()(stream.cuda_stream, table_dev.data_ptr(), batch.n_masses, pos.data_ptr(), vel.data_ptr(),
               batch.n_springs, pairs.data_ptr(), mat.data_ptr(), lbar.data_ptr(),
               stress.data_ptr() if track else None, dt, t0, steps, int(track), ctypes.byref(t_end))
    assert st == 0, st
    return pos.cpu().numpy(), vel.cpu().numpy(), stress.cpu().numpy(), t_end.value


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def test_noalloc_matches_batched_entry_point_on_two_calls():
    torch = pytest.importorskip("torch")
    table_dev = torch.from_numpy(mb.material_table()).to("cuda:0")
    big = mb.pack([robots.voxel_robot(robots.random_cells(8, np.random.default_rng(91)))])
    small = mb.pack([robots.voxel_robot(robots.random_cells(4, np.random.default_rng(92)))])
    for batch, dt, t0, steps, track in ((big, 1e-3, 0.0, 1234, False), (small, 5e-3, 2.5, 777, True)):
        p, v, s, t = _noalloc(torch, batch, table_dev, dt, t0, steps, track)
        rp, rv, rs, rt = _batched(batch, dt, t0, steps, track)
        assert np.array_equal(_bits(p), _bits(rp))
        assert np.array_equal(_bits(v), _bits(rv))
        if track:
            assert np.array_equal(_bits(s), _bits(rs))
        assert t == rt


def test_noalloc_rejects_robot_over_the_limit():
    grid = np.full((13, 13, 13), 22, np.uint8)  # 2197 masses > MB_NOALLOC_MAX_MASSES
    b = mb.pack([robots.lattice_robot(grid)])
    st = _fn()(None, None, b.n_masses, None, None, b.n_springs, None, None, None, None,
               1e-3, 0.0, 1, 0, None)
    assert st == 1  # null device arrays are rejected before any size logic
    torch = pytest.importorskip("torch")
    z = torch.zeros(16, device="cuda:0")
    st = _fn()(None, z.data_ptr(), b.n_masses, z.data_ptr(), z.data_ptr(), b.n_springs, z.data_ptr(),
               z.data_ptr(), z.data_ptr(), None, 1e-3, 0.0, 1, 0, None)
    assert st == 3  # MB_ERR_CAPACITY, nothing launched


def _call(torch, batch, pairs, table_dev, dt=1e-3, steps=50):
    dev = torch.device("cuda", 0)
    pos = torch.from_numpy(batch.pos.copy()).to(dev)
    vel = torch.from_numpy(batch.vel.copy()).to(dev)
    pr = torch.from_numpy(np.ascontiguousarray(pairs).view(np.int16).copy()).to(dev)
    mat = torch.from_numpy(batch.spring_material.copy()).to(dev)
    lbar = torch.from_numpy(batch.lbar.copy()).to(dev)
    return _fn()(torch.cuda.current_stream(dev).cuda_stream, table_dev.data_ptr(), batch.n_masses,
                 pos.data_ptr(), vel.data_ptr(), batch.n_springs, pr.data_ptr(), mat.data_ptr(),
                 lbar.data_ptr(), None, dt, 0.0, steps, 0, None)


def test_noalloc_device_side_rejections_then_a_valid_call():
    """The statuses the build and step kernels report, each followed by a
    valid call that must still match the batched path bit for bit (the
    scratch keeps what the rejected call left): a spring whose end is out
    of range (MB_ERR_ARGUMENT: the build kernel's bounds check leaves the bin
    empty), a hub mass whose incidence row is too wide for the scratch
    (MB_ERR_CAPACITY), and a non-finite position (MB_ERR_NONFINITE)."""
    torch = pytest.importorskip("torch")
    table_dev = torch.from_numpy(mb.material_table()).to("cuda:0")
    good = mb.pack([robots.voxel_robot(robots.random_cells(5, np.random.default_rng(93)))])

    bad = good.pairs.copy()
    bad[3, 1] = good.n_masses  # one past the last mass
    hub_n = 1500  # mass 0 joined to every other: a slice of width 1,499 > the incidence limit
    hub = mb.Batch(np.array([0, hub_n], np.int64), np.zeros((hub_n, 4), np.float32),
                   np.zeros((hub_n, 4), np.float32), np.full(hub_n, 22, np.uint8),
                   np.array([0, hub_n - 1], np.int64),
                   np.stack([np.zeros(hub_n - 1), np.arange(1, hub_n)], 1).astype(np.uint16),
                   np.full(hub_n - 1, 22, np.uint8), np.full(hub_n - 1, 0.1, np.float32))
    hub.pos[:, 0] = np.linspace(0.0, 1.0, hub_n, dtype=np.float32)
    hub.pos[:, 3] = 1.0
    nan = mb.Batch(**{k: getattr(good, k) for k in ("mass_offsets", "pos", "vel", "mass_material",
                                                    "spring_offsets", "pairs", "spring_material", "lbar")})
    nan.pos = good.pos.copy()
    nan.pos[7, 0] = np.nan
    for batch, pairs, expect in ((good, bad, 1), (hub, hub.pairs, 3), (nan, nan.pairs, 5)):
        assert _call(torch, batch, pairs, table_dev) == expect
        p, v, _, t = _noalloc(torch, good, table_dev, 1e-3, 0.25, 300, False)
        rp, rv, _, rt = _batched(good, 1e-3, 0.25, 300, False)
        assert np.array_equal(_bits(p), _bits(rp)) and np.array_equal(_bits(v), _bits(rv)) and t == rt
