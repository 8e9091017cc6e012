"""The C++ drop-in Simulator (mercury_b200/compat): the reference's callers
compile against it unchanged, and a C++ program that uses it the way the
reference's TestSimulator does gets deterministic fitness and states equal
to the oracle's bit for bit."""
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "tests", "cpp", "_bin", "test_dropin")


def _reference_dir():
    sys.path.insert(0, ROOT)
    import __graft_entry__
    return __graft_entry__.reference_dir()


@pytest.mark.skipif(_reference_dir() is None, reason="needs the reference sources")
def test_reference_callers_compile_against_dropin():
    r = subprocess.run(["make", "-C", os.path.join(ROOT, "tests", "cpp"), "check-callers",
                        f"REF={_reference_dir()}"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]


def _read(path):
    buf = open(path, "rb").read()
    off = 0

    def take(dtype, n):
        nonlocal off
        a = np.frombuffer(buf, dtype, n, off)
        off += a.nbytes
        return a.copy()

    R = int(take(np.uint32, 1)[0])
    robots = []
    for _ in range(R):
        nm, ns = (int(x) for x in take(np.uint32, 2))
        masses = [(take(np.float32, 4), int(take(np.uint8, 1)[0])) for _ in range(nm)]
        springs = [(take(np.uint16, 2), int(take(np.uint8, 1)[0]), float(take(np.float32, 1)[0])) for _ in range(ns)]
        out = take(np.float32, 6 * nm).reshape(nm, 6)
        st = take(np.float32, ns)
        devo = [(take(np.uint16, 2), int(take(np.uint8, 1)[0]), take(np.float32, 1)[0]) for _ in range(ns)]
        robots.append((masses, springs, out, st, devo))
    tt = float(take(np.float32, 1)[0])
    return robots, tt


@pytest.mark.gpu
def test_dropin_matches_oracle(tmp_path):
    if not os.path.exists(BIN):
        pytest.skip("tests/cpp/_bin/test_dropin not built")
    import mercury_b200 as mb
    from oracle import core
    out = str(tmp_path / "dropin.bin")
    r = subprocess.run([BIN, out], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    robots, tt = _read(out)
    els = []
    for masses, springs, _, _, _ in robots:
        pos = np.array([m[0][:3] for m in masses], np.float32)
        els.append(mb.Element(pos, np.array([m[1] for m in masses], np.uint8),
                              np.array([s[0] for s in springs], np.uint16),
                              np.array([s[2] for s in springs], np.float32),
                              np.array([s[1] for s in springs], np.uint8),
                              mass=np.array([m[0][3] for m in masses], np.float32)))
    b = mb.pack(els)
    n = core.step_count(0.25, 1e-3)
    p, v = b.pos.copy(), b.vel.copy()
    s = np.zeros(b.n_springs, np.float32)
    core.xpbd_run(b, p, v, s, core.material_table(), 1e-3, 0.0, n, True)
    assert tt == core.advance_clock(0.0, 1e-3, n)
    for k, (_, _, o, st, _) in enumerate(robots):
        ms, ss = b.robot_slices(k)
        assert np.array_equal(o[:, :3].view(np.uint32), p[ms, :3].view(np.uint32))
        assert np.array_equal(o[:, 3:].view(np.uint32), v[ms, :3].view(np.uint32))
        assert np.array_equal(st.view(np.uint32), s[ss].view(np.uint32))
    # Devo(): replaced_springs_per_element = 128 (config.h:18), seed 0
    pairs, mat, lbar, recs = core.devo(b, p, s, core.material_table(), tt, 128, 0)
    assert len(recs) > 0
    for k, (_, _, _, _, devo) in enumerate(robots):
        ss = b.robot_slices(k)[1]
        assert np.array_equal(np.array([d[0] for d in devo], np.uint16).reshape(-1, 2), pairs[ss])
        assert np.array_equal(np.array([d[1] for d in devo], np.uint8), mat[ss])
        assert np.array_equal(np.array([d[2] for d in devo], np.float32).view(np.uint32),
                              lbar[ss].view(np.uint32))


@pytest.mark.gpu
def test_screened_evaluation_in_the_reference_evaluator_loop():
    """ScreenedEvaluator<VoxelRobot> (mercury_b200/compat/ScreenedEvaluator.h)
    in place of Evaluator<VoxelRobot>::BatchEvaluate, on children of the
    reference's own VoxelRobot::Crossover: warm-up evaluations equal the full
    ones, then only the screened children are evaluated (bit for bit what the
    full evaluation gives them), the rest carry fitness 0, a child outside the
    surrogate's classes is always evaluated, and the screen finds the best
    children better than chance (tests/cpp/test_screened.cpp)."""
    exe = os.path.join(ROOT, "tests", "cpp", "_bin", "test_screened")
    if not os.path.exists(exe):
        pytest.skip("tests/cpp/_bin/test_screened not built")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    kv = dict(x.split("=") for x in r.stdout.strip().splitlines()[-1].split())
    assert kv["ok"] == "1" and int(kv["unrepresentable"]) == 1
    assert float(kv["recall"]) > float(kv["chance"]) + 0.1, r.stdout
