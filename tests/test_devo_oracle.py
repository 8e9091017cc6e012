"""The oracle's development step (or_devo) against an independent Python
restatement and against the properties of Simulator::Devo
(Simulator.cu:640-668, devo_kernel.cu:81-168): the highest-stress springs of
every robot are rewired to random pairs of distinct masses, with the
composite material of the pair and the mean length at the current clock."""
import math
import struct

import numpy as np
import pytest

import mercury_b200 as mb
from mercury_b200 import robots
from mercury_b200.materials import composite_id, material_table
from oracle import core

M64 = (1 << 64) - 1


def _mix64(z):
    z ^= z >> 30
    z = (z * 0xBF58476D1CE4E5B9) & M64
    z ^= z >> 27
    z = (z * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


def _pair(seed, robot, j, m):
    key = _mix64((seed + 0x9E3779B97F4A7C15 * (robot + 1)) & M64)

    def draw(n):
        u = _mix64((key + 0xD1B54A32D192ED03 * (((j << 8) | n) + 1)) & M64)
        return ((u >> 32) * m) >> 32

    a, b = draw(0), draw(1)
    n = 2
    while b == a and n < 64:
        b = draw(n)
        n += 1
    if b == a:
        b = (a + 1) % m
    return a, b


def _key(s):
    u = struct.unpack("<I", struct.pack("<f", s))[0]
    if u == 0x80000000:
        u = 0
    ordv = (~u & 0xFFFFFFFF) if u & 0x80000000 else (u | 0x80000000)
    return ~ordv & 0xFFFFFFFF


def _f32(x):
    return float(np.float32(x))


def _fmaf(a, b, c):
    return _f32(a * b + c)  # a*b is exact in double for float32 operands


def py_devo(batch, pos, stress, table, t, k, seed, flags=0):
    """Straight restatement, one spring at a time."""
    pairs, mat, lbar = batch.pairs.copy(), batch.spring_material.copy(), batch.lbar.copy()
    recs = []
    for r in range(batch.n_robots):
        m0, m1 = int(batch.mass_offsets[r]), int(batch.mass_offsets[r + 1])
        s0, s1 = int(batch.spring_offsets[r]), int(batch.spring_offsets[r + 1])
        m, n = m1 - m0, s1 - s0
        if m < 2 or n == 0 or k == 0:
            continue
        lo, hi = 0, min(k, n)
        if flags & core.DEVO_REFERENCE_RANKS:
            lo, hi = min(r * k, n), min(r * k + k, n)
        ranked = sorted(range(n), key=lambda i: (_key(float(stress[s0 + i])), i))
        for q in range(lo, hi):
            j, s = q - lo, s0 + ranked[q]
            a, b = _pair(seed, r, j, m)
            cid = composite_id(int(batch.mass_material[m0 + a]), int(batch.mass_material[m0 + b]))
            pa, pb = pos[m0 + a].astype(np.float64), pos[m0 + b].astype(np.float64)
            dx, dy, dz = (_f32(pa[c] - pb[c]) for c in range(3))
            d = _f32(math.sqrt(_fmaf(dx, dx, _fmaf(dy, dy, _f32(dz * dz)))))
            arg = _fmaf(float(table[cid, 2]), t, float(table[cid, 3]))
            sn = _f32(core.sin(arg))
            den = _f32(1.0 + _f32(float(table[cid, 1]) * sn))
            L = np.float32(d) / np.float32(den)
            pairs[s] = (a, b)
            mat[s] = cid
            lbar[s] = L
            recs.append((s, a | (b << 16), cid, int(np.float32(L).view(np.uint32))))
    return pairs, mat, lbar, np.array(recs, np.uint32).reshape(-1, 4)


def _population(n=6, seed=3):
    els = robots.population("uneven", n)
    b = mb.pack(els)
    rng = np.random.default_rng(seed)
    pos = b.pos.copy()
    pos[:, :3] += rng.normal(0, 0.01, (b.n_masses, 3)).astype(np.float32)
    stress = rng.normal(0, 1, b.n_springs).astype(np.float32)
    # ties, signed zeros
    stress[::7] = 0.5
    stress[1::11] = 0.0
    stress[2::13] = -0.0
    return b, pos, stress


@pytest.mark.parametrize("flags", [0, core.DEVO_REFERENCE_RANKS])
def test_oracle_devo_matches_python_restatement(flags):
    b, pos, stress = _population()
    table = material_table()
    t = 0.123
    got = core.devo(b, pos, stress, table, t, 40, 17, flags)
    exp = py_devo(b, pos, stress, table, np.float32(t), 40, 17, flags)
    assert np.array_equal(got[3], exp[3])
    assert np.array_equal(got[0], exp[0])
    assert np.array_equal(got[1], exp[1])
    assert np.array_equal(got[2].view(np.uint32), exp[2].view(np.uint32))


def test_devo_replaces_the_highest_stresses():
    b, pos, stress = _population(8)
    table = material_table()
    k = 25
    pairs, mat, lbar, recs = core.devo(b, pos, stress, table, 0.5, k, 3)
    assert len(recs) == 8 * k
    for r in range(8):
        s0, s1 = int(b.spring_offsets[r]), int(b.spring_offsets[r + 1])
        rec = recs[r * k:(r + 1) * k]
        chosen = rec[:, 0].astype(np.int64) - s0
        assert ((chosen >= 0) & (chosen < s1 - s0)).all()
        st = stress[s0:s1]
        # rank order: descending stress (signed zeros equal), ties by index
        keys = [(-float(st[c]), int(c)) for c in chosen]
        assert keys == sorted(keys)
        others = np.setdiff1d(np.arange(s1 - s0), chosen)
        assert float(st[chosen].min()) >= float(st[others].max())
        a, c = rec[:, 1] & 0xFFFF, rec[:, 1] >> 16
        m = int(b.mass_offsets[r + 1] - b.mass_offsets[r])
        assert (a != c).all() and (a < m).all() and (c < m).all()
        m0 = int(b.mass_offsets[r])
        for (sp, pr, cid, lb), x, y in zip(rec, a, c):
            assert cid == composite_id(int(b.mass_material[m0 + x]), int(b.mass_material[m0 + y]))
            d = np.linalg.norm(pos[m0 + x, :3].astype(np.float64) - pos[m0 + y, :3])
            rc = table[cid, 1] * math.sin(table[cid, 2] * 0.5 + table[cid, 3])
            assert np.float32(lb).dtype == np.float32
            assert abs(np.uint32(lb).view(np.float32) - d / (1 + rc)) <= 1e-5 * d + 1e-12
    # untouched springs keep their topology
    untouched = np.ones(b.n_springs, bool)
    untouched[recs[:, 0]] = False
    assert np.array_equal(pairs[untouched], b.pairs[untouched])
    assert np.array_equal(mat[untouched], b.spring_material[untouched])
    assert np.array_equal(lbar[untouched], b.lbar[untouched])


def test_devo_is_deterministic_and_seeded():
    b, pos, stress = _population(4)
    table = material_table()
    x = core.devo(b, pos, stress, table, 0.0, 16, 5)
    y = core.devo(b, pos, stress, table, 0.0, 16, 5)
    z = core.devo(b, pos, stress, table, 0.0, 16, 6)
    assert np.array_equal(x[3], y[3])
    assert not np.array_equal(x[3][:, 1], z[3][:, 1])
    assert np.array_equal(x[3][:, 0], z[3][:, 0])  # same springs, other pairs


def test_devo_window_edges():
    b, pos, stress = _population(5)
    table = material_table()
    n = np.diff(b.spring_offsets)
    # k larger than a robot: every spring replaced
    big = int(n.max()) + 10
    *_, recs = core.devo(b, pos, stress, table, 0.0, big, 1)
    assert len(recs) == int(n.sum())
    # reference ranks: robot r gets ranks [r k, r k + k) clipped to its springs
    k = int(n.min()) // 2
    *_, recs = core.devo(b, pos, stress, table, 0.0, k, 1, core.DEVO_REFERENCE_RANKS)
    exp = sum(max(0, min(r * k + k, int(n[r])) - min(r * k, int(n[r]))) for r in range(5))
    assert len(recs) == exp
    # k = 0: nothing
    *_, recs = core.devo(b, pos, stress, table, 0.0, 0, 1)
    assert len(recs) == 0


def test_devo_skips_robots_with_one_mass():
    e = mb.Element(np.zeros((1, 3)), np.array([1]), np.zeros((1, 2)), np.ones(1), np.array([1]))
    big = robots.population("small", 1)[0]
    b = mb.pack([e, big])
    stress = np.arange(b.n_springs, dtype=np.float32)
    *_, recs = core.devo(b, b.pos, stress, material_table(), 0.0, 4, 1)
    assert len(recs) == 4 and (recs[:, 0] >= 1).all()


def test_devo_pairs_are_uniform():
    m = 6
    counts = np.zeros((m, m), np.int64)
    for j in range(6000):
        a, b = core.devo_pair(11, 0, j, m)
        counts[a, b] += 1
    assert np.trace(counts) == 0
    off = counts[~np.eye(m, dtype=bool)]
    exp = 6000 / (m * (m - 1))
    chi2 = float(((off - exp) ** 2 / exp).sum())
    assert chi2 < 70  # 29 degrees of freedom; p ~ 1e-5


def test_stress_key_order():
    vals = [float("-inf"), -2.0, -1e-30, -0.0, 0.0, 1e-30, 3.0, float("inf")]
    keys = [core.stress_key(v) for v in vals]
    assert keys == sorted(keys, reverse=True)
    assert core.stress_key(-0.0) == core.stress_key(0.0)
