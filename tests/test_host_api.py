"""Host-only entry points of the drop-in module, on the CPU (no device):
compute_combined_inv_masses / compute_areal_inv_masses (a2; mesh.rs:237-312,
lib.rs:553-640) and color_edge_pairs (coloring.rs:180-233, lib.rs:642-652).

Pinned against the reference's own tests (mesh.rs:1795-1830, :1916-1948,
tests/core/test_geometry_public_api.py) and against restatements written
here: a float32 loop in the reference's operation order for the masses
(bit-exact), and a plain Welsh-Powell for the colours (equal lists).
"""
import numpy as np
import pytest

import taremin_cloth_core as core


def _masses_f32(pos, faces, strands, pins, areal, linear):
    f32 = np.float32
    n = len(pos)
    m = np.zeros(n, f32)
    if areal > 0 and faces is not None:
        for a, b, c in faces:
            if a >= n or b >= n or c >= n or a == b or b == c or c == a:
                continue
            ab, ac = pos[b] - pos[a], pos[c] - pos[a]
            cr = np.array([ab[1] * ac[2] - ab[2] * ac[1], ab[2] * ac[0] - ab[0] * ac[2],
                           ab[0] * ac[1] - ab[1] * ac[0]], f32)
            area = f32(0.5) * np.sqrt(f32(f32(cr[0] * cr[0] + cr[1] * cr[1]) + cr[2] * cr[2]))
            share = f32(f32(area * f32(areal)) / f32(3.0))
            m[a] += share; m[b] += share; m[c] += share
    if linear > 0 and strands is not None:
        for a, b in strands:
            if a >= n or b >= n or a == b:
                continue
            d = pos[a] - pos[b]
            ln = np.sqrt(f32(f32(d[0] * d[0] + d[1] * d[1]) + d[2] * d[2]))
            share = f32(f32(ln * f32(linear)) / f32(2.0))
            m[a] += share; m[b] += share
    w = np.zeros(n, f32)
    for i in range(n):
        p = f32(pins[i]) if pins is not None and i < len(pins) else f32(0)
        p = min(max(p, f32(0)), f32(1))
        w[i] = f32(0) if p >= 1 else f32(f32(1) - p) / max(m[i], f32(1e-9))
    return w


def test_combined_areal_and_linear():
    """mesh.rs:1916-1948"""
    pos = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 2, 0], [0, 3, 0]], np.float32)
    inv = core.compute_combined_inv_masses(pos, np.array([[0, 1, 2]], np.uint32),
                                           np.array([[2, 3], [3, 4]], np.uint32), None, 0.30, 0.02)
    assert inv.shape == (5,)
    assert abs(inv[0] - 20.0) < 1e-4 and abs(inv[1] - 20.0) < 1e-4
    assert abs(inv[2] - 1.0 / 0.06) < 1e-3
    assert abs(inv[3] - 50.0) < 1e-4 and abs(inv[4] - 100.0) < 1e-3


def test_areal_physical_units_and_pins():
    """mesh.rs:1795-1830 and test_geometry_public_api.py (edge cases)"""
    pos = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0]], np.float32)
    faces = np.array([[0, 1, 2], [0, 2, 3]], np.uint32)
    inv = core.compute_areal_inv_masses(pos, faces, None, 0.15)
    m = 1.0 / inv
    assert abs(m.sum() - 0.15) < 1e-5 and m[0] > m[1] and abs(m[1] - m[3]) < 1e-7
    pinned = core.compute_areal_inv_masses(pos, faces, np.array([1.0, 0, 0, 0], np.float32), 0.15)
    assert pinned[0] == 0.0 and pinned[1] > 0
    bare = core.compute_areal_inv_masses(pos, None, None, 0.15)
    assert np.all(np.isfinite(bare)) and np.all(bare > 0)
    z = np.zeros((3, 3), np.float32)
    assert np.all(np.isfinite(core.compute_areal_inv_masses(z, None, None, 0.15)))
    got = core.compute_areal_inv_masses(z, np.array([[0, 1, 2]], np.uint32), np.array([1.0, 0, 0], np.float32), 0.15)
    assert got[0] == 0.0


@pytest.mark.parametrize("seed", range(4))
def test_masses_bit_exact_against_restatement(seed):
    rng = np.random.default_rng(seed)
    n = 60
    pos = rng.normal(size=(n, 3)).astype(np.float32)
    faces = rng.integers(0, n + 3, size=(80, 3)).astype(np.uint32)   # some out of range / degenerate
    strands = rng.integers(0, n, size=(25, 2)).astype(np.uint32)
    pins = rng.uniform(-0.5, 1.5, size=n - 7).astype(np.float32)      # shorter than n: the rest count as 0
    got = core.compute_combined_inv_masses(pos, faces, strands, pins, 0.2, 0.05)
    want = _masses_f32(pos, faces.astype(np.int64), strands.astype(np.int64), pins, 0.2, 0.05)
    np.testing.assert_array_equal(got, want)


def _welsh_powell(n, edges):
    v2c = [[] for _ in range(n)]
    for i, (a, b) in enumerate(edges):
        if a < n:
            v2c[a].append(i)
        if b < n:
            v2c[b].append(i)
    deg = lambda v: len(v2c[v]) if v < n else 0
    order = sorted(range(len(edges)), key=lambda i: (-(deg(edges[i][0]) + deg(edges[i][1])), i))
    col = [None] * len(edges)
    for i in order:
        used = {col[j] for v in edges[i] if v < n for j in v2c[v] if j != i and col[j] is not None}
        c = 0
        while c in used:
            c += 1
        col[i] = c
    return col


def test_color_edge_pairs():
    rng = np.random.default_rng(1)
    for _ in range(5):
        n, m = 30, 60
        a, b = rng.integers(0, n, size=m), rng.integers(0, n, size=m)
        keep = a != b
        e = np.stack([np.minimum(a, b), np.maximum(a, b)], 1)[keep].astype(np.uint32)
        got = core.color_edge_pairs(n, e)
        assert got == _welsh_powell(n, e.tolist())
        by_v = {}
        for i, (x, y) in enumerate(e.tolist()):
            by_v.setdefault(x, []).append(got[i])
            by_v.setdefault(y, []).append(got[i])
        assert all(len(c) == len(set(c)) for c in by_v.values())
    assert core.color_edge_pairs(10, np.empty((0, 2), np.uint32)) == []
    # out-of-range ends register nothing; no vertices: all colour 0
    assert core.color_edge_pairs(3, np.array([[0, 1], [1, 9], [0, 9]], np.uint32)) == _welsh_powell(3, [[0, 1], [1, 9], [0, 9]])
    assert core.color_edge_pairs(0, np.array([[0, 1], [1, 2]], np.uint32)) == [0, 0]
