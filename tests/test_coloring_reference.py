"""Welsh-Powell colourings against the reference's own Python colouring.

tests/golden/coloring.npz holds pair lists and the colours that the
reference's log tool gave them (python/taremin_cloth/log_tools.py:609-636,
the in-tree twin of crates/cloth_core/src/coloring.rs:6-79, :180-233 and
:236-300); tests/golden/make_coloring_fixtures.py made it.  Checked here,
without a GPU:
* the host entry point color_edge_pairs (tc_color_edge_pairs) gives the
  same colour to every pair;
* the topology builder's distance colouring of an edges-only mesh and its
  sewing colouring give the same colour classes: class c holds the pairs of
  colour c in their input order, and the classes are stored in colour order.
"""
import os

import numpy as np
import pytest

from hostbuild import host_build
from taremincloth_b200 import simulator as core

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "coloring.npz")


def _cases():
    d = np.load(GOLDEN)
    names = sorted({k.split("/")[0] for k in d.files})
    return {k: (int(d[f"{k}/n"]), d[f"{k}/pairs"], str(d[f"{k}/kind"]), d[f"{k}/colors"]) for k in names}


CASES = _cases()


def _classes(pairs, colors):
    """(pairs in colour order, input order inside a colour, offsets, counts)."""
    k = int(colors.max()) + 1 if len(colors) else 0
    rows = [pairs[colors == c] for c in range(k)]
    cnt = np.array([len(r) for r in rows], np.uint32)
    off = np.concatenate([[0], np.cumsum(cnt)[:-1]]).astype(np.uint32)
    return np.concatenate(rows), off, cnt


def _grid(nx, ny, dx, x0=0.0):
    return np.array([[x0 + ix * dx, iy * dx, 0.0] for iy in range(ny) for ix in range(nx)], np.float32)


def _grid_edges(nx, ny, base=0):
    out = []
    for iy in range(ny):
        for ix in range(nx):
            v = base + iy * nx + ix
            if ix + 1 < nx:
                out.append((v, v + 1))
            if iy + 1 < ny:
                out.append((v, v + nx))
            if ix + 1 < nx and iy + 1 < ny:
                out.append((v, v + nx + 1))
    return np.array(out, np.uint32)


def test_fixture_cases_present():
    assert set(CASES) == {"grid_distance", "random_distance", "two_sheet_sewing", "random_pairs", "hub_pairs"}
    for n, pairs, kind, col in CASES.values():
        assert len(col) == len(pairs) > 0


@pytest.mark.parametrize("name", sorted(CASES))
def test_color_edge_pairs_matches_reference(name):
    n, pairs, _, col = CASES[name]
    assert core.color_edge_pairs(n, pairs) == col.tolist()


@pytest.mark.parametrize("name", ["grid_distance", "random_distance"])
def test_distance_colouring_matches_reference(name):
    n, pairs, kind, col = CASES[name]
    assert kind == "distance"
    pos = np.random.default_rng(7).random((n, 3)).astype(np.float32)
    got = host_build(pos, pairs)
    want_v, want_off, want_cnt = _classes(pairs, col)
    np.testing.assert_array_equal(got["dist_v"], want_v)
    np.testing.assert_array_equal(got["dist_off"], want_off)
    np.testing.assert_array_equal(got["dist_cnt"], want_cnt)


def test_sewing_colouring_matches_reference():
    n, pairs, kind, col = CASES["two_sheet_sewing"]
    assert kind == "sewing" and n == 72
    pos = np.concatenate([_grid(6, 6, 0.01), _grid(6, 6, 0.01, 0.06)])
    edges = np.concatenate([_grid_edges(6, 6), _grid_edges(6, 6, 36)])
    got = host_build(pos, edges, sewing_springs=pairs)
    want_v, want_off, want_cnt = _classes(pairs, col)
    np.testing.assert_array_equal(got["sew_v"], want_v)
    np.testing.assert_array_equal(got["sew_off"], want_off)
    np.testing.assert_array_equal(got["sew_cnt"], want_cnt)
