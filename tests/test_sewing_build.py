"""Sewing in the host-side builder (no GPU): sewing constraints and their
colouring, seam-gated bending, the sewing-extended adjacency, the two-hop
rest lengths of the contracted mesh and the open-boundary bits.

* The reference's own mesh tests for sewing
  (crates/cloth_core/src/mesh.rs:1671-1704, :1859-1909, :1995-2200) restated
  against both the product (tc_mesh_build_sewn) and the oracle.
* The product against the oracle, bit for bit, on a sewn garment (two panels
  sewn along both sides).
"""
import numpy as np
import pytest

from hostbuild import host_build
from taremincloth_b200 import scenes


def _builds(oracle_lib, **kw):
    o = oracle_lib.OracleSim(**kw)
    h = host_build(**kw)
    return o, h


def _two_hop(topo, a, b):
    """Rest length recorded for the pair (a, b), or None when b is not in a's two-hop set."""
    o, e = topo["th_off"][a], topo["th_off"][a + 1]
    hit = np.nonzero(topo["th_idx"][o:e] == b)[0]
    return None if len(hit) == 0 else float(topo["th_rest"][o + hit[0]])


def _adj(topo, v):
    return set(topo["adj_idx"][topo["adj_off"][v]:topo["adj_off"][v + 1]].tolist())


def test_sewing_shares_neighbours_of_the_sewn_pair(oracle_lib):
    """mesh.rs:1671-1704: edges 0-1 and 2-3, 1 sewn to 2: vertex 1 also
    neighbours 3, vertex 2 also neighbours 0."""
    pos = np.array([[0, 0, 0], [1, 0, 0], [2, 0, 0], [3, 0, 0]], np.float32)
    kw = dict(positions=pos, edges=np.array([[0, 1], [2, 3]]), sewing_springs=np.array([[1, 2]]))
    o, h = _builds(oracle_lib, **kw)
    for topo in (o.topology(), h):
        assert {0, 2, 3} <= _adj(topo, 1)
        assert {0, 1, 3} <= _adj(topo, 2)


def test_two_hop_rest_lengths_of_strand_seams(oracle_lib):
    """mesh.rs:1859-1909: direct, sewn and strand pairs are always excluded (rest 0)."""
    pos = np.array([[0, 0, 0], [0.1, 0, 0], [1.0, 0, 0], [1.1, 0, 0]], np.float32)
    kw = dict(positions=pos, edges=np.array([[0, 1], [2, 3]]), sewing_springs=np.array([[1, 2]]))
    o, h = _builds(oracle_lib, **kw)
    for topo in (o.topology(), h):
        assert _two_hop(topo, 0, 1) == 0.0
        for b in (2, 3):
            assert _two_hop(topo, 0, b) in (None, 0.0)
        assert _two_hop(topo, 1, 0) == 0.0
        assert _two_hop(topo, 1, 2) in (None, 0.0)


def test_seam_gated_bending_across_sewn_panels(oracle_lib):
    """mesh.rs:1995-2050: one bending constraint across the seam between the
    opposite vertices 2 and 5, rest = the unfolded distance 2.0 (not the 3D
    distance 7.0), seam-gated with gate 1.0."""
    pos = np.array([[0, 0, 0], [0, 1, 0], [-1, 0.5, 0], [5, 0, 0], [5, 1, 0], [6, 0.5, 0]], np.float32)
    edges = np.array([[0, 1], [1, 2], [2, 0], [3, 4], [4, 5], [5, 3]])
    faces = np.array([[0, 1, 2], [4, 3, 5]])
    kw = dict(positions=pos, edges=edges, faces=faces, sewing_springs=np.array([[0, 3], [1, 4]]), stiffness=1000.0,
              compression_stiffness=1000.0, shear_stiffness=1000.0)
    o, h = _builds(oracle_lib, **kw)
    ob = o.bending_constraints()
    for v, rest, kind, gate in ((ob["v"], ob["rest"], ob["pad0"], ob["pad1"]),
                                (h["bend_v"], h["bend_par"][:, 0], h["bend_par"][:, 2], h["bend_par"][:, 3])):
        assert len(v) == 1
        assert (min(v[0][2], v[0][3]), max(v[0][2], v[0][3])) == (2, 5)
        assert abs(rest[0] - 2.0) < 1e-5 and kind[0] > 0.5 and abs(gate[0] - 1.0) < 1e-5
    np.testing.assert_array_equal(ob["v"], h["bend_v"])
    np.testing.assert_array_equal(ob["rest"], h["bend_par"][:, 0])


def test_seam_unfolded_two_hop_and_boundary_bits(oracle_lib):
    """mesh.rs:2052-2139: sewn and contracted-adjacent pairs rest 0; the pair
    2-6 across the seam gets the unfolded rest 2.0, the same both ways; the
    seam edges and the inner diagonals are not open boundary, the outer
    edges are."""
    pos = np.array([[0, 1, 0], [0, 0, 0], [-1, 1, 0], [-1, 0, 0], [10, 1, 0], [10, 0, 0], [11, 1, 0], [11, 0, 0]],
                   np.float32)
    edges = np.array([[0, 1], [0, 2], [1, 2], [1, 3], [2, 3], [4, 5], [4, 6], [5, 6], [5, 7], [6, 7]])
    faces = np.array([[0, 2, 1], [1, 2, 3], [4, 5, 6], [5, 7, 6]])
    kw = dict(positions=pos, edges=edges, faces=faces, sewing_springs=np.array([[0, 4], [1, 5]]))
    o, h = _builds(oracle_lib, **kw)
    oe, obits = o.edges()
    for topo, e, bits in ((o.topology(), oe, obits), (h, h["edges"], h["edge_bits"])):
        for a, b in ((0, 4), (4, 0), (1, 5), (5, 1), (0, 5), (4, 1)):
            assert _two_hop(topo, a, b) == 0.0, (a, b)
        d26, d62 = _two_hop(topo, 2, 6), _two_hop(topo, 6, 2)
        assert abs(d26 - 2.0) < 1e-4 and d26 == d62
        for k, (a, b) in enumerate(e):
            open_ = (int(bits[k >> 5]) >> (k & 31)) & 1
            inner = (min(a, b), max(a, b)) in {(0, 1), (4, 5), (1, 2), (5, 6)}
            assert open_ == (0 if inner else 1), (a, b)


def test_point_seam_slit_two_hop(oracle_lib):
    """mesh.rs:2141-2200: a single sewn point joins two triangles; the pair
    1-4 across it gets the summed edge lengths 2.0, the same both ways."""
    pos = np.array([[0, 0, 0], [0, 1, 0], [-1, 0, 0], [5, 0, 0], [5, 1, 0], [6, 0, 0]], np.float32)
    edges = np.array([[0, 1], [1, 2], [2, 0], [3, 4], [4, 5], [5, 3]])
    faces = np.array([[0, 1, 2], [3, 4, 5]])
    o, h = _builds(oracle_lib, positions=pos, edges=edges, faces=faces, sewing_springs=np.array([[0, 3]]))
    for topo in (o.topology(), h):
        d14, d41 = _two_hop(topo, 1, 4), _two_hop(topo, 4, 1)
        assert abs(d14 - 2.0) < 1e-4 and d14 == d41


@pytest.mark.parametrize("n", [8, 24])
def test_sewn_garment_build_matches_oracle(oracle_lib, n):
    """Every built array of a sewn garment, product against oracle, bit for bit."""
    sc = scenes.sewn_garment(n=n)
    kw = dict(positions=sc["positions"], edges=sc["edges"], faces=sc["faces"], inv_masses=sc["inv_masses"],
              thickness=sc["thickness"], sewing_springs=sc["sewing"], sewing_shrink_speed=sc["sewing_shrink_speed"])
    o, h = _builds(oracle_lib, **kw)
    c = o.counts()
    for k in ["nd", "nb", "n_dist_colors", "n_bend_colors", "n_edges", "table_size", "num_virtual", "multi_layer"]:
        assert c[k] == h[k], k
    d, b, col = o.distance_constraints(), o.bending_constraints(), o.colors()
    np.testing.assert_array_equal(d["v"], h["dist_v"])
    np.testing.assert_array_equal(d["rest"], h["dist_par"][:, 0])
    np.testing.assert_array_equal(b["v"], h["bend_v"])
    for k, j in (("rest", 0), ("comp", 1), ("pad0", 2), ("pad1", 3)):
        np.testing.assert_array_equal(b[k], h["bend_par"][:, j], err_msg=k)
    assert int((b["pad0"] == 1.0).sum()) == 2 * (n - 1)  # one seam constraint per sewn quad row and side
    for k in ["dist_off", "dist_cnt", "bend_off", "bend_cnt"]:
        np.testing.assert_array_equal(col[k], h[k], err_msg=k)
    s = o.sewing()
    np.testing.assert_array_equal(s["v"], h["sew_v"])
    np.testing.assert_array_equal(s["cur"], h["sew_par"][:, 0])
    np.testing.assert_array_equal(s["off"], h["sew_off"])
    np.testing.assert_array_equal(s["cnt"], h["sew_cnt"])
    np.testing.assert_array_equal(s["rep"], h["sew_rep"])
    assert len(h["sew_v"]) == 2 * n and np.all(h["sew_par"][:, 2] == np.float32(sc["sewing_shrink_speed"]))
    t = o.topology()
    for k in ["adj_off", "adj_idx", "th_off", "th_idx", "th_rest", "local_len", "star_off", "star_idx", "island",
              "layer"]:
        np.testing.assert_array_equal(t[k], h[k], err_msg=k)
    e, bits = o.edges()
    np.testing.assert_array_equal(e, h["edges"])
    np.testing.assert_array_equal(bits, h["edge_bits"])
    # the sewn panels form one island, and each side seam closes a tube
    assert len(np.unique(h["island"])) == 1


def test_sewing_colouring_is_conflict_free():
    sc = scenes.sewn_garment(n=24)
    h = host_build(positions=sc["positions"], edges=sc["edges"], faces=sc["faces"], sewing_springs=sc["sewing"])
    for o, c in zip(h["sew_off"], h["sew_cnt"]):
        verts = h["sew_v"][o:o + c].reshape(-1)
        assert len(np.unique(verts)) == len(verts)
