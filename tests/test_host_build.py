"""The product's host-side builder (libtcloth.so, tc_mesh_*) against the oracle.

Constraints, their Welsh-Powell colouring, the topology CSRs, the Morton-sorted
edge list, boundary bits and hash sizing must be bit-exact.  Runs without a GPU.
Also restates the reference's mesh unit tests (crates/cloth_core/src/mesh.rs:1574-1994).
"""
import numpy as np
import pytest

import golden_cases as gc
from hostbuild import host_build
from taremincloth_b200 import scenes


def _inputs(name):
    if name.startswith("case"):
        c, d, pos, inv = gc.load(name)
        return dict(positions=pos, edges=d["edges"], faces=d["faces"], inv_masses=inv, thickness=0.005,
                    stiffness=c["stiffness"], bending_stiffness=c["bending"])
    if name == "config1":
        s = scenes.config1()
        return dict(positions=s["positions"], edges=s["edges"], faces=s["faces"], inv_masses=s["inv_masses"],
                    thickness=0.005)
    if name == "config2":
        s = scenes.config2()
        return dict(positions=s["positions"], edges=s["edges"], faces=s["faces"], inv_masses=s["inv_masses"],
                    layer_ids=s["layer_ids"], thickness=0.002)
    if name == "config2_small":
        s = scenes.config2(n=48, subdiv=3)
        return dict(positions=s["positions"], edges=s["edges"], faces=s["faces"], inv_masses=s["inv_masses"],
                    layer_ids=s["layer_ids"], thickness=0.002)
    if name == "islands":
        p, e, f, _ = scenes.tri_grid(8, 0.2, 0.0)
        q, e2, f2, _ = scenes.tri_grid(8, 0.2, 0.01, 64)
        return dict(positions=np.concatenate([p, q + np.array([0, 0, 0.05], np.float32)]),
                    edges=np.concatenate([e, e2]), faces=np.concatenate([f, f2]))
    raise KeyError(name)


@pytest.mark.parametrize("name", ["case1", "case2", "case3", "case4", "config1", "config2", "config2_small",
                                  "islands"])
def test_host_build_matches_oracle(oracle_lib, name):
    kw = _inputs(name)
    o = oracle_lib.OracleSim(**kw)
    h = host_build(**kw)
    c = o.counts()
    for k in ["nd", "nb", "n_dist_colors", "n_bend_colors", "n_edges", "table_size", "num_virtual", "multi_layer"]:
        assert c[k] == h[k], k
    d, b, col = o.distance_constraints(), o.bending_constraints(), o.colors()
    np.testing.assert_array_equal(d["v"], h["dist_v"])
    np.testing.assert_array_equal(d["rest"], h["dist_par"][:, 0])
    np.testing.assert_array_equal(d["tc"], h["dist_par"][:, 1])
    np.testing.assert_array_equal(d["cc"], h["dist_par"][:, 2])
    np.testing.assert_array_equal(d["type"], h["dist_par"][:, 3].astype(np.uint32))
    np.testing.assert_array_equal(b["v"], h["bend_v"])
    np.testing.assert_array_equal(b["rest"], h["bend_par"][:, 0])
    np.testing.assert_array_equal(b["comp"], h["bend_par"][:, 1])
    for k in ["dist_off", "dist_cnt", "bend_off", "bend_cnt"]:
        np.testing.assert_array_equal(col[k], h[k], err_msg=k)
    t = o.topology()
    for k in ["adj_off", "adj_idx", "th_off", "th_idx", "th_rest", "local_len", "star_off", "star_idx", "island",
              "layer"]:
        np.testing.assert_array_equal(t[k], h[k], err_msg=k)
    e, bits = o.edges()
    np.testing.assert_array_equal(e, h["edges"])
    np.testing.assert_array_equal(bits, h["edge_bits"])
    assert o.cell_size() == h["cell"]


def _conflict_free(v, off, cnt):
    for o, c in zip(off, cnt):
        verts = v[o:o + c].reshape(-1)
        assert len(np.unique(verts)) == len(verts)


@pytest.mark.parametrize("name", ["config1", "config2"])
def test_colouring_is_conflict_free(name):
    """Independent check: no two constraints of one colour share a vertex."""
    h = host_build(**_inputs(name))
    _conflict_free(h["dist_v"], h["dist_off"], h["dist_cnt"])
    _conflict_free(h["bend_v"][:, 2:], h["bend_off"], h["bend_cnt"])
    assert int(h["dist_cnt"].sum()) == h["nd"] and int(h["bend_cnt"].sum()) == h["nb"]


def test_config_counts():
    """Constraint counts of the two benchmark shapes."""
    h1 = host_build(**_inputs("config1"))
    assert (h1["n"], h1["nd"], h1["nb"]) == (8065, 31878, 7812)
    h2 = host_build(**_inputs("config2"))
    assert (h2["n"], h2["nd"], h2["nb"]) == (131072, 521220, 259080)
    assert h2["cell"] == pytest.approx(0.01) and h2["table_size"] == 65536


def test_mesh_topology_and_star_pairs():
    """mesh.rs:1574-1648"""
    pos = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [1, 1, 0]], np.float32)
    h = host_build(pos, np.array([[0, 1], [1, 2], [2, 0], [1, 3], [3, 2]]), np.array([[0, 1, 2], [2, 1, 3]]),
                   stiffness=1000.0, bending_stiffness=10.0, shear_stiffness=1000.0)
    assert list(h["adj_idx"][h["adj_off"][0]:h["adj_off"][1]]) == [1, 2]
    assert list(h["adj_idx"][h["adj_off"][1]:h["adj_off"][2]]) == [0, 2, 3]
    assert h["star_off"][1] - h["star_off"][0] == 1
    assert list(h["star_idx"][h["star_off"][0]]) == [1, 2]
    assert h["star_off"][2] - h["star_off"][1] == 2
    assert list(h["island"]) == [0, 0, 0, 0]


def test_multiple_disconnected_islands():
    """mesh.rs:1651-1668"""
    pos = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [10, 0, 0], [11, 0, 0], [10, 1, 0]], np.float32)
    e = np.array([[0, 1], [1, 2], [2, 0], [3, 4], [4, 5], [5, 3]])
    h = host_build(pos, e, np.array([[0, 1, 2], [3, 4, 5]]))
    assert list(h["island"]) == [0, 0, 0, 1, 1, 1]


def test_two_hop_topology_csr():
    """mesh.rs:1706-1753"""
    pos = np.array([[i, 0, 0] for i in range(5)], np.float32)
    h = host_build(pos, np.array([[0, 1], [1, 2], [2, 3], [3, 4]]))
    get = lambda v: list(h["th_idx"][h["th_off"][v]:h["th_off"][v + 1]])
    assert get(0) == [0, 1, 2] and get(1) == [0, 1, 2, 3] and get(2) == [0, 1, 2, 3, 4]
    assert get(3) == [1, 2, 3, 4] and get(4) == [2, 3, 4]
    assert abs(h["th_rest"][0]) < 1e-6


def test_strand_1d_bending_constraints():
    """mesh.rs:1951-1993"""
    pos = np.array([[i, 0, 0] for i in range(4)], np.float32)
    h = host_build(pos, np.array([[0, 1], [1, 2], [2, 3]]))
    assert h["nb"] == 2
    pairs = {tuple(sorted(v[2:])) for v in h["bend_v"]}
    assert pairs == {(0, 2), (1, 3)}
    assert np.allclose(h["bend_par"][:, 0], 2.0)


def test_quad_shear_and_bending_disjoint():
    """crates/cloth_core/src/simulation/tests.rs:2333-2412: a triangulated quad
    gets shear on its diagonal pair and no bending across the diagonal."""
    pos = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0]], np.float32)
    h = host_build(pos, np.array([[0, 1], [1, 2], [2, 3], [3, 0]]), np.array([[0, 1, 2], [0, 2, 3]]))
    shear = {tuple(v) for v, p in zip(h["dist_v"], h["dist_par"]) if p[3] == 1}
    assert shear == {(0, 2), (1, 3)}
    assert h["nb"] == 0


def test_invalid_index_raises_value_error():
    pos = np.zeros((3, 3), np.float32)
    with pytest.raises(ValueError):
        host_build(pos, np.array([[0, 5]]))
    with pytest.raises(ValueError):
        host_build(pos, np.array([[0, 1]]), np.array([[0, 1, 7]]))


def test_empty_mesh():
    h = host_build(np.zeros((0, 3), np.float32), np.zeros((0, 2), np.uint32))
    assert h["n"] == 0 and h["nd"] == 0 and h["nb"] == 0


def test_union_colouring_equals_instance_colourings():
    """Batching relies on this: Welsh-Powell over a disjoint union of meshes
    gives every constraint the colour it gets in its own mesh."""
    sc = scenes.config4(n_instances=6, seed=3, side_range=(6, 20))
    insts = sc["instances"]
    off = np.concatenate([[0], np.cumsum([len(i["positions"]) for i in insts])])
    union = host_build(np.concatenate([i["positions"] for i in insts]),
                       np.concatenate([i["edges"] + off[k] for k, i in enumerate(insts)]),
                       np.concatenate([i["faces"] + off[k] for k, i in enumerate(insts)]),
                       layer_ids=np.zeros(off[-1], np.uint32))
    ucol = np.repeat(np.arange(len(union["dist_cnt"])), union["dist_cnt"])
    for k, inst in enumerate(insts):
        h = host_build(inst["positions"], inst["edges"], inst["faces"])
        icol = np.repeat(np.arange(len(h["dist_cnt"])), h["dist_cnt"])
        mine = (union["dist_v"][:, 0] >= off[k]) & (union["dist_v"][:, 0] < off[k + 1])
        np.testing.assert_array_equal(union["dist_v"][mine] - off[k], h["dist_v"])
        np.testing.assert_array_equal(ucol[mine], icol)
