"""Contact-pair cache ("Active Pair Caching", self-collision algorithm 1) on the GPU.

* Against the oracle, two stacked sheets over an icosphere (config 2 shape,
  48 x 48 per sheet): the stored vertex-triangle and edge-edge pairs of the
  broad phase and its accepted / dropped counts bit-exact, and positions
  within 1e-5 of the extent per frame, with the final fallback on (last
  substep direct) and off (every substep from the cache), quota 8 and 2,
  persistent and per-colour solver paths.
* The reference's tests (crates/cloth_core/src/simulation/tests.rs:128-145,
  :2061-2195, :2734-2780): enabling mid-simulation, a pinned lower layer
  pushing the upper layer out, and an edge-edge CCD stop of a high-speed
  crossing with the pair cache on.
"""
import numpy as np
import pytest

from gpu_common import compare_frames, extent
from taremincloth_b200 import ClothSimulator, scenes

pytestmark = pytest.mark.gpu


def _pair_sets(vt, ee):
    return np.asarray(vt, np.uint32).reshape(-1, 4), np.asarray(ee, np.uint32).reshape(-1, 4)


@pytest.mark.parametrize("fallback,max_pairs,persistent", [(True, None, True), (False, None, False),
                                                          (False, 9216, True), (True, 9216, False)])
def test_pair_cache_matches_oracle(oracle_lib, fallback, max_pairs, persistent):
    sc = scenes.config2(n=48, subdiv=3)
    g = scenes.build(ClothSimulator, sc)
    o = scenes.build(oracle_lib.OracleSim, sc)
    g.set_persistent_solver(persistent)
    g.set_enable_pair_cache(True)
    g.set_enable_pair_cache_final_fallback(fallback)
    o.set_pair_cache(True, fallback)
    if max_pairs is not None:
        g.set_pair_cache_options(max_pairs, max_pairs)
        o.set_pair_cache_options(max_pairs, max_pairs)
        assert g.get_pair_cache_stats()[2:] == (max_pairs, max_pairs)
    ext = extent(sc["positions"])
    for frame in range(6):
        worst, same = compare_frames(g, o, 1, sc["dt"], sc["substeps"], ext)
        assert worst.max() <= 1e-5, (frame, worst, same)
        gvt_n, gee_n, gvt, gee = g.get_active_pairs()
        ovt_n, oee_n, ovt, oee = o.active_pairs()
        gvt, gee = _pair_sets(gvt, gee)
        assert (gvt_n, gee_n) == (ovt_n, oee_n), frame
        np.testing.assert_array_equal(gvt, ovt)
        np.testing.assert_array_equal(gee, oee)
    assert len(gvt) > 0 and len(gee) > 0
    # every stored pair names four distinct vertices; V-T triangles start at their smallest id
    assert (gvt[:, 1] < gvt[:, 2]).all() and (gvt[:, 1] < gvt[:, 3]).all()
    assert (gee[:, 2] < gee[:, 3]).all()


def _by_vertex(pairs):
    d = {}
    for p in np.asarray(pairs, np.uint32).reshape(-1, 4):
        d.setdefault(int(p[0]), []).append(tuple(int(x) for x in p[1:]))
    return d


def test_pair_cache_quota_keeps_nearest():
    """The broad phase runs once, at the first substep, where both runs hold
    the same positions: each vertex's quota-2 list is the head of its
    quota-8 list (top-K by distance, then key)."""
    sc = scenes.config2(n=48, subdiv=3)
    out = {}
    for mp in (36864, 9216):
        g = scenes.build(ClothSimulator, sc)
        g.set_enable_pair_cache(True)
        g.set_enable_pair_cache_final_fallback(False)
        g.set_pair_cache_options(mp, mp)
        g.step(sc["dt"], sc["substeps"])
        out[mp] = g.get_active_pairs()
    for k in (2, 3):
        big, small = _by_vertex(out[36864][k]), _by_vertex(out[9216][k])
        assert small and set(small) == set(big)
        for v, lst in small.items():
            assert lst == big[v][:2], v


def test_lazy_enable_mid_simulation():
    """tests.rs:128-145: enable and disable the pair cache between frames."""
    pos = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0]], np.float32)
    s = ClothSimulator(pos, np.array([[0, 1], [1, 2], [2, 3], [3, 0], [0, 2]]), np.array([[0, 1, 2], [0, 2, 3]]))
    s.set_enable_self_collision(True)
    s.set_enable_pair_cache(True)
    s.set_enable_edge_collision(True)
    s.step(1.0 / 60.0, 2)
    s.set_enable_edge_collision(False)
    s.set_enable_pair_cache(False)
    s.set_enable_self_collision(False)
    s.step(1.0 / 60.0, 2)
    x, _, _ = s.get_state()
    assert np.isfinite(x).all()
    s.set_self_collision_algorithm(1)
    assert s.get_enable_pair_cache() and s.get_self_collision_algorithm() == 1
    s.set_self_collision_algorithm(0)
    assert not s.get_enable_pair_cache()
    with pytest.raises(NotImplementedError):
        s.set_self_collision_algorithm(2)


def _two_layers(nx=8, ny=7, spacing=0.15):
    per = nx * ny
    pos, edges, faces, layers, inv = [], [], [], [], []
    for layer in range(2):
        z = 0.0 if layer == 0 else 0.005
        off = layer * per
        for iy in range(ny):
            for ix in range(nx):
                pos.append([ix * spacing, iy * spacing, z])
                layers.append(layer)
                inv.append(0.0 if layer == 0 else 1.0)
        for iy in range(ny):
            for ix in range(nx):
                v0 = off + iy * nx + ix
                if ix + 1 < nx:
                    edges.append([v0, v0 + 1])
                if iy + 1 < ny:
                    edges.append([v0, v0 + nx])
                if ix + 1 < nx and iy + 1 < ny:
                    edges.append([v0, v0 + nx + 1])
                    faces.append([v0, v0 + 1, v0 + nx + 1])
                    faces.append([v0, v0 + nx + 1, v0 + nx])
    return (np.array(pos, np.float32), np.array(edges), np.array(faces), np.array(layers, np.uint32),
            np.array(inv, np.float32), per)


def test_pinned_lower_layer_pushes_upper_layer(oracle_lib):
    """tests.rs:2061-2148: the upper layer (index >= 56), 5 mm over a pinned
    lower layer with 4 cm thickness, is pushed above 2 cm within one frame
    with the pair cache on; the oracle agrees."""
    pos, e, f, layers, inv, per = _two_layers()
    kw = dict(layer_ids=layers, inv_masses=inv, thickness=0.04, stiffness=10000.0, compression_stiffness=10000.0,
              shear_stiffness=5000.0, bending_stiffness=0.0)
    s = ClothSimulator(pos, e, f, **kw)
    o = oracle_lib.OracleSim(pos, e, f, **kw)
    for sim in (s, o):
        sim.set_enable_self_collision(True)
        sim.set_gravity(0.0, 0.0, 0.0)
    s.set_enable_pair_cache(True)
    o.set_pair_cache(True, True)
    s.step(1.0 / 60.0, 4)
    o.step(1.0 / 60.0, 4)
    x, _, _ = s.get_state()
    xo, _, _ = o.get_state()
    assert (x[per:, 2] > 0.02).sum() > per // 2
    assert np.abs(x.astype(np.float64) - xo).max() <= 1e-5 * extent(pos)
    # after switching the pair cache off the free layer falls under gravity
    s.set_enable_self_collision(False)
    s.set_enable_pair_cache(False)
    s.set_positions_and_velocities(pos, np.zeros_like(pos))
    s.set_gravity(0.0, 0.0, -9.81)
    s.step(1.0 / 60.0, 2)
    x2, _, _ = s.get_state()
    assert (x2[per:, 2] < pos[per:, 2] - 1e-4).all()


@pytest.mark.parametrize("fallback", [True, False])
def test_pair_cache_ee_ccd_blocks_high_speed_crossing(oracle_lib, fallback):
    """tests.rs:2734-2780: two crossing interior edges 6 mm apart, the upper
    pair moving at 0.9 m/s down for one substep, stay uncrossed.  With one
    substep the final fallback (default on) runs the direct pass, which stops
    the crossing.  With the fallback off the crossing pair is not in the cache
    (each endpoint of one edge sits two 2.5 cm cells from both endpoints of the
    other), as in the reference's broad phase, so only parity is checked."""
    z = 0.006
    pos = np.array([[-0.05, 0, 0], [0.05, 0, 0], [0, 0.03, -0.05], [0, -0.03, -0.05],
                    [0, -0.05, z], [0, 0.05, z], [0.03, 0, z + 0.05], [-0.03, 0, z + 0.05]], np.float32)
    e = np.array([[0, 1], [1, 2], [2, 0], [0, 3], [3, 1], [4, 5], [5, 6], [6, 4], [4, 7], [7, 5]])
    f = np.array([[0, 1, 2], [1, 0, 3], [4, 5, 6], [5, 4, 7]])
    kw = dict(thickness=0.005, stiffness=10000.0, compression_stiffness=10000.0, shear_stiffness=5000.0,
              bending_stiffness=0.0)
    vel = np.zeros_like(pos)
    vel[4:, 2] = -0.9
    s = ClothSimulator(pos, e, f, **kw)
    o = oracle_lib.OracleSim(pos, e, f, **kw)
    s.set_self_collision_algorithm(1)
    s.set_enable_pair_cache_final_fallback(fallback)
    o.set_pair_cache(True, fallback)
    s.set_positions_and_velocities(pos, vel)
    o.set_state(pos, vel)
    for sim in (s, o):
        sim.set_enable_self_collision(True)
        sim.set_gravity(0.0, 0.0, 0.0)
        sim.step(1.0 / 60.0, 1)
    x, _, _ = s.get_state()
    xo, _, _ = o.get_state()
    za, zb = 0.5 * (x[0, 2] + x[1, 2]), 0.5 * (x[4, 2] + x[5, 2])
    assert np.abs(x.astype(np.float64) - xo).max() <= 1e-6
    if fallback:
        assert zb >= za - 1e-4, (za, zb)
    else:
        _, _, _, ee = s.get_active_pairs()
        assert [0, 1, 4, 5] not in ee and len(ee) > 0


@pytest.mark.parametrize("case", ["sewn", "intervals"])
def test_pair_cache_with_sewing_and_intervals(oracle_lib, case):
    """The pair cache over a sewn garment (sewing-contracted topology, seams
    closing), and with self-collision every 3rd substep and no edge-edge pass:
    pairs, counters and positions against the oracle."""
    if case == "sewn":
        sc = scenes.sewn_garment(n=24)
    else:
        sc = scenes.config2(n=32, subdiv=2)
    g = scenes.build(ClothSimulator, sc)
    o = scenes.build(oracle_lib.OracleSim, sc)
    g.set_enable_pair_cache(True)
    g.set_enable_pair_cache_final_fallback(False)
    o.set_pair_cache(True, False)
    if case == "intervals":
        for sim in (g, o):
            sim.set_self_collision_substep_interval(3)
            sim.set_self_collision_ee_substep_interval(0)
    ext = extent(sc["positions"])
    for frame in range(4):
        worst, same = compare_frames(g, o, 1, sc["dt"], sc["substeps"], ext)
        assert worst.max() <= 1e-5, (frame, worst, same)
        gvt_n, gee_n, gvt, gee = g.get_active_pairs()
        ovt_n, oee_n, ovt, oee = o.active_pairs()
        gvt, gee = _pair_sets(gvt, gee)
        assert (gvt_n, gee_n) == (ovt_n, oee_n), frame
        np.testing.assert_array_equal(gvt, ovt)
        np.testing.assert_array_equal(gee, oee)


def test_pair_cache_600_substeps_within_tolerance(oracle_lib):
    """600 substeps (30 frames x 20) with the pair cache on: positions within
    1e-4 of the extent of the oracle's, and the stored pairs equal at the end."""
    sc = scenes.config2(n=48, subdiv=3)
    g = scenes.build(ClothSimulator, sc)
    o = scenes.build(oracle_lib.OracleSim, sc)
    g.set_enable_pair_cache(True)
    o.set_pair_cache(True, True)
    worst, same = compare_frames(g, o, 30, sc["dt"], sc["substeps"], extent(sc["positions"]), 1e-4)
    assert worst.max() <= 1e-4, (worst.max(), same.min())
    _, _, gvt, gee = g.get_active_pairs()
    _, _, ovt, oee = o.active_pairs()
    gvt, gee = _pair_sets(gvt, gee)
    np.testing.assert_array_equal(gvt, ovt)
    np.testing.assert_array_equal(gee, oee)


def test_pair_cache_options_and_empty_state():
    """Option clamps (simulation/mod.rs:826-848) and the state before any
    broad phase: no counters, no stored pairs."""
    pos = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0]], np.float32)
    s = ClothSimulator(pos, np.array([[0, 1], [1, 2], [2, 3], [3, 0], [0, 2]]), np.array([[0, 1, 2], [0, 2, 3]]))
    assert s.get_pair_cache_stats() == (0, 0, 8192, 8192)
    assert not s.get_enable_pair_cache() and s.get_enable_pair_cache_final_fallback()
    s.set_enable_pair_cache(True)
    assert s.get_active_pairs() == (0, 0, [], [])
    s.set_pair_cache_options(10, 10 ** 7, 5, 1.0, 9.0, 1.0)
    assert s.get_pair_cache_stats()[2:] == (64, 262144)
    s.set_enable_pair_cache_final_fallback(False)
    assert not s.get_enable_pair_cache_final_fallback()
    s.set_enable_self_collision(True)
    s.step(1.0 / 60.0, 2)
    x, _, _ = s.get_state()
    assert np.isfinite(x).all()
