"""CUDA path (through the C ABI) against the oracle and the reference goldens.

Tolerances (floating point, stated by the build's target): positions within
1e-5 of the cloth extent per frame and 1e-4 of the extent after 600 substeps.
The kernels are built with --fmad=false and IEEE div/sqrt and follow the
oracle's operation order, so in practice the match is bit-exact; the tests
also report the fraction of bit-identical coordinates.  Integer outputs (hash
cell starts, sorted indices) must be bit-exact.
"""
import os

import numpy as np
import pytest

import golden_cases as gc
from gpu_common import compare_frames, extent
from taremincloth_b200 import ClothSimulator, scenes

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("case", ["case1", "case2", "case3"])
def test_golden_single_step_exact(oracle_lib, case):
    pin, pout = gc.step_input(case)
    s = gc.make(ClothSimulator, case, positions=pin)
    s.step(1.0 / 60.0, 20, 2)
    out = np.empty(len(pin) * 3, np.float32)
    s.get_positions(out)
    out = out.reshape(-1, 3)
    assert float(np.linalg.norm(out - pout, axis=1).max()) < 1e-5
    o = gc.make(oracle_lib.OracleSim, case, positions=pin)
    o.step(1.0 / 60.0, 20, 2)
    assert float(np.abs(out - o.get_positions().reshape(-1, 3)).max()) <= 1e-6


@pytest.mark.parametrize("case", ["case1", "case2", "case3", "case4"])
def test_golden_trajectories_match_oracle(oracle_lib, case):
    c, d, pos, inv = gc.load(case)
    g = gc.make(ClothSimulator, case)
    o = gc.make(oracle_lib.OracleSim, case)
    worst, same = compare_frames(g, o, 25, 1.0 / 60.0, 20, extent(pos))
    assert worst.max() <= 1e-4, worst
    assert worst[:5].max() <= 1e-5, worst


@pytest.mark.parametrize("case", ["case1", "case2", "case3", "case4"])
def test_golden_regression_criteria(case):
    """The reference's test_golden_regression.py:76-300 criteria on the CUDA path."""
    gc.golden_trajectory(ClothSimulator, case)


@pytest.mark.xfail(strict=True, reason="like the oracle, the CUDA path reaches about 19 mm (frame 25) against the "
                                       "reference's 15 mm all-frame bound for case 2 (test_golden_regression.py:170)")
def test_golden_case2_all_frame_bound():
    assert gc.golden_trajectory(ClothSimulator, "case2") < 15e-3


def test_config1_600_substeps(oracle_lib):
    sc = scenes.config1()
    g = scenes.build(ClothSimulator, sc)
    o = scenes.build(oracle_lib.OracleSim, sc)
    worst, same = compare_frames(g, o, sc["frames"], sc["dt"], sc["substeps"], extent(sc["positions"]))
    assert worst[0] <= 1e-5 and worst.max() <= 1e-4, (worst.max(), same.min())


def test_config2_small_with_mesh_and_self_collision(oracle_lib):
    sc = scenes.config2(n=40, subdiv=3)
    g = scenes.build(ClothSimulator, sc)
    o = scenes.build(oracle_lib.OracleSim, sc)
    worst, same = compare_frames(g, o, 12, sc["dt"], sc["substeps"], extent(sc["positions"]))
    assert worst[0] <= 1e-5 and worst.max() <= 1e-4, (worst, same)


def test_config2_small_with_per_triangle_collider_attributes(oracle_lib):
    """Per-triangle friction, thickness, restitution and one-sided flags
    (set_mesh_collider_triangles(attributes=...)) on the CUDA path and the oracle."""
    sc = scenes.config2(n=40, subdiv=3)
    g = scenes.build(ClothSimulator, sc)
    o = scenes.build(oracle_lib.OracleSim, sc)
    tris = np.asarray(sc["mesh"]["triangles"], np.float32)
    rng = np.random.default_rng(11)
    attr = np.stack([rng.uniform(0.0, 0.5, len(tris)), rng.uniform(0.005, 0.015, len(tris)),
                     np.zeros(len(tris)), rng.integers(0, 2, len(tris))], 1).astype(np.float32)
    for s in (g, o):
        s.set_mesh_collider_triangles(tris, friction=0.3, thickness=0.01, single_sided=True, attributes=attr)
    worst, same = compare_frames(g, o, 8, sc["dt"], sc["substeps"], extent(sc["positions"]))
    assert worst[0] <= 1e-5 and worst.max() <= 1e-4, (worst, same)


def test_config2_full_one_substep(oracle_lib):
    """Full-size configuration, one substep (the oracle takes ~30 s), with
    the direct pass's V-T and E-E pair lists bit-exact."""
    sc = scenes.config2()
    g = scenes.build(ClothSimulator, sc)
    o = scenes.build(oracle_lib.OracleSim, sc)
    g.set_pair_recording(True, 1 << 22, 1 << 22)
    o.set_pair_recording(True)
    dts = sc["dt"] / sc["substeps"]
    g.step(dts, 1)
    o.step(dts, 1)
    xg, _, _ = g.get_state()
    xo, _, _ = o.get_state()
    assert float(np.abs(xg - xo).max()) / extent(sc["positions"]) <= 1e-5
    a, b = g.get_pair_lists(), o.get_pair_lists()
    assert len(b["vt"]) > 10000 and len(b["ee"]) > 10000, (len(b["vt"]), len(b["ee"]))
    np.testing.assert_array_equal(a["vt"], b["vt"])
    np.testing.assert_array_equal(a["ee"], b["ee"])


@pytest.mark.parametrize("n,subdiv,frames", [(48, 3, 3), (96, 4, 6)])
def test_pair_lists_bit_exact(oracle_lib, n, subdiv, frames):
    """Pair lists of one direct pass from the same draped state: every V-T
    pair that reaches the contact math and every counted E-E pair."""
    sc = scenes.config2(n=n, subdiv=subdiv)
    o = scenes.build(oracle_lib.OracleSim, sc)
    for _ in range(frames):
        o.step(sc["dt"], sc["substeps"])
    x, _, v = o.get_state()
    g = scenes.build(ClothSimulator, sc)
    g.set_positions_and_velocities(x, v)
    o.set_state(x, v)
    g.set_pair_recording(True)
    o.set_pair_recording(True)
    dts = sc["dt"] / sc["substeps"]
    for _ in range(2):  # two passes in a row: the lists restart every pass
        g.step(dts, 1)
        o.step(dts, 1)
        a, b = g.get_pair_lists(), o.get_pair_lists()
        assert len(b["vt"]) > 500 and len(b["ee"]) > 500, (len(b["vt"]), len(b["ee"]))
        np.testing.assert_array_equal(a["vt"], b["vt"])
        np.testing.assert_array_equal(a["ee"], b["ee"])
    g.set_pair_recording(False)
    with pytest.raises(ValueError):
        g.get_pair_lists()


def test_pair_record_overflow_is_reported():
    sc = scenes.config2(n=48, subdiv=3)
    g = scenes.build(ClothSimulator, sc)
    for _ in range(3):  # into contact
        g.step(sc["dt"], sc["substeps"])
    g.set_pair_recording(True)
    g.step(sc["dt"] / sc["substeps"], 1)
    n_vt, n_ee = (len(v) for v in g.get_pair_lists().values())
    assert n_vt > 16 and n_ee > 16, (n_vt, n_ee)
    g.set_pair_recording(True, 16, 16)
    g.step(sc["dt"] / sc["substeps"], 1)
    with pytest.raises(ValueError, match="overflowed"):
        g.get_pair_lists()


def test_config2_full_frame_against_oracle_fixture():
    """One full-size frame (20 substeps) against the oracle's frame from
    tests/golden/make_oracle_frames.py, within 1e-5 of the extent; colouring,
    vertex and edge hash of the full scene bit-exact against the oracle."""
    sc = scenes.config2()
    g = scenes.build(ClothSimulator, sc)
    g.step(sc["dt"], sc["substeps"])
    ref = np.load(os.path.join(GOLDEN, "oracle_frames.npz"))["full_f1"]
    xg, _, _ = g.get_state()
    assert float(np.abs(xg.astype(np.float64) - ref).max()) / extent(sc["positions"]) <= 1e-5


def test_config2_full_coloring_and_hash_bit_exact(oracle_lib):
    sc = scenes.config2()
    g = scenes.build(ClothSimulator, sc)
    o = scenes.build(oracle_lib.OracleSim, sc)
    col, oc = g.get_coloring(), o.colors()
    for k in ("dist_off", "dist_cnt", "bend_off", "bend_cnt"):
        np.testing.assert_array_equal(col[k], oc[k])
    np.testing.assert_array_equal(col["dist_v"], o.distance_constraints()["v"])
    g.step(sc["dt"], 2)
    x, _, v = g.get_state()
    o.set_state(x, v)
    g.set_positions_and_velocities(x, v)
    for which in (0, 1):
        cs_g, s_g = g.get_hash_state(which)
        cs_o, s_o = o.build_hash(which)
        np.testing.assert_array_equal(cs_g, cs_o)
        np.testing.assert_array_equal(s_g, s_o)


def test_config2_128_600_substeps_against_oracle_fixture():
    """Two 128 x 128 sheets on the icosphere, 600 substeps (30 frames),
    within 1e-4 of the extent of the oracle's frames 1, 10, 20, 30."""
    sc = scenes.config2(n=128)
    g = scenes.build(ClothSimulator, sc)
    ref = np.load(os.path.join(GOLDEN, "oracle_frames.npz"))
    ext = extent(sc["positions"])
    for f in range(1, 31):
        g.step(sc["dt"], sc["substeps"])
        if f in (1, 10, 20, 30):
            xg, _, _ = g.get_state()
            err = float(np.abs(xg.astype(np.float64) - ref[f"mid_f{f}"]).max()) / ext
            assert err <= (1e-5 if f == 1 else 1e-4), (f, err)


def test_hash_state_bit_exact(oracle_lib):
    """Cell starts and sorted indices of the vertex and edge grids."""
    sc = scenes.config2(n=64, subdiv=3)
    g = scenes.build(ClothSimulator, sc)
    o = scenes.build(oracle_lib.OracleSim, sc)
    for _ in range(3):
        o.step(sc["dt"], sc["substeps"])
    x, _, v = o.get_state()
    g.set_positions_and_velocities(x, v)
    o.set_state(x, v)
    for which in (0, 1):
        cs_g, s_g = g.get_hash_state(which)
        cs_o, s_o = o.build_hash(which)
        np.testing.assert_array_equal(cs_g, cs_o)
        np.testing.assert_array_equal(s_g, s_o)


@pytest.mark.parametrize("cell", [0.08, 0.12, 0.5])
def test_hash_crowded_buckets_match_static_build(cell):
    """Coarse hash cells crowd the buckets past the 64 entries of the
    register sort (rank sort in shared memory up to 1,024, the serial
    fallback beyond): the simulator's vertex hash equals the allocation-free
    build's (whose bucket sort is a separate kernel) bit for bit."""
    import ctypes as C
    import torch
    from taremincloth_b200 import _lib
    L = _lib.load()
    sc = scenes.config2(n=96, subdiv=3)
    g = scenes.build(ClothSimulator, sc)
    g.step(sc["dt"], sc["substeps"])
    g.set_hash_cell_size(cell)
    cs_ref, srt_ref = g.get_hash_state(0)
    _, p, _ = g.get_state()
    n, table = len(p), g.get_counts()["table_size"]
    assert np.diff(cs_ref.astype(np.int64)).max() > 64
    pos = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    pos[:, :3] = torch.from_numpy(np.ascontiguousarray(p)).cuda()
    cs = torch.full((table + 1,), -1, dtype=torch.int32, device="cuda")
    srt = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    _lib.check(L.tc_hash_build_static(C.c_void_p(pos.data_ptr()), n, float(cell), int(table),
                                      C.c_void_p(cs.data_ptr()), C.c_void_p(srt.data_ptr()),
                                      C.c_void_p(torch.cuda.current_stream().cuda_stream)))
    torch.cuda.synchronize()
    np.testing.assert_array_equal(cs.cpu().numpy().view(np.uint32), cs_ref)
    np.testing.assert_array_equal(srt.cpu().numpy().view(np.uint32), srt_ref)


def test_colouring_on_device_matches_oracle(oracle_lib):
    sc = scenes.config1()
    g = scenes.build(ClothSimulator, sc)
    o = scenes.build(oracle_lib.OracleSim, sc)
    col = g.get_coloring()
    oc = o.colors()
    np.testing.assert_array_equal(col["dist_cnt"], oc["dist_cnt"])
    np.testing.assert_array_equal(col["dist_v"], o.distance_constraints()["v"])


def test_config2_full_frame_properties():
    """Size-independent properties at full size: finite, no deep penetration of
    the sphere, pinned-free cloth falls, residual reported."""
    sc = scenes.config2()
    g = scenes.build(ClothSimulator, sc)
    g.set_residual_tracking(True)
    y0 = float(sc["positions"][:, 1].mean())
    for _ in range(3):
        g.step(sc["dt"], sc["substeps"])
    x, _, v = g.get_state()
    assert np.isfinite(x).all() and np.isfinite(v).all()
    assert float(x[:, 1].mean()) < y0
    r = np.linalg.norm(x - np.array([0.5, 0.0, 0.5], np.float32), axis=1)
    assert float(r.min()) > 0.4 - 0.01
    res = g.get_residuals()
    assert np.isfinite(res["dist_rms_total"]) and res["dist_rms_total"] >= 0.0


def test_reset_and_state_roundtrip():
    sc = scenes.config1()
    g = scenes.build(ClothSimulator, sc)
    x0, _, _ = g.get_state()
    g.step(sc["dt"], sc["substeps"])
    x1, _, v1 = g.get_state()
    assert not np.array_equal(x0, x1)
    g.reset()
    xr, _, vr = g.get_state()
    np.testing.assert_array_equal(xr, x0)
    assert not vr.any()
    g.set_positions_and_velocities(x1, v1)
    x2, _, v2 = g.get_state()
    np.testing.assert_array_equal(x2, x1)
    np.testing.assert_array_equal(v2, v1)


def test_invalid_inputs_raise():
    with pytest.raises(ValueError):
        ClothSimulator(np.zeros((3, 3), np.float32), np.array([[0, 9]], np.uint32))
    with pytest.raises(ValueError):
        ClothSimulator(np.zeros((3, 2), np.float32), np.array([[0, 1]], np.uint32))
    s = ClothSimulator(np.zeros((3, 3), np.float32), np.array([[0, 1]], np.uint32))
    with pytest.raises(ValueError):
        s.get_positions(np.empty(2, np.float32))


@pytest.mark.parametrize("persistent", [True, False])
def test_solver_paths_match_oracle(oracle_lib, persistent):
    """Persistent cooperative solver and launch-per-colour path, config 1
    (whole frame in one launch) and reduced config 2 (self-collision between
    persistent launches)."""
    for sc, frames in ((scenes.config1(), 20), (scenes.config2(n=32, subdiv=3), 6)):
        g = scenes.build(ClothSimulator, sc)
        g.set_persistent_solver(persistent)
        o = scenes.build(oracle_lib.OracleSim, sc)
        worst, same = compare_frames(g, o, frames, sc["dt"], sc["substeps"], extent(sc["positions"]))
        assert worst.max() <= 1e-5, (persistent, worst, same)


def test_barrier_timeout_reports_status_and_context_survives(oracle_lib):
    """A grid barrier that can never be released ends by its poll limit with
    TC_ERR_TIMEOUT; the context stays usable and the next frame is exact."""
    from taremincloth_b200._lib import BarrierTimeout
    sc = scenes.config1()
    g = scenes.build(ClothSimulator, sc)
    with pytest.raises(BarrierTimeout):
        g.check_barrier_timeout(2000)
    o = scenes.build(oracle_lib.OracleSim, sc)
    worst, _ = compare_frames(g, o, 2, sc["dt"], sc["substeps"], extent(sc["positions"]))
    assert worst.max() <= 1e-5


@pytest.mark.parametrize("variant,list_cap,n,subdiv,frames", [
    (1, 0, 96, 4, 3), (1, 0, 256, 5, 1),  # grouped by cell
    (2, 0, 96, 4, 3), (2, 0, 256, 5, 1),  # contact work in the edge's warp
    (0, 256 * 6, 96, 4, 3),               # pair list of 6 per segment: most pairs overflow
    (0, 256, 96, 4, 2),                   # 1 per segment
    (0, 1, 96, 4, 2),                     # none: every pair worked by the search kernel
])
def test_ee_kernel_variants_match(oracle_lib, variant, list_cap, n, subdiv, frames):
    """The edge-edge kernel shapes against the default (warp per edge, counted
    pairs listed and worked one lane each): identical pair lists and
    bit-identical positions; the default with a pair list too small for the
    scene works the overflowing pairs in the search kernel with the same
    results.  At the smaller size also the oracle's pair lists."""
    sc = scenes.config2(n=n, subdiv=subdiv)
    a = scenes.build(ClothSimulator, sc)
    b = scenes.build(ClothSimulator, sc)
    b.set_self_collision_variant(variant)
    b.set_ee_pair_list_capacity(list_cap)
    for s in (a, b):
        s.set_pair_recording(True, 1 << 24, 1 << 23)
    for _ in range(frames):
        a.step(sc["dt"], sc["substeps"])
        b.step(sc["dt"], sc["substeps"])
        la, lb = a.get_pair_lists(), b.get_pair_lists()
        assert len(la["ee"]) > 100
        np.testing.assert_array_equal(la["ee"], lb["ee"])
        np.testing.assert_array_equal(la["vt"], lb["vt"])
        np.testing.assert_array_equal(a.get_state()[0], b.get_state()[0])
        np.testing.assert_array_equal(a.get_state()[2], b.get_state()[2])
    if n <= 96:
        x, _, v = b.get_state()
        o = scenes.build(oracle_lib.OracleSim, sc)
        o.set_state(x, v)
        b.set_positions_and_velocities(x, v)
        o.set_pair_recording(True)
        dts = sc["dt"] / sc["substeps"]
        b.step(dts, 1)
        o.step(dts, 1)
        np.testing.assert_array_equal(b.get_pair_lists()["ee"], o.get_pair_lists()["ee"])
