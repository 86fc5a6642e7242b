"""The reference's analytic simulator tests on the oracle (CPU) and on the
CUDA path (GPU), with the reference's own pass criteria, and the CUDA path's
final positions against the oracle's for every scenario.

These pin the pieces no golden vector covers: the triangle-mesh collider
(CCD, closest-point contact, single-sided recovery, segment culling),
boundary / one-sided / internal edge-edge CCD, vertex-triangle CCD against a
moving triangle, multi-layer untangling, compliant pins, air and Rayleigh
damping, and action/reaction of the self-collision penalty.  Scenario
sources are listed in reference_scenarios.py.

Not restated: the V-V virtual-particle test (simulation/tests.rs:838-903,
self-collision algorithm 2) and the Atomic-mode halves of :2539-2670
(solver_mode 1), both modes this library does not build.
"""
import numpy as np
import pytest

import reference_scenarios as rs

KINDS = [pytest.param("oracle", id="oracle"), pytest.param("gpu", id="gpu", marks=pytest.mark.gpu)]


@pytest.fixture
def sim_cls(request, oracle_lib):
    if request.param == "oracle":
        return oracle_lib.OracleSim
    from taremincloth_b200 import ClothSimulator
    return ClothSimulator


def kinds(fn):
    return pytest.mark.parametrize("sim_cls", KINDS, indirect=True)(fn)


@kinds
def test_mesh_triangle_collision(sim_cls):
    r = rs.mesh_triangle_collision(sim_cls)
    assert r["z"] >= 0.04 - 1e-3, r["z"]        # triangle 0.02 + cloth 0.02


@kinds
def test_mesh_triangle_single_sided_recovery(sim_cls):
    r = rs.mesh_triangle_single_sided(sim_cls)
    assert r["z"] >= 0.04 - 1e-3, r["z"]        # pushed from the back side to the front


@kinds
def test_collision_departure_velocity_and_segment_culling(sim_cls):
    r = rs.collision_departure(sim_cls)
    assert r["z_dep"] >= 0.04 - 1e-3, r
    assert np.isfinite(r["vz_dep"]) and -1e-4 <= r["vz_dep"] <= 1.0 + 1e-4, r
    assert r["z_seg_0"] >= 0.0 and r["z_seg_1"] >= 0.0, r


@kinds
def test_compliant_pin_full_hold(sim_cls):
    r = rs.compliant_pin(sim_cls, 1.0, 30)
    assert abs(r["y1"] - 0.5) < 1e-2, r["y1"]


@kinds
def test_compliant_pin_partial_blend(sim_cls):
    r = rs.compliant_pin(sim_cls, 0.5, 150)
    assert 1e-3 < r["y1"] < 0.5 - 1e-3, r["y1"]


@kinds
def test_self_collision_options_no_nan(sim_cls):
    r = rs.self_collision_options(sim_cls)
    assert np.isfinite(r["x"]).all()


@kinds
def test_boundary_ee_ccd_blocking(sim_cls):
    r = rs.boundary_ee_ccd(sim_cls)
    assert r["xa0"] <= r["xb0"] + 1e-4 and r["xa1"] <= r["xb1"] + 1e-4, r


@kinds
def test_one_sided_boundary_ee_ccd_blocking(sim_cls):
    r = rs.one_sided_boundary_ee_ccd(sim_cls)
    assert not r["open_34"]                      # 3-4 is shared by two faces
    assert r["xa0"] <= r["xb0"] + 1e-4 and r["xa1"] <= r["xb1"] + 1e-4, r


@kinds
def test_vt_ccd_moving_triangle_penetration_blocking(sim_cls):
    r = rs.vt_ccd_moving_triangle(sim_cls)
    assert r["z_pt3"] <= r["z_tri"] + 1e-4, r


@kinds
def test_internal_ee_ccd_blocking(sim_cls):
    r = rs.internal_ee_ccd(sim_cls)
    assert r["opens"] == (False, False)
    assert r["z_mid_b"] >= r["z_mid_a"] - 1e-4, r


@kinds
def test_internal_ee_ccd_low_speed_close_crossover_blocking(sim_cls):
    r = rs.internal_ee_low_speed_crossover(sim_cls)
    assert r["opens"] == (False, False)
    assert r["z_mid_b"] > r["z_mid_a"], r


@kinds
def test_internal_ee_ccd_folded_hinge_no_self_excitation(sim_cls):
    r = rs.folded_hinge(sim_cls)
    assert np.isfinite(r["x"]).all()
    assert r["max_disp"] < 0.05, r["max_disp"]


@kinds
def test_internal_ee_ccd_concurrent_double_hit_no_dilution(sim_cls):
    r = rs.double_hit_no_dilution(sim_cls)
    assert r["z_b"] >= r["z_a1"] - 1e-4 and r["z_b"] >= r["z_a2"] - 1e-4, r


@kinds
def test_internal_ee_discrete_untangling_symmetry_across_rotation(sim_cls):
    up = rs.discrete_untangling_rotation(sim_cls, False)["z_outer"]
    rot = rs.discrete_untangling_rotation(sim_cls, True)["z_outer"]
    assert abs(up - rot) < 1e-5, (up, rot)


@kinds
def test_static_pin_edge_low_index_blocks_dynamic_edge(sim_cls):
    r = rs.static_pin_edge(sim_cls)
    assert abs(r["z_mid_a"]) < 1e-6, r
    assert r["z_mid_b"] >= r["z_mid_a"] - 1e-4, r


@kinds
def test_pair_cache_ee_ccd_blocks_high_speed_crossing(sim_cls):
    r = rs.pair_cache_ee_ccd(sim_cls)
    assert r["z_mid_b"] >= r["z_mid_a"] - 1e-4, r


@kinds
def test_air_damping_single_application_and_internal_damping_rigid_invariance(sim_cls):
    expected = rs.air_damping_expected()
    v_air = rs.air_damping(sim_cls, 2.0, (0.0,) * 4)["vz"]
    v_int = rs.air_damping(sim_cls, 0.0, (20.0,) * 4)["vz"]
    v_zero = rs.air_damping(sim_cls, 0.0, (0.0,) * 4)["vz"]
    v_both = rs.air_damping(sim_cls, 2.0, (20.0,) * 4)["vz"]
    assert abs(v_air - expected) < 1e-3, (v_air, expected)
    assert abs(v_int - v_zero) < 1e-4, (v_int, v_zero)
    assert abs(v_both - v_air) < 1e-4, (v_both, v_air)


@kinds
def test_xpbd_rayleigh_internal_damping(sim_cls):
    for sub in (20, 10, 40):
        undamped = rs.rayleigh_stretch(sim_cls, sub, 0.0)["tail"]
        damped = rs.rayleigh_stretch(sim_cls, sub, 25.0)["tail"]
        assert damped < undamped * 0.4, (sub, damped, undamped)
    b0 = rs.rayleigh_bend(sim_cls, 0.0)["tail"]
    b1 = rs.rayleigh_bend(sim_cls, 15.0)["tail"]
    assert b1 < b0 * 0.5, (b1, b0)


@kinds
def test_untangling_no_false_positive_on_wrinkled_inner(sim_cls):
    r = rs.untangle_wrinkled_inner(sim_cls)
    assert (r["z_out"] > r["z_in"] - 1e-4).all(), (r["z_out"] - r["z_in"]).min()
    assert (np.abs(r["z_out"] - r["z_out0"]) < 0.008).all(), np.abs(r["z_out"] - r["z_out0"]).max()


@kinds
def test_untangling_no_false_positive_on_face_to_face_flip(sim_cls):
    r = rs.untangle_face_to_face(sim_cls)
    assert not np.isnan(r["gaps"]).any(), "an outer vertex left the inner layer's XY region"
    assert (r["gaps"] > 0.0005).all(), r["gaps"].min()


@kinds
def test_untangling_1d_strand_behind_dynamic_inner_escapes(sim_cls):
    r = rs.strand_escape(sim_cls)
    assert (r["z_strand"] > 0.0015).all(), r["z_strand"]


@kinds
def test_self_collision_equal_mass_symmetry(sim_cls):
    r = rs.self_collision_symmetry(sim_cls, 1.0, 1.0)
    assert r["bottom"] < 0.0 and r["top"] > 0.0, r
    rel = abs(r["bottom"] + r["top"]) / max(abs(r["bottom"]), abs(r["top"]), 1e-6)
    assert rel < 0.05, rel


@kinds
def test_self_collision_unequal_mass_momentum_conservation(sim_cls):
    r = rs.self_collision_symmetry(sim_cls, 0.5, 1.0)
    pb, pt = r["bottom"] / 1.0, r["top"] / 0.5
    rel = abs(pb + pt) / max(abs(pb), abs(pt), 1e-6)
    assert abs(r["bottom"]) > abs(r["top"]), r
    assert rel < 0.10, rel


# --------------------------------------------------------------------------
# the CUDA path against the oracle on every scenario

SCENARIOS = {
    "mesh_triangle_collision": rs.mesh_triangle_collision,
    "mesh_triangle_single_sided": rs.mesh_triangle_single_sided,
    "collision_departure": rs.collision_departure,
    "compliant_pin_full": lambda c: rs.compliant_pin(c, 1.0, 30),
    "compliant_pin_partial": lambda c: rs.compliant_pin(c, 0.5, 150),
    "self_collision_options": rs.self_collision_options,
    "boundary_ee_ccd": rs.boundary_ee_ccd,
    "one_sided_boundary_ee_ccd": rs.one_sided_boundary_ee_ccd,
    "vt_ccd_moving_triangle": rs.vt_ccd_moving_triangle,
    "internal_ee_ccd": rs.internal_ee_ccd,
    "internal_ee_low_speed_crossover": rs.internal_ee_low_speed_crossover,
    "folded_hinge": rs.folded_hinge,
    "double_hit_no_dilution": rs.double_hit_no_dilution,
    "discrete_untangling_rotated": lambda c: rs.discrete_untangling_rotation(c, True),
    "static_pin_edge": rs.static_pin_edge,
    "pair_cache_ee_ccd": rs.pair_cache_ee_ccd,
    "air_damping": lambda c: rs.air_damping(c, 2.0, (20.0,) * 4),
    "rayleigh_stretch": lambda c: rs.rayleigh_stretch(c, 20, 25.0),
    "rayleigh_bend": lambda c: rs.rayleigh_bend(c, 15.0),
    "untangle_wrinkled_inner": rs.untangle_wrinkled_inner,
    "untangle_face_to_face": rs.untangle_face_to_face,
    "strand_escape": rs.strand_escape,
    "self_collision_symmetry": lambda c: rs.self_collision_symmetry(c, 0.5, 1.0),
}


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(SCENARIOS))
def test_scenario_matches_oracle(oracle_lib, name):
    """Final positions of the CUDA path within 1e-5 of the scene's extent of
    the oracle's (bit-identical where no reduction order differs)."""
    from taremincloth_b200 import ClothSimulator
    g = SCENARIOS[name](ClothSimulator)["x"]
    o = SCENARIOS[name](oracle_lib.OracleSim)["x"]
    ext = max(float(np.linalg.norm(o.max(0) - o.min(0))), 1e-3)
    err = float(np.abs(g - o).max()) / ext
    assert err <= 1e-5, (name, err)


@pytest.mark.gpu
def test_bone_sdf_collision(oracle_lib):
    """simulation/tests.rs:443-554: a vertex falling onto a bone SDF whose
    surface is z = 0 stops at the summed thickness (0.04, within 2 mm, not
    above 0.06); moving the bone up 0.1 pushes it to z >= 0.14 - 2 mm.  The
    CUDA path's positions are also compared with the oracle's, given the same
    atlas, bone infos and transforms."""
    from taremincloth_b200 import ClothSimulator
    tex, info = rs.bone_plane_atlas()
    g = rs._mk(ClothSimulator, [[0.0, 0.0, 0.4]], np.zeros((0, 2)))
    o = rs._mk(oracle_lib.OracleSim, [[0.0, 0.0, 0.4]], np.zeros((0, 2)))
    g.set_bone_sdf_colliders(16, 16, 16, tex.tobytes(), info)

    def pose(dz):
        w, iw = rs.bone_mats(dz)
        g.update_bone_transforms(w, iw)
        xf = np.concatenate([w.reshape(1, 16), iw.reshape(1, 16)], 1)
        o.set_bone_sdf((16, 16, 16), tex, g.get_bone_infos(), xf)

    pose(0.0)
    for _ in range(60):
        g.step(1.0 / 60.0, 20)
        o.step(1.0 / 60.0, 20)
    z = float(g.get_state()[0][0, 2])
    assert 0.04 - 2e-3 <= z <= 0.06, z
    assert abs(z - float(o.get_state()[0][0, 2])) <= 1e-6
    pose(0.1)
    for _ in range(30):
        g.step(1.0 / 60.0, 20)
        o.step(1.0 / 60.0, 20)
    zm = float(g.get_state()[0][0, 2])
    assert zm >= 0.14 - 2e-3, zm
    assert abs(zm - float(o.get_state()[0][0, 2])) <= 1e-6


@pytest.mark.gpu
def test_single_layer_disables_effective_untangling():
    """simulation/tests.rs:392-441: untangling is on by default but effective
    only with several layers; turning the option off disables it."""
    from taremincloth_b200 import ClothSimulator
    quad = dict(positions=[[0, 0, 0.5], [1, 0, 0.5], [1, 1, 0.5], [0, 1, 0.5]],
                edges=[[0, 1], [1, 2], [2, 3], [3, 0], [0, 2]], faces=[[0, 1, 2], [0, 2, 3]])
    s = rs._mk(ClothSimulator, quad["positions"], quad["edges"], faces=quad["faces"])
    assert not s.get_has_multiple_layers()
    assert not s.get_effective_normal_untangling()
    s2 = rs._mk(ClothSimulator, quad["positions"], quad["edges"], faces=quad["faces"], layer_ids=[0, 0, 1, 1])
    assert s2.get_has_multiple_layers()
    assert s2.get_effective_normal_untangling()
    s2.set_self_collision_options(0.2, 0.2, True, False, 128)
    assert not s2.get_effective_normal_untangling()
