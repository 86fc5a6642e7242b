"""Per-edge rest lengths, compliance reset and single-substep stepping on the
GPU (lib.rs:1809-1813, :2684-2733; simulation/mod.rs:1450-1568;
dispatch.rs:674-688).

* set_edge_rest_length_scales: the constraint of each listed input edge gets
  initial rest x max(scale, 0.01); the getters report it; reset restores it;
  a sheet whose rest lengths are all scaled by 0.9 contracts.
* reset_edge_stiffness_multipliers restores the tension compliance.
* step_single_substep(dt) gives the same bits as step(dt, 1).
"""
import numpy as np
import pytest

from taremincloth_b200 import ClothSimulator, scenes

pytestmark = pytest.mark.gpu


def _sheet():
    sc = scenes.config1()
    s = ClothSimulator(sc["positions"], sc["edges"], sc["faces"], sc["inv_masses"], thickness=0.005,
                       stiffness=1000.0)
    return sc, s


def test_edge_rest_length_scales():
    sc, s = _sheet()
    e = np.asarray(sc["edges"])
    L0 = np.linalg.norm(sc["positions"][e[:, 0]] - sc["positions"][e[:, 1]], axis=1)
    for k in (0, 5, 100):
        assert s.get_edge_initial_rest_length(k) == pytest.approx(L0[k], rel=1e-6)
        assert s.get_edge_rest_length(k) == s.get_edge_initial_rest_length(k)
    s.set_edge_rest_length_scales([0, 5, 100], [0.5, 1.2, -3.0])
    assert s.get_edge_rest_length(0) == np.float32(s.get_edge_initial_rest_length(0)) * np.float32(0.5)
    assert s.get_edge_rest_length(5) == np.float32(s.get_edge_initial_rest_length(5)) * np.float32(1.2)
    assert s.get_edge_rest_length(100) == np.float32(s.get_edge_initial_rest_length(100)) * np.float32(0.01)
    assert s.get_edge_rest_length(len(e) + 10) == 0.0
    s.reset_edge_rest_lengths()
    assert s.get_edge_rest_length(0) == s.get_edge_initial_rest_length(0)
    # every edge at 0.9: the free sheet contracts against an unscaled twin
    _, twin = _sheet()
    s.set_edge_rest_length_scales(np.arange(len(e)), np.full(len(e), 0.9, np.float32))
    ratio = []
    for sim in (s, twin):
        sim.set_gravity(0.0, 0.0, 0.0)
        for _ in range(20):
            sim.step(1.0 / 60.0, 10)
        x, _, _ = sim.get_state()
        ratio.append(float(np.median(np.linalg.norm(x[e[:, 0]] - x[e[:, 1]], axis=1) / L0)))
    assert ratio[0] < 0.98 and ratio[0] < ratio[1] - 0.02, ratio


def test_reset_edge_stiffness_multipliers():
    _, s = _sheet()
    c0 = s.get_edge_tension_compliance(3)
    assert c0 == pytest.approx(1.0 / 1000.0, rel=1e-6)
    s.set_edge_stiffness_multipliers([3], [4.0])
    assert s.get_edge_tension_compliance(3) == pytest.approx(c0 / 4.0, rel=1e-6)
    s.reset_edge_stiffness_multipliers()
    assert s.get_edge_tension_compliance(3) == c0


def test_step_single_substep_equals_one_substep_frame():
    sc = scenes.config1()
    a = scenes.build(ClothSimulator, sc)
    b = scenes.build(ClothSimulator, sc)
    for _ in range(3):
        a.step(sc["dt"] / 10, 1)
        b.step_single_substep(sc["dt"] / 10)
        xa, _, va = a.get_state()
        xb, _, vb = b.get_state()
        np.testing.assert_array_equal(xa, xb)
        np.testing.assert_array_equal(va, vb)
    assert b.get_workgroup_size() == 32 and b.get_solver_mode() == 0
    b.set_coupled_self_collision_options(0, 0)
    with pytest.raises(NotImplementedError):
        b.set_coupled_self_collision_options(2, 0)
    assert b.get_effective_normal_untangling() == bool(b.get_counts()["multi_layer"])
    b.set_self_collision_options(enable_normal_untangling=False)
    assert not b.get_effective_normal_untangling()
    assert b.get_num_virtual_vertices() >= 0


def test_config_json_roundtrip_and_hash():
    """get_config_json / apply_config_json / get_config_hash (lib.rs:3029-3047,
    config_impl.rs:16-160): a fresh simulator exports the constructor's
    settings; a changed record applied to another simulator exports the same
    text and hash; the hash follows every setter; bad text raises ValueError."""
    import json
    sc, s = _sheet()
    d = json.loads(s.get_config_json())
    assert d["gravity"] == [0.0, 0.0, -9.81] and d["damping"] == 1.0 and d["solver_iterations"] == 2
    assert d["enable_self_collision"] is True and d["relief_factor"] == 0.2
    # stiffness is exported from the stored f32 compliance 1/k (config_impl.rs:80-91)
    # (the text holds the shortest f32 digits: compare as f32)
    back = lambda k: np.float32(1.0) / (np.float32(1.0) / np.float32(k))  # noqa: E731
    f32 = lambda key: np.float32(d[key])  # noqa: E731
    assert f32("tension_stiffness") == back(1000.0) and f32("compression_stiffness") == back(1000.0)
    assert f32("shear_stiffness") == back(500.0) and f32("bending_stiffness") == back(10.0)
    h0 = s.get_config_hash()
    d.update(damping=2.5, tension_damping=3.0, solver_iterations=5, enable_edge_collision=True,
             edge_margin_offset=0.002, strain_tolerance=0.01, areal_density=0.2, gravity=[0.0, -9.81, 0.0],
             tension_stiffness=800.0, sewing_lock_distance=0.03)
    s.apply_config_json(json.dumps(d))
    text = s.get_config_json()
    assert json.loads(text)["solver_iterations"] == 5 and json.loads(text)["gravity"] == [0.0, -9.81, 0.0]
    assert s.get_config_hash() != h0
    _, s2 = _sheet()
    s2.apply_config_json(text)
    assert s2.get_config_json() == text and s2.get_config_hash() == s.get_config_hash()
    s2.set_damping(1.5)
    assert s2.get_config_hash() != s.get_config_hash()
    # absent fields take SimConfig::default
    _, s3 = _sheet()
    s3.apply_config_json("{}")
    assert json.loads(s3.get_config_json())["tension_damping"] == 5.0
    for bad in ("not json", "[1, 2]", '{"solver_iterations": -1}', '{"damping": "x"}'):
        with pytest.raises(ValueError):
            s3.apply_config_json(bad)


def test_device_lost_marks_and_recovers():
    """context.rs:499 restated: a device marked lost is re-initialised by the
    next simulator creation (new epoch); a simulator of the old epoch refuses
    calls with RuntimeError and can still be destroyed."""
    from taremincloth_b200.simulator import device_status, mark_device_lost
    _, old = _sheet()
    old.step(1.0 / 60.0, 2)
    lost, epoch = device_status(0)
    assert not lost
    mark_device_lost(0)
    assert device_status(0) == (True, epoch)
    with pytest.raises(RuntimeError, match="lost"):
        old.step(1.0 / 60.0, 2)
    _, fresh = _sheet()
    assert device_status(0) == (False, epoch + 1)
    fresh.step(1.0 / 60.0, 2)
    out = np.empty(fresh.get_num_vertices() * 3, np.float32)
    fresh.get_positions(out)
    assert np.isfinite(out).all()
    with pytest.raises(RuntimeError, match="epoch"):
        old.get_positions(out)
    del old


def test_nonfinite_readback_check():
    """The NaN / Inf sentinel on the host copy: off by default (positions are
    returned as they are), FloatingPointError when on."""
    sc, s = _sheet()
    p = np.array(sc["positions"], np.float32)
    p[7, 1] = np.nan
    s.set_positions_and_velocities(p)
    out = np.empty(len(p) * 3, np.float32)
    s.get_positions(out)
    assert np.isnan(out[3 * 7 + 1])
    s.set_nonfinite_check(True)
    with pytest.raises(FloatingPointError, match="vertex 7"):
        s.get_positions(out)
    s.set_nonfinite_check(False)
    s.get_positions(out)


def test_launch_block_and_cell_knobs():
    """Threads per block of the per-colour launches change no bit; a hash cell
    override changes the cell, None restores the reference formula's value,
    and the autotuner returns its launch and cell choices."""
    from taremincloth_b200.autotune import autotune
    sc = scenes.config2(n=32, subdiv=2)
    a = scenes.build(ClothSimulator, sc)
    b = scenes.build(ClothSimulator, sc)
    for s_ in (a, b):
        s_.set_launch_config(False)
    b.set_launch_block(128)
    for _ in range(3):
        a.step(sc["dt"], sc["substeps"])
        b.step(sc["dt"], sc["substeps"])
    np.testing.assert_array_equal(a.get_state()[0], b.get_state()[0])
    with pytest.raises(ValueError):
        b.set_launch_block(100)
    ref = a.get_cell_size()
    a.set_hash_cell_size(0.02)
    assert abs(a.get_cell_size() - 0.02) < 1e-9
    a.set_hash_cell_size(None)
    assert a.get_cell_size() == ref
    t = autotune(a, sc["dt"], sc["substeps"], frames=1, tune_cell_sizes=[1.5 * ref])
    assert t["block"] in (128, 256, 512) and len(t["hash_cell_trials"]) == 2
    assert t["hash_cell_trials"][0]["accepted"]
