"""Sewing on the GPU (through the C ABI).

* A sewn garment (two panels sewn along both sides, self-collision on,
  shrinking seams) against the oracle: positions within 1e-5 of the extent
  per frame, in the persistent and the per-colour launch modes; the sewing
  rest lengths bit-exact.
* The reference's simulation tests for sewing restated
  (crates/cloth_core/src/simulation/tests.rs:637-740, :1453-1530,
  :2998-3031): shrink speed changed mid-run keeps the progress; a flat seam
  closes to under 1 mm; the sewing priority latches, ramps and falls back.
"""
import numpy as np
import pytest

from gpu_common import compare_frames, extent
from taremincloth_b200 import ClothSimulator, scenes

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("persistent", [True, False])
def test_sewn_garment_matches_oracle(oracle_lib, persistent):
    sc = scenes.sewn_garment(n=24)
    g = scenes.build(ClothSimulator, sc)
    g.set_persistent_solver(persistent)
    o = scenes.build(oracle_lib.OracleSim, sc)
    assert g.get_num_sewing_constraints() == 48
    worst, same = compare_frames(g, o, sc["frames"], sc["dt"], sc["substeps"], extent(sc["positions"]))
    assert worst.max() <= 1e-5, (persistent, worst, same)
    np.testing.assert_array_equal(np.asarray(g.get_sewing_current_rest_lengths(), np.float32), o.sewing()["cur"])


def test_sewn_garment_seams_close():
    """The side seams shrink at 0.5 m/s from 6 cm and latch within the lock
    distance: after 12 frames every spring's rest length is 0 and every pair
    whose vertices are not pinned (the top corners are) is within a few
    millimetres."""
    sc = scenes.sewn_garment(n=24)
    g = scenes.build(ClothSimulator, sc)
    for _ in range(sc["frames"]):
        g.step(sc["dt"], sc["substeps"])
    x, _, _ = g.get_state()
    pinned = {v for v, _ in sc["pins"]}
    free = np.array([a not in pinned and b not in pinned for a, b in sc["sewing"]])
    d = np.linalg.norm(x[sc["sewing"][:, 0]] - x[sc["sewing"][:, 1]], axis=1)
    assert np.all(np.asarray(g.get_sewing_current_rest_lengths()) == 0.0)
    assert free.sum() == len(free) - 2 and d[free].max() < 5e-3, d[free].max()


def test_shrink_speed_change_keeps_progress():
    """simulation/tests.rs:2998-3031: one spring 1 m long, 0.5 m/s: after a
    0.1 s frame the rest length is 0.95; at 2 m/s the next frame gives 0.75."""
    pos = np.array([[0, 0, 0], [1, 0, 0]], np.float32)
    s = ClothSimulator(pos, np.zeros((0, 2), np.uint32), sewing_springs=np.array([[0, 1]]), stiffness=1000.0,
                       shear_stiffness=500.0, bending_stiffness=0.0, sewing_shrink_speed=0.5,
                       sewing_stiffness=1000.0, enable_sewing_lock=False)
    s.set_gravity(0.0, 0.0, 0.0)
    s.step(0.1, 4)
    r1 = s.get_sewing_current_rest_lengths()[0]
    assert abs(r1 - 0.95) < 1e-3, r1
    s.set_sewing_shrink_speed(2.0)
    assert abs(s.get_sewing_shrink_speed() - 2.0) < 1e-6
    assert abs(s.get_sewing_current_rest_lengths()[0] - 0.95) < 1e-3
    s.step(0.1, 4)
    r2 = s.get_sewing_current_rest_lengths()[0]
    assert abs(r2 - 0.75) < 1e-3, r2
    s.set_sewing_current_rest_lengths([0.5])
    assert s.get_sewing_current_rest_lengths()[0] == 0.5
    s.set_sewing_current_rest_lengths([0.5, 0.1])  # wrong length: ignored, as in the reference
    assert s.get_sewing_current_rest_lengths()[0] == 0.5


def test_flat_seam_closes():
    """simulation/tests.rs:1453-1530: two flat quads 5 cm apart, sewn along
    the facing edges, self-collision on, no gravity: after 30 frames of 15
    substeps both pairs are closer than 1 mm."""
    pos = np.array([[-0.05, 0, 0], [0, 0, 0], [0, 0.1, 0], [-0.05, 0.1, 0],
                    [0.05, 0, 0], [0.05, 0.1, 0], [0.10, 0.1, 0], [0.10, 0, 0]], np.float32)
    edges = np.array([[0, 1], [1, 2], [2, 3], [3, 0], [0, 2], [4, 5], [5, 6], [6, 7], [7, 4], [4, 6]])
    faces = np.array([[0, 1, 2], [0, 2, 3], [4, 5, 6], [4, 6, 7]])
    s = ClothSimulator(pos, edges, faces, sewing_springs=np.array([[1, 4], [2, 5]]), stiffness=10000.0,
                       compression_stiffness=10000.0, shear_stiffness=5000.0, bending_stiffness=0.0)
    s.set_enable_self_collision(True)
    s.set_gravity(0.0, 0.0, 0.0)
    for _ in range(30):
        s.step(1.0 / 60.0, 15)
    x, _, _ = s.get_state()
    assert np.linalg.norm(x[1] - x[4]) < 1e-3 and np.linalg.norm(x[2] - x[5]) < 1e-3


def _two_point(**kw):
    pos = np.array([[0, 0, 0], [1, 0, 0]], np.float32)
    return pos, ClothSimulator(pos, np.zeros((0, 2), np.uint32), sewing_springs=np.array([[0, 1]]),
                               stiffness=10000.0, compression_stiffness=10.0, shear_stiffness=5000.0,
                               bending_stiffness=0.0, **kw)


def test_sewing_priority_latch_and_ramp():
    """simulation/tests.rs:657-696: held at 0 until closed, then smoothstep
    0.5, 1.0; the latch is one-way."""
    pos, s = _two_point()
    s.set_sewing_priority_options(True, 0.9, 0.005, 2, 0)
    assert s.update_sewing_priority(pos) == (0.0, 0.0, False)
    assert s.is_sewing_priority_active()
    closed = np.array([[0, 0, 0], [0.001, 0, 0]], np.float32)
    r1, s1, l1 = s.update_sewing_priority(closed)
    assert r1 == 1.0 and l1 and abs(s1 - 0.5) < 1e-6
    _, s2, _ = s.update_sewing_priority(closed)
    assert abs(s2 - 1.0) < 1e-6
    _, s3, l3 = s.update_sewing_priority(pos)
    assert l3 and s3 == 1.0 and not s.is_sewing_priority_active()


def test_sewing_priority_max_frames_and_default():
    """simulation/tests.rs:698-739: an unreachable threshold latches at
    max_frames; off by default, the priority is the identity."""
    pos, s = _two_point()
    assert s.get_sewing_priority_scale() == 1.0 and not s.is_sewing_priority_active()
    assert s.update_sewing_priority(pos) == (1.0, 1.0, True)
    s.set_sewing_priority_options(True, 1.0, 0.005, 0, 2)
    assert s.update_sewing_priority(pos)[1:] == (0.0, False)
    assert s.update_sewing_priority(pos)[1:] == (1.0, True)


def test_sewing_priority_holds_gravity():
    """While the priority holds, a frame runs without gravity: a free vertex
    pair (no edges) does not fall; after the latch it does."""
    pos, s = _two_point()
    s.set_gravity(0.0, -9.81, 0.0)
    s.set_sewing_priority_options(True, 0.9, 0.005, 0, 0)
    s.update_sewing_priority(pos)
    s.step(1.0 / 60.0, 4)
    x, _, v = s.get_state()
    assert np.all(v[:, 1] == 0.0)
    s.set_sewing_priority_state(True, 1, 1.0, 1.0)
    s.step(1.0 / 60.0, 4)
    _, _, v = s.get_state()
    assert np.all(v[:, 1] < 0.0)


def test_invalid_sewing_springs_raise():
    pos = np.zeros((3, 3), np.float32)
    with pytest.raises(ValueError):
        ClothSimulator(pos, np.array([[0, 1]]), sewing_springs=np.array([[0, 3]]))
    with pytest.raises(ValueError):
        ClothSimulator(pos, np.array([[0, 1]]), sewing_springs=np.array([0, 1, 2]))


@pytest.mark.parametrize("persistent", [True, False])
def test_zero_network_warm_start_with_sewing_is_plain(persistent):
    """The warm-started substep with sewing (shrink, sewing colours in the
    iterations and in the gated fallback iterations, final sewing): with an
    all-zero network it gives the bits of the plain solver with n - k
    iterations (threshold +inf) or all n (threshold -1)."""
    from taremincloth_b200 import warmstart
    sc = scenes.sewn_garment(n=12)
    it, k = sc["iterations"], 2
    a, b, c, d = (scenes.build(ClothSimulator, sc) for _ in range(4))
    for s in (a, b, c, d):
        s.set_persistent_solver(persistent)
    zeros = np.zeros(warmstart.PARAM_COUNT, np.float32)
    a.ws_set_params(zeros)
    a.ws_enable(k, float("inf"))
    b.set_solver_iterations(it - k)
    c.ws_set_params(zeros)
    c.ws_enable(k, -1.0)
    for _ in range(3):
        for s in (a, b, c, d):
            s.step(sc["dt"], sc["substeps"])
    assert np.array_equal(a.get_state()[0], b.get_state()[0])
    assert np.array_equal(c.get_state()[0], d.get_state()[0])
    assert a.get_sewing_current_rest_lengths() == b.get_sewing_current_rest_lengths()
