"""Edge colliders on the GPU (edge_collision.wgsl; simulation/mod.rs:1007-1025).

* The reference's tests (crates/cloth_core/src/simulation/tests.rs:775-830,
  :2890-2960): a collider triangle's edges (3) push a crossing cloth edge up;
  a single-sided roof ridge pushes a chord that dips behind it outward.
* Two sheets with self-collision over a low-poly icosphere with edge
  collision on, against the oracle: positions within 1e-5 of the extent per
  frame, persistent and per-colour; the collider-edge count equal.
"""
import numpy as np
import pytest

from gpu_common import compare_frames, extent
from taremincloth_b200 import ClothSimulator, scenes

pytestmark = pytest.mark.gpu


def _edge_sim(pos, thickness):
    s = ClothSimulator(np.asarray(pos, np.float32), np.array([[0, 1]]), thickness=thickness, stiffness=10000.0,
                       compression_stiffness=10000.0, shear_stiffness=5000.0, bending_stiffness=0.0)
    s.set_enable_edge_collision(True)
    s.set_gravity(0.0, 0.0, 0.0)
    return s


def test_collider_edge_pushes_crossing_cloth_edge_up():
    s = _edge_sim([[-0.5, 0, 0], [0.5, 0, 0]], 0.02)
    tri = np.array([[[0.0, -0.5, -0.01], [0.0, 0.5, -0.01], [0.5, 0.0, -0.01]]], np.float32)
    s.set_mesh_collider_triangles(tri, friction=0.1, thickness=0.02, single_sided=False)
    assert s.get_num_collider_edges() == 3
    s.step(0.016, 5)
    x, _, _ = s.get_state()
    assert 0.5 * (x[0, 2] + x[1, 2]) > 0.0


def test_single_sided_ridge_pushes_chord_outward():
    s = _edge_sim([[0.0, -0.08, -0.025], [0.0, 0.08, -0.025]], 0.01)
    s.set_damping(0.0)
    roof = np.array([[[-0.5, 0, 0], [0.5, 0, 0], [0, 0.5, -0.5]],
                     [[-0.5, 0, 0], [0, -0.5, -0.5], [0.5, 0, 0]]], np.float32)
    s.set_mesh_collider_triangles(roof, friction=0.0, thickness=0.02, single_sided=True)
    assert s.get_num_collider_edges() == 5
    s.step(0.016, 5)
    x, _, _ = s.get_state()
    assert 0.5 * (x[0, 2] + x[1, 2]) > 0.0


@pytest.mark.parametrize("persistent", [True, False])
def test_edge_collision_matches_oracle(oracle_lib, persistent):
    sc = scenes.config2(n=32, subdiv=1)
    g = scenes.build(ClothSimulator, sc)
    g.set_persistent_solver(persistent)
    g.set_enable_edge_collision(True)
    g.set_edge_margin_offset(0.002)
    o = scenes.build(oracle_lib.OracleSim, sc)
    o.set_edge_collision(True, 1.0, 0.002)
    assert g.get_num_collider_edges() == o.num_collider_edges() == 120
    worst, same = compare_frames(g, o, 30, sc["dt"], sc["substeps"], extent(sc["positions"]))
    assert worst.max() <= 1e-5, (persistent, worst, same)
