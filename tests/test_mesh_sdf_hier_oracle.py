"""The oracle's two-pass (hierarchical) mesh-SDF bake against the reference's
own expectations, on the CPU:
* sdf_baker.rs:1997-2056: the coarse pass of the unit cube (voxel 5 cm,
  margin 20 %) is 8 x 8 x 8 at 0.2 m, indices below 12, a corner cell
  outside (positive) and the centre inside (negative);
* sdf_baker.rs:2058-2120 and tests/core/test_mesh_sdf_hierarchical.py:
  against the single-pass bake, voxels within the band bit-equal, farther
  ones with the same sign and within the coarse half-diagonal (cube at 5 cm;
  the double wall at 4 mm);
* the band check: a band wider than two coarse cells is an error.
"""
import numpy as np
import pytest

from mesh_fixtures import CUBE_T, CUBE_V, double_wall, equivalence


def test_coarse_cube(oracle_lib):
    dims, cv, dist, near = oracle_lib.bake_mesh_sdf_coarse(CUBE_V, CUBE_T, 0.05, 0.2, 0.01)
    assert tuple(int(x) for x in dims) == (8, 8, 8)
    assert abs(cv - 0.2) < 1e-6
    assert dist.size == 512 and near.size == 512 * 8
    assert near.max() < 12
    assert not dist[0, 0, 0] & 0x8000 and dist[4, 4, 4] & 0x8000
    # the 8 indices of a cell are distinct triangles (12 > 8)
    assert all(len(set(r)) == 8 for r in near.reshape(-1, 8).tolist())


def test_cube_hierarchical_matches_single_pass(oracle_lib):
    _, _, legacy = oracle_lib.bake_mesh_sdf(CUBE_V, CUBE_T, 0.05, 0.2, 0.5, 0.01, 0.0)
    dims, _, hier = oracle_lib.bake_mesh_sdf_hierarchical(CUBE_V, CUBE_T, 0.05, 0.2, 0.5, 0.01, 0.0)
    assert hier.shape == legacy.shape
    near_mm, far_sign, far_diff = equivalence(legacy, hier, 0.21)
    assert near_mm == 0 and far_sign == 0 and far_diff <= 0.18


def test_double_wall_hierarchical_matches_single_pass(oracle_lib):
    v, t = double_wall()
    _, _, legacy = oracle_lib.bake_mesh_sdf(v, t, 0.004, 0.02, 0.5, 0.005, 0.0)
    _, _, hier = oracle_lib.bake_mesh_sdf_hierarchical(v, t, 0.004, 0.02, 0.5, 0.005, 0.0)
    near_mm, far_sign, far_diff = equivalence(legacy, hier, 0.02)
    assert near_mm == 0 and far_sign == 0 and far_diff <= 0.03


def test_band_wider_than_two_coarse_cells_is_an_error(oracle_lib):
    # a flat mesh 2 km wide: the fine grid clamps at 2048 voxels, so the fine
    # voxel (and band) grows while the coarse grid keeps its 8-voxel floor
    v = np.array([[0, 0, 0], [2000, 0, 0], [0, 0.01, 0]], np.float32)
    t = np.array([[0, 1, 2]], np.int32)
    with pytest.raises(RuntimeError):
        oracle_lib.bake_mesh_sdf_hierarchical(v, t, 0.004, 0.02, 0.5, 0.005, 0.0)
