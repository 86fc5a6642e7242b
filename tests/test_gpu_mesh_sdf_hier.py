"""Two-pass (hierarchical) mesh-SDF bake and its coarse pass on the GPU
(bake_mesh_sdf_hierarchical_gpu / bake_mesh_sdf_coarse_gpu, lib.rs:1418-1540;
sdf_baker.rs:1328-1900; bake_mesh_sdf_hier_*.wgsl).

* Against the oracle: the coarse pass's packed distances and 8 nearest
  triangles per cell, and the hierarchical texels, bit-exact (cube, double
  wall, icosphere), with equal dimensions and info.
* The reference's tests on the GPU results (sdf_baker.rs:1997-2120,
  tests/core/test_mesh_sdf_hierarchical.py): the coarse cube; within the band
  bit-equal to the single-pass bake, beyond it the same sign within the coarse
  half-diagonal; the band and empty-mesh errors.
"""
import numpy as np
import pytest

from mesh_fixtures import CUBE_T, CUBE_V, double_wall, equivalence
from taremincloth_b200 import scenes
from taremincloth_b200.simulator import bake_mesh_sdf_coarse_gpu, bake_mesh_sdf_gpu, bake_mesh_sdf_hierarchical_gpu

pytestmark = pytest.mark.gpu


def _icosphere(subdiv, r, c):
    tris = scenes.icosphere(subdiv, r, c).reshape(-1, 3)
    verts, inv = np.unique(tris, axis=0, return_inverse=True)
    return verts.astype(np.float32), inv.reshape(-1, 3).astype(np.int32)


def _tex(r):
    return np.frombuffer(r["texture_bytes"], np.uint32).reshape(r["depth"], r["height"], r["width"])


def test_coarse_cube():
    r = bake_mesh_sdf_coarse_gpu(CUBE_V, CUBE_T, voxel_size=0.05, margin=0.2, friction=0.5, thickness=0.01)
    assert (r["width"], r["height"], r["depth"]) == (8, 8, 8)
    assert abs(r["coarse_voxel"] - 0.2) < 1e-6
    assert r["dist_packed"].size == 512 and r["nearest_tri"].size == 512 * 8
    assert r["nearest_tri"].max() < 12
    flat = lambda x, y, z: (z * 8 + y) * 8 + x
    assert not r["dist_packed"][flat(0, 0, 0)] & 0x8000
    assert r["dist_packed"][flat(4, 4, 4)] & 0x8000


@pytest.mark.parametrize("case", ["cube", "wall", "sphere"])
def test_matches_oracle(oracle_lib, case):
    if case == "cube":
        v, t, vox, margin, th = CUBE_V, CUBE_T, 0.05, 0.2, 0.01
    elif case == "wall":
        (v, t), vox, margin, th = double_wall(), 0.004, 0.02, 0.005
    else:
        (v, t), vox, margin, th = _icosphere(3, 0.12, (0.1, 0.2, -0.3)), 0.003, 0.02, 0.005
    c = bake_mesh_sdf_coarse_gpu(v, t, voxel_size=vox, margin=margin, thickness=th)
    dims, cv, dist, near = oracle_lib.bake_mesh_sdf_coarse(v, t, vox, margin, th)
    assert (c["width"], c["height"], c["depth"]) == tuple(int(x) for x in dims) and c["coarse_voxel"] == cv
    np.testing.assert_array_equal(c["dist_packed"], dist.ravel())
    np.testing.assert_array_equal(c["nearest_tri"], near.ravel())
    h = bake_mesh_sdf_hierarchical_gpu(v, t, voxel_size=vox, margin=margin, friction=0.5, thickness=th)
    dims, info, tex = oracle_lib.bake_mesh_sdf_hierarchical(v, t, vox, margin, 0.5, th, 0.0)
    assert (h["width"], h["height"], h["depth"]) == tuple(int(x) for x in dims)
    np.testing.assert_array_equal(h["bone_info"], info)
    np.testing.assert_array_equal(_tex(h), tex)


@pytest.mark.parametrize("case", ["cube", "wall"])
def test_equivalent_to_single_pass(case):
    if case == "cube":
        v, t, vox, margin, th, nb, fb = CUBE_V, CUBE_T, 0.05, 0.2, 0.01, 0.21, 0.18
    else:
        (v, t), vox, margin, th, nb, fb = double_wall(), 0.004, 0.02, 0.005, 0.02, 0.03
    leg = bake_mesh_sdf_gpu(v, t, voxel_size=vox, margin=margin, thickness=th)
    hie = bake_mesh_sdf_hierarchical_gpu(v, t, voxel_size=vox, margin=margin, thickness=th)
    assert (hie["width"], hie["height"], hie["depth"]) == (leg["width"], leg["height"], leg["depth"])
    near_mm, far_sign, far_diff = equivalence(_tex(leg), _tex(hie), nb)
    assert near_mm == 0 and far_sign == 0 and far_diff <= fb, (near_mm, far_sign, far_diff)


def test_errors():
    with pytest.raises(RuntimeError):
        bake_mesh_sdf_hierarchical_gpu(np.zeros((0, 3), np.float32), np.zeros((0, 3), np.int32))
    with pytest.raises(RuntimeError):
        bake_mesh_sdf_coarse_gpu(np.zeros((0, 3), np.float32), np.zeros((0, 3), np.int32))
    v = np.array([[0, 0, 0], [2000, 0, 0], [0, 0.01, 0]], np.float32)
    with pytest.raises(RuntimeError):
        bake_mesh_sdf_hierarchical_gpu(v, np.array([[0, 1, 2]], np.int32), voxel_size=0.004)
