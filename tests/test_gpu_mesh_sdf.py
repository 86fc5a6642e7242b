"""Single-mesh SDF bake on the GPU (bake_mesh_sdf_gpu, lib.rs:1349-1416;
sdf_baker.rs:939-1060, :1114-1326; bake_mesh_sdf.wgsl).

* A closed icosphere against the oracle's in-order scan of every triangle
  per voxel: dimensions, the 20-float info and every texel bit-exact (the
  culled scan of the GPU kernel skips only triangles that cannot win).
* Signs: negative inside the sphere, positive outside, |d| near the radius
  difference; alpha 1 everywhere.
* An open tube: with its boundary loops capped the centre is inside
  (negative); the reference's error on an empty mesh.
"""
import numpy as np
import pytest

from taremincloth_b200 import scenes
from taremincloth_b200.simulator import bake_mesh_sdf_gpu

pytestmark = pytest.mark.gpu


def _halves(tex_bytes, shape):
    u = np.frombuffer(tex_bytes, np.uint32).reshape(shape)
    d = (u & 0xFFFF).astype(np.uint16).view(np.float16).astype(np.float32)
    a = (u >> 16).astype(np.uint16).view(np.float16).astype(np.float32)
    return u, d, a


def _icosphere(subdiv, r, c):
    tris = scenes.icosphere(subdiv, r, c).reshape(-1, 3)
    verts, inv = np.unique(tris, axis=0, return_inverse=True)
    return verts.astype(np.float32), inv.reshape(-1, 3).astype(np.int32)


def test_icosphere_bake_matches_oracle(oracle_lib):
    v, t = _icosphere(2, 0.1, (0.3, -0.2, 0.5))
    r = bake_mesh_sdf_gpu(v, t, voxel_size=0.008, margin=0.02, friction=0.4, thickness=0.005)
    dims, info, tex = oracle_lib.bake_mesh_sdf(v, t, 0.008, 0.02, 0.4, 0.005, 0.0)
    assert (r["width"], r["height"], r["depth"]) == tuple(int(x) for x in dims)
    np.testing.assert_array_equal(r["bone_info"], info)
    u, d, a = _halves(r["texture_bytes"], tex.shape)
    np.testing.assert_array_equal(u, tex)
    assert np.all(a == 1.0)
    # voxel centres: the closest point is on the sphere, the sign says which side
    W, H, D = r["width"], r["height"], r["depth"]
    lo, hi = info[0:3], info[4:7]
    zz, yy, xx = np.meshgrid(np.arange(D), np.arange(H), np.arange(W), indexing="ij")
    p = lo + (np.stack([xx, yy, zz], -1) + 0.5) / np.array([W, H, D]) * (hi - lo)
    rad = np.linalg.norm(p - np.array([0.3, -0.2, 0.5]), axis=-1) - 0.1
    far = np.abs(rad) > 0.01
    assert np.all(np.sign(d[far]) == np.sign(rad[far]))
    assert np.abs(d - rad)[far].max() < 0.01


def test_open_tube_is_capped():
    n, m = 24, 6
    ang = np.linspace(0, 2 * np.pi, n, endpoint=False)
    rings = [np.stack([0.05 * np.cos(ang), 0.05 * np.sin(ang), np.full(n, z)], 1) for z in np.linspace(0, 0.2, m)]
    v = np.concatenate(rings).astype(np.float32)
    t = []
    for k in range(m - 1):
        for i in range(n):
            a, b, c, dd = k * n + i, k * n + (i + 1) % n, (k + 1) * n + (i + 1) % n, (k + 1) * n + i
            t += [[a, b, c], [a, c, dd]]
    t = np.asarray(t, np.int32)
    capped = bake_mesh_sdf_gpu(v, t, voxel_size=0.01, close_open_boundaries=True)
    W, H, D = capped["width"], capped["height"], capped["depth"]
    _, d, _ = _halves(capped["texture_bytes"], (D, H, W))
    lo, hi = capped["bone_info"][0:3], capped["bone_info"][4:7]
    centre = ((np.array([0.0, 0.0, 0.1]) - lo) / (hi - lo) * np.array([W, H, D])).astype(int)
    assert d[centre[2], centre[1], centre[0]] < 0.0
    with pytest.raises(RuntimeError):
        bake_mesh_sdf_gpu(np.zeros((0, 3), np.float32), np.zeros((0, 3), np.int32))
