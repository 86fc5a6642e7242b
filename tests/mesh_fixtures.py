"""Closed test meshes of the reference's mesh-SDF tests
(crates/cloth_core/src/sdf_baker.rs:1997-2120, tests/core/test_mesh_sdf_hierarchical.py):
the unit cube, and two 2 mm plates with a 3 mm gap."""
import numpy as np

CUBE_V = np.array([[-0.5, -0.5, -0.5], [0.5, -0.5, -0.5], [0.5, 0.5, -0.5], [-0.5, 0.5, -0.5],
                   [-0.5, -0.5, 0.5], [0.5, -0.5, 0.5], [0.5, 0.5, 0.5], [-0.5, 0.5, 0.5]], np.float32)
_BOX_T = np.array([[0, 2, 1], [0, 3, 2], [4, 5, 6], [4, 6, 7], [0, 1, 5], [0, 5, 4],
                   [2, 3, 7], [2, 7, 6], [0, 4, 7], [0, 7, 3], [1, 2, 6], [1, 6, 5]], np.int32)
CUBE_T = _BOX_T.copy()


def double_wall():
    """Two 0.3 m square plates, 2 mm thick, 3 mm apart."""
    def plate(z0, t=0.002, s=0.15):
        return np.array([[-s, -s, z0], [s, -s, z0], [s, s, z0], [-s, s, z0],
                         [-s, -s, z0 + t], [s, -s, z0 + t], [s, s, z0 + t], [-s, s, z0 + t]], np.float32)
    v1, v2 = plate(0.0), plate(0.005)
    return np.vstack([v1, v2]), np.vstack([_BOX_T, _BOX_T + len(v1)]).astype(np.int32)


def decode(u):
    """fp16 distances of packed texels (low half)."""
    return (np.asarray(u, np.uint32) & 0xFFFF).astype(np.uint16).view(np.float16).astype(np.float32)


def equivalence(legacy, hier, near_bound):
    """(near mismatches, far sign mismatches, far max |diff|) of two packed fields,
    near = |legacy distance| <= near_bound (the reference's criteria)."""
    lp, hp = np.asarray(legacy, np.uint32).ravel(), np.asarray(hier, np.uint32).ravel()
    ld, hd = decode(lp), decode(hp)
    near = np.abs(ld) <= near_bound
    far = ~near
    return (int(((lp & 0xFFFF) != (hp & 0xFFFF))[near].sum()), int(((ld < 0) != (hd < 0))[far].sum()),
            float(np.abs(ld - hd)[far].max()) if far.any() else 0.0)
