"""CPU checks for the bone SDF row: the oracle's binary16 packing against
IEEE round-to-nearest-even (numpy), and the config 3 scene generator (closed
outward-facing capsules, rest pose, pose cycle, triangle sources grouped by
bone)."""
import numpy as np

from oracle import oracle as O
from taremincloth_b200 import scenes


def test_oracle_half_packing_matches_ieee():
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.normal(0, 1, 20000), rng.normal(0, 1e-5, 20000), rng.normal(0, 3e4, 20000),
                        [0.0, -0.0, 65504.0, 65519.0, 65520.0, 6.103515625e-05, 5.960464477539063e-08,
                         2.9802322387695312e-08, 1.00048828125, 1.000732421875]]).astype(np.float32)
    bits, back = O.half_roundtrip(x)
    with np.errstate(over="ignore"):
        ref = x.astype(np.float16)
    assert np.array_equal(bits, ref.view(np.uint16))
    assert np.array_equal(back, ref.astype(np.float32))


def test_mannequin_capsules_are_closed_and_outward():
    b = scenes.mannequin(body_vertices=3000, seed=1)
    V = b["verts"].astype(np.float64)
    T = b["tris"]
    edges = np.sort(np.concatenate([T[:, [0, 1]], T[:, [1, 2]], T[:, [2, 0]]]), axis=1)
    _, cnt = np.unique(edges, axis=0, return_counts=True)
    assert (cnt == 2).all()  # every edge shared by two triangles: closed surfaces
    # outward: the signed volume of each closed capsule is positive
    vol = np.einsum("ij,ij->i", V[T[:, 0]], np.cross(V[T[:, 1]], V[T[:, 2]])).sum() / 6.0
    assert vol > 0.0
    w = b["weights"]
    assert np.allclose(w.sum(0), 1.0, atol=1e-5) and ((w > 0).sum(0) <= 4).all()


def test_pose_cycle_and_tri_sources():
    b = scenes.mannequin(body_vertices=3000, seed=1)
    assert np.allclose(scenes.pose(b, 0), b["frames"])
    assert np.allclose(scenes.pose(b, 120), b["frames"], atol=1e-9)
    p30 = scenes.pose(b, 30)
    delta = [p30[k] @ np.linalg.inv(b["frames"][k]) for k in range(20)]
    r = (delta[7] @ np.linalg.inv(delta[6]))[:3, :3]  # upper arm relative to the clavicle
    assert abs(np.degrees(np.arccos((np.trace(r) - 1) / 2)) - 40.0) < 1e-6  # +-40 degrees at the peak
    w, iw = scenes.shader_mats(p30)
    assert np.allclose(np.einsum("bij,bjk->bik", w, iw), np.eye(4), atol=1e-5)
    bake = {"active_bones": b["names"], "bone_infos": np.zeros((20, 20), np.float32)}
    bake["bone_infos"][:, 0:3] = -10.0
    bake["bone_infos"][:, 4:7] = 10.0
    src, tw = scenes.bone_tri_sources(b, bake)
    assert (np.diff(src[:, 3].astype(np.int64)) >= 0).all()  # grouped by bone
    assert src.shape[0] == tw.shape[0] and (tw.max(1) > 0).all()
