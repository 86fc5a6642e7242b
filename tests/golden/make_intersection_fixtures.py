"""Golden self-intersection lists from the reference's own finder.

Runs the reference's NumPy find_triangle_intersections
(python/taremin_cloth/analysis.py:638-760, the Python twin of
crates/cloth_core/src/geometry.rs:627-633) on seeded meshes built here and
stores meshes and pair lists in tests/golden/intersections.npz.  Run once in
a container where the reference checkout is mounted:
    python tests/golden/make_intersection_fixtures.py <reference checkout>
"""
import importlib.util
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def grid(nx, ny, dx, base=0):
    """Vertices (ix * dx, iy * dx, 0) and two triangles per quad."""
    pos = np.array([[ix * dx, iy * dx, 0.0] for iy in range(ny) for ix in range(nx)], np.float64)
    faces = []
    for iy in range(ny - 1):
        for ix in range(nx - 1):
            v0 = base + iy * nx + ix
            faces += [[v0, v0 + 1, v0 + nx + 1], [v0, v0 + nx + 1, v0 + nx]]
    return pos, np.array(faces, np.int64)


def cases():
    rng = np.random.default_rng(20261204)
    out = {}
    # two sheets crossing at right angles
    a, fa = grid(12, 12, 0.01)
    b, fb = grid(12, 12, 0.01, base=len(a))
    b = b[:, [0, 2, 1]] + np.array([0.003, 0.052, -0.047])
    out["crossing"] = (np.vstack([a, b]), np.vstack([fa, fb]), None)
    # a sheet with seeded 3D noise of about one edge length (a height field
    # never intersects itself, so the noise moves x and y too)
    c, fc = grid(16, 16, 0.01)
    c += rng.uniform(-0.012, 0.012, c.shape)
    out["crumpled"] = (c, fc, None)
    # a sheet folded back through itself
    d, fd = grid(20, 10, 0.01)
    x = d[:, 0].copy()
    fold = x > 0.1
    ang = np.deg2rad(172.0)
    d[fold, 0] = 0.1 + (x[fold] - 0.1) * np.cos(ang)
    d[fold, 2] = (x[fold] - 0.1) * np.sin(ang) - 0.004 * (x[fold] - 0.1) / 0.09
    d[:, 2] += rng.uniform(-0.002, 0.002, len(d))
    out["folded"] = (d, fd, None)
    # the crossing sheets with sewing springs joining a few vertex pairs
    p, f, _ = out["crossing"]
    # (vertex 60 + i of the flat sheet lies on the crossing line, 204 + i of
    # the upright one next to it)
    sew = np.array([[60 + i, 204 + i] for i in (2, 6, 9)], np.int64)
    out["crossing_sewn"] = (p, f, sew)
    # the reference's case 4 drape, last golden frame, with seeded jitter
    g = np.load(os.path.join(HERE, "case4_self_collision_drape.npz"))
    q = g["positions"][-1].astype(np.float64) + rng.normal(0.0, 0.015, g["positions"][-1].shape)
    out["drape_jitter"] = (q, g["faces"].astype(np.int64), None)
    return out


def main(ref_root):
    spec = importlib.util.spec_from_file_location(
        "reference_analysis", os.path.join(ref_root, "python", "taremin_cloth", "analysis.py"))
    analysis = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(analysis)
    if getattr(analysis, "_RUST_GEOMETRY", False):
        sys.exit("the reference's compiled core is importable; this script records its NumPy path only")
    store = {}
    for name, (pos, faces, sew) in cases().items():
        pos = pos.astype(np.float32)
        faces = faces.astype(np.uint32)
        pairs = analysis.find_triangle_intersections(pos, faces, sewing_springs=sew)
        pairs = np.array(sorted(pairs), np.uint32).reshape(-1, 2)
        store[f"{name}_pos"] = pos
        store[f"{name}_faces"] = faces
        store[f"{name}_pairs"] = pairs
        if sew is not None:
            store[f"{name}_sew"] = sew.astype(np.uint32)
        print(f"{name}: {len(faces)} faces, {len(pairs)} intersecting pairs")
    np.savez_compressed(os.path.join(HERE, "intersections.npz"), **store)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_intersection_fixtures.py <reference checkout root>")
    main(sys.argv[1])
