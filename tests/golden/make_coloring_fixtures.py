"""Golden Welsh-Powell colourings from the reference's own Python colouring.

The reference's log tool colours a log's distance or sewing constraints
(python/taremin_cloth/log_tools.py:553-640, cmd_render_coloring).  Without
the compiled core it runs its in-tree Python Welsh-Powell (:609-636), the
twin of crates/cloth_core/src/coloring.rs:6-79 / :180-233: order the pairs
by (adjacent-pair degree desc, index asc), give each the first colour not
used by a pair sharing a vertex.

This script writes each seeded pair list as a one-frame log in the format
the tool reads (python/taremin_cloth/replayer.py:28-63), runs
cmd_render_coloring on it with the image step replaced by a no-op, takes
the tool's per-pair colour list from its frame when it returns, and stores
pair lists and colours in tests/golden/coloring.npz.  The reference package
is loaded without its Blender-only package initialiser, and the compiled
core is replaced by an empty module so that the Python colouring runs.  Run
once in a container where the reference checkout is mounted:
    python tests/golden/make_coloring_fixtures.py <reference checkout>
"""
import argparse
import gzip
import json
import os
import sys
import tempfile
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def grid_edges(nx, ny, base=0):
    """Unique edges of an nx x ny grid with one diagonal per quad."""
    out = []
    for iy in range(ny):
        for ix in range(nx):
            v = base + iy * nx + ix
            if ix + 1 < nx:
                out.append((v, v + 1))
            if iy + 1 < ny:
                out.append((v, v + nx))
            if ix + 1 < nx and iy + 1 < ny:
                out.append((v, v + nx + 1))
    return out


def cases():
    """name -> (num_vertices, pairs (k, 2) uint32, kind); pairs of "distance"
    cases are unique unordered pairs without self-loops (a mesh's edges),
    "sewing" cases join two sheets, "pairs" cases are free pair lists."""
    rng = np.random.default_rng(20261204)
    out = {}
    e = np.array(grid_edges(9, 7), np.uint32)
    e = e[rng.permutation(len(e))]
    flip = rng.random(len(e)) < 0.5
    e[flip] = e[flip][:, ::-1]
    out["grid_distance"] = (63, e, "distance")
    n = 48
    seen, pairs = set(), []
    while len(pairs) < 140:
        a, b = (int(x) for x in rng.integers(0, n, 2))
        if a != b and (min(a, b), max(a, b)) not in seen:
            seen.add((min(a, b), max(a, b)))
            pairs.append((a, b))
    out["random_distance"] = (n, np.array(pairs, np.uint32), "distance")
    # two 6 x 6 sheets, the left column of the second sewn to the right
    # column of the first, plus a few diagonal springs sharing vertices
    sew = [(iy * 6 + 5, 36 + iy * 6) for iy in range(6)]
    sew += [(iy * 6 + 5, 36 + (iy + 1) * 6) for iy in range(5)]
    sew += [(0, 36), (0, 41), (35, 71)]
    out["two_sheet_sewing"] = (72, np.array(sew, np.uint32), "sewing")
    # free pair lists: repeats, both orientations, a hub of high degree
    m = 30
    a, b = rng.integers(0, m, 90), rng.integers(0, m, 90)
    keep = a != b
    out["random_pairs"] = (m, np.stack([a, b], 1)[keep].astype(np.uint32), "pairs")
    hub = [(0, k) for k in range(1, 25)] + [(k, k + 1) for k in range(1, 24)] + [(3, 7), (7, 3), (5, 20)]
    out["hub_pairs"] = (25, np.array(hub, np.uint32), "pairs")
    return out


def load_log_tools(ref):
    core = types.ModuleType("taremin_cloth_core")
    core.ClothSimulator = object  # annotation target only; no colouring here
    sys.modules["taremin_cloth_core"] = core
    pkg = types.ModuleType("taremin_cloth")
    pkg.__path__ = [os.path.join(ref, "python", "taremin_cloth")]
    sys.modules["taremin_cloth"] = pkg
    import taremin_cloth.log_tools as lt  # noqa: E402
    lt.mesh_renderer.render_scene_to_file = lambda *a, **k: None
    return lt


def reference_colours(lt, num_vertices, pairs, kind, tmp):
    meta = dict(num_vertices=int(num_vertices), faces=[], edges=[], sewing_springs=[])
    meta["sewing_springs" if kind == "sewing" else "edges"] = pairs.tolist()
    path = os.path.join(tmp, "log.jsonl.gz")
    with gzip.open(path, "wt", encoding="utf-8") as f:
        f.write(json.dumps(dict(record_type="metadata", metadata=meta)) + "\n")
        pos = np.zeros(3 * num_vertices).tolist()
        f.write(json.dumps(dict(record_type="frame", frame_index=0, positions=pos)) + "\n")
    args = argparse.Namespace(log_file=path, output=os.path.join(tmp, "out.png"),
                              type="sewing" if kind == "sewing" else "distance", frame=0, width=16, height=16)
    seen = {}

    def tracer(frame, event, arg):
        if frame.f_code is lt.cmd_render_coloring.__code__:
            if event == "return":
                seen["colors"] = list(frame.f_locals["colors"])
            return tracer
        return None

    sys.settrace(tracer)
    try:
        lt.cmd_render_coloring(args)
    finally:
        sys.settrace(None)
    return np.array(seen["colors"], np.uint32)


def main():
    if len(sys.argv) != 2:
        sys.exit(__doc__)
    lt = load_log_tools(sys.argv[1])
    store = {}
    with tempfile.TemporaryDirectory() as tmp:
        for name, (n, pairs, kind) in cases().items():
            col = reference_colours(lt, n, pairs, kind, tmp)
            assert len(col) == len(pairs)
            store[f"{name}/n"] = np.uint32(n)
            store[f"{name}/pairs"] = pairs
            store[f"{name}/kind"] = np.array(kind)
            store[f"{name}/colors"] = col
            print(name, kind, len(pairs), "pairs,", int(col.max()) + 1, "colours")
    np.savez_compressed(os.path.join(HERE, "coloring.npz"), **store)


if __name__ == "__main__":
    main()
