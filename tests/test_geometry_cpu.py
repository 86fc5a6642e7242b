"""find_triangle_intersections (host only, no GPU) against the pair lists the
reference's own finder (python/taremin_cloth/analysis.py:638-760) produced on
the seeded meshes of tests/golden/make_intersection_fixtures.py: two crossing
sheets, a crumpled sheet, a sheet folded through itself, the crossing sheets
with sewn vertex clusters, and the reference's case-4 drape with jitter."""
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "intersections.npz")
NAMES = ["crossing", "crumpled", "folded", "crossing_sewn", "drape_jitter"]


@pytest.mark.parametrize("name", NAMES)
def test_matches_reference_finder(name):
    import taremin_cloth_core as core
    d = np.load(GOLDEN)
    sew = d[f"{name}_sew"] if f"{name}_sew" in d.files else None
    got = core.find_triangle_intersections(d[f"{name}_pos"], d[f"{name}_faces"], sewing_springs=sew)
    want = [tuple(int(v) for v in r) for r in d[f"{name}_pairs"]]
    assert got == want


def test_adjacency_and_degenerate_faces():
    import taremin_cloth_core as core
    pos = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0.2, 0.2, -0.5], [0.2, 0.2, 0.5], [0.6, 0.1, 0.0]],
                   np.float32)
    # face 1 pierces face 0; face 2 is degenerate; face 3 shares vertex 0 with face 0
    faces = np.array([[0, 1, 2], [3, 4, 5], [1, 1, 2], [0, 3, 4]], np.uint32)
    assert core.find_triangle_intersections(pos, faces) == [(0, 1)]
    # without the adjacency rule the pair sharing vertex 0 counts too
    assert (0, 3) in core.find_triangle_intersections(pos, faces, ignore_adjacent=False)
    assert core.find_triangle_intersections(pos, np.zeros((0, 3), np.uint32)) == []
    with pytest.raises(ValueError):
        core.find_triangle_intersections(pos[:, :2], faces)
