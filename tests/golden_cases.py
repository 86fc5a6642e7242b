"""The reference's golden-master cases (tests/regression/test_single_step_exact.py:46-140,
test_golden_regression.py:76-300): constructor arguments and colliders per case."""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def areal_inv_masses(pos, faces, density):
    """float64 areal masses, as the reference's fixture regeneration does."""
    masses = np.zeros(len(pos), dtype=np.float64)
    for f in np.asarray(faces, dtype=np.int64):
        a, b, c = int(f[0]), int(f[1]), int(f[2])
        if a == b or b == c or c == a:
            continue
        ab = pos[b].astype(np.float64) - pos[a].astype(np.float64)
        ac = pos[c].astype(np.float64) - pos[a].astype(np.float64)
        share = 0.5 * float(np.linalg.norm(np.cross(ab, ac))) * density / 3.0
        masses[a] += share
        masses[b] += share
        masses[c] += share
    return (1.0 / np.maximum(masses, 1e-9)).astype(np.float32)


CASES = {
    "case1": dict(file="case1_cloth_body.npz", stiffness=1500.0, bending=15.0, density=None, colliders=[],
                  short=(10, 1e-3), full=10e-3, com=10e-3),
    "case2": dict(file="case2_plane_sphere.npz", stiffness=1200.0, bending=5.0, density=None,
                  colliders=[("sphere", ([0.0, 0.0, 0.16], 0.14), dict(friction=0.4, restitution=0.0))],
                  short=(10, 1e-3), full=15e-3, com=15e-3),
    "case3": dict(file="case3_multi_collider.npz", stiffness=1000.0, bending=10.0, density=0.15,
                  colliders=[("capsule", ([-0.3, -0.3, 0.4], [0.3, -0.3, 0.5], 0.08), dict(friction=0.4)),
                             ("capsule", ([-0.3, 0.3, 0.5], [0.3, 0.3, 0.4], 0.08), dict(friction=0.4)),
                             ("sphere", ([0.0, 0.0, 0.3], 0.12), dict(friction=0.5)),
                             ("plane", ([0.0, 0.0, 0.0], [0.0, 0.0, 1.0]), dict(friction=0.6))],
                  short=(10, 1e-3), full=None, com=25e-3),
    "case4": dict(file="case4_self_collision_drape.npz", stiffness=800.0, bending=5.0, density=0.10,
                  colliders=[("sphere", ([0.0, 0.0, 0.2], 0.20), dict(friction=0.6))],
                  sc=dict(relief_factor=1.0, max_displacement_ratio=0.5, exclude_neighbors=True,
                          enable_normal_untangling=True, max_iterations=256),
                  short=(5, 5e-3), full=None, com=20e-3),
}


def load(case):
    c = CASES[case]
    d = np.load(os.path.join(GOLDEN, c["file"]))
    pos = d["initial_pos"]
    inv = d["inv_masses"] if "inv_masses" in d.files else areal_inv_masses(pos, d["faces"], c["density"])
    return c, d, pos, inv


def make(sim_cls, case, positions=None):
    c, d, pos, inv = load(case)
    s = sim_cls(positions if positions is not None else pos, d["edges"], d["faces"], inv, thickness=0.005,
                stiffness=c["stiffness"], bending_stiffness=c["bending"])
    s.set_gravity(0.0, 0.0, -9.81)
    if "sc" in c:
        s.set_enable_self_collision(True)
        s.set_self_collision_options(**c["sc"])
    for kind, args, kw in c["colliders"]:
        getattr(s, f"add_{kind}_collider")(*args, **kw)
    return s


def step_input(case):
    """(pos_in, pos_out) of the one-frame golden pair."""
    c, d, pos, inv = load(case)
    sd = np.load(os.path.join(GOLDEN, f"step_{case}_f1.npz"))
    pin = sd["pos_in"] if "pos_in" in sd.files else pos
    return pin, sd["pos_out"]


def _edge_len(p, e):
    e = np.asarray(e, np.int64)
    return np.linalg.norm(p[e[:, 0]] - p[e[:, 1]], axis=1)


def _segment_distance(points, a, b):
    """Smallest distance of the points to segment ab
    (test_golden_regression.py:53-66)."""
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    ab = b - a
    ap = points.astype(np.float64) - a
    t = np.clip(ap @ ab / float(ab @ ab), 0.0, 1.0)
    return float(np.linalg.norm(points - (a + t[:, None] * ab), axis=1).min())


# the reference's per-case strain limits (test_golden_regression.py:123, :176, :238, :297)
STRAIN = {"case1": 1.15, "case2": 1.15, "case3": 1.20, "case4": 1.25}


def golden_trajectory(sim_cls, case):
    """Steps a simulator through a golden case and checks every criterion of
    the reference's test_golden_regression.py:76-300 except case 2's
    all-frame bound (test_case2_all_frame_bound).  Returns the largest
    all-frame vertex error."""
    import taremin_cloth_core as core
    c, d, pos, inv = load(case)
    s = make(sim_cls, case)
    gp = d["positions"]
    rest = _edge_len(pos, d["edges"])
    nshort, tol_short = c["short"]
    worst = 0.0
    a = None
    for fi in range(1, len(gp)):
        s.step(1.0 / 60.0, 20, 2)
        out = np.empty(len(pos) * 3, np.float32)
        s.get_positions(out)
        a = out.reshape(-1, 3)
        assert not np.isnan(a).any()
        diff = float(np.linalg.norm(a - gp[fi], axis=1).max())
        worst = max(worst, diff)
        if fi <= nshort:
            assert diff < tol_short, f"{case} frame {fi}: {diff * 1e3:.4f} mm"
        if c["full"] is not None and case != "case2":
            assert diff < c["full"], f"{case} frame {fi}: {diff * 1e3:.4f} mm over all frames"
        com = float(np.linalg.norm(a.mean(0) - gp[fi].mean(0)))
        assert com < c["com"], f"{case} frame {fi}: centre of mass {com * 1e3:.3f} mm"
        strain = float((_edge_len(a, d["edges"]) / np.maximum(rest, 1e-6)).max())
        assert strain < STRAIN[case], f"{case} frame {fi}: strain {strain:.4f}"
        if case == "case1":
            pinned = inv == 0.0
            assert float(np.linalg.norm(a[pinned] - pos[pinned], axis=1).max()) < 1e-5
        if case == "case2":
            assert float(np.linalg.norm(a - np.array([0, 0, 0.16], np.float32), axis=1).min()) >= 0.14 - 0.002
        if case == "case3":
            assert float(a[:, 2].min()) >= -0.002
            assert float(np.linalg.norm(a - np.array([0, 0, 0.3], np.float32), axis=1).min()) >= 0.12 - 0.003
            assert _segment_distance(a, [-0.3, -0.3, 0.4], [0.3, -0.3, 0.5]) >= 0.08 - 0.003
            assert _segment_distance(a, [-0.3, 0.3, 0.5], [0.3, 0.3, 0.4]) >= 0.08 - 0.003
        if case == "case4":
            assert float(np.linalg.norm(a - np.array([0, 0, 0.2], np.float32), axis=1).min()) >= 0.20 - 0.003
            if fi >= 20:
                n_x = len(core.find_triangle_intersections(a, d["faces"]))
                assert n_x <= 12, f"case4 frame {fi}: {n_x} self-intersections"
    if case == "case4":
        n_x = len(core.find_triangle_intersections(a, d["faces"]))
        assert n_x <= 2, f"case4 final frame: {n_x} self-intersections"
    return worst
