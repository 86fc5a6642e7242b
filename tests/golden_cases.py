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
