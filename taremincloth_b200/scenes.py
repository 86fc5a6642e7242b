"""Seeded synthetic cloth scenes with the shapes of the benchmark configurations.

* ``config1``: 64 x 64 vertex quad grid, 1 m side, poke-faced (a centre vertex
  per quad, 4 triangles), edges = quad edges only, Y-up with U(+-1 mm) jitter,
  areal density 0.15 kg/m^2, compliance 1e-8 / 1e-5 / 1e-6 (distance /
  bending / shear), two top corners pinned, sphere r = 0.25 m below the centre.
  N = 8,065 vertices, 31,878 distance and 7,812 bending constraints.
* ``config2``: two 256 x 256 sheets (2 triangles per quad, edges = quad edges),
  layer ids 0 / 1, 5 mm apart, 2 mm thickness, dropped onto an icosphere
  (subdivision 5, 20,480 triangles, r = 0.4 m, friction 0.3, thickness 0.01,
  single sided) with self-collision on.  N = 131,072, Nd = 521,220, Nb = 259,080.

All inputs are synthetic (no dataset); the same seed gives the same arrays.
"""
from __future__ import annotations

import numpy as np

F = np.float32


def areal_inv_masses(pos, faces, density):
    """Per-vertex inverse mass from area x density / 3 per triangle, in f32 in
    the operation order of compute_combined_inv_masses
    (crates/cloth_core/src/mesh.rs:237-312)."""
    pos = np.asarray(pos, F)
    faces = np.asarray(faces, np.int64)
    a, b, c = faces[:, 0], faces[:, 1], faces[:, 2]
    ok = (a != b) & (b != c) & (c != a)
    a, b, c = a[ok], b[ok], c[ok]
    ab = pos[b] - pos[a]
    ac = pos[c] - pos[a]
    cx = ab[:, 1] * ac[:, 2] - ab[:, 2] * ac[:, 1]
    cy = ab[:, 2] * ac[:, 0] - ab[:, 0] * ac[:, 2]
    cz = ab[:, 0] * ac[:, 1] - ab[:, 1] * ac[:, 0]
    area = F(0.5) * np.sqrt(cx * cx + cy * cy + cz * cz)
    share = area * F(density) / F(3.0)
    # sequential f32 accumulation in face order (a, b, c of face 0, then face 1, ...)
    order = np.stack([a, b, c], 1).reshape(-1)
    m = np.zeros(len(pos), F)
    np.add.at(m, order, np.repeat(share, 3).astype(F))
    return (F(1.0) / np.maximum(m, F(1e-9))).astype(F)


def quad_grid_edges(nx, ny, idx):
    e = []
    for j in range(ny):
        for i in range(nx - 1):
            e.append((idx[j, i], idx[j, i + 1]))
    for j in range(ny - 1):
        for i in range(nx):
            e.append((idx[j, i], idx[j + 1, i]))
    return np.asarray(e, np.uint32)


def poke_grid(n=64, side=1.0, seed=0, jitter=1e-3, y0=0.0):
    """n x n corner vertices in XZ plus one centre vertex per quad."""
    rng = np.random.default_rng(seed)
    xs = np.linspace(0.0, side, n, dtype=np.float64)
    idx = np.arange(n * n, dtype=np.int64).reshape(n, n)  # [z, x]
    corner = np.zeros((n * n, 3))
    corner[:, 0] = np.tile(xs, n)
    corner[:, 2] = np.repeat(xs, n)
    h = side / (n - 1)
    cidx = n * n + np.arange((n - 1) * (n - 1)).reshape(n - 1, n - 1)
    centre = np.zeros(((n - 1) * (n - 1), 3))
    centre[:, 0] = np.tile(xs[:-1] + 0.5 * h, n - 1)
    centre[:, 2] = np.repeat(xs[:-1] + 0.5 * h, n - 1)
    pos = np.concatenate([corner, centre]).astype(F)
    pos[:, 1] = (y0 + rng.uniform(-jitter, jitter, len(pos))).astype(F)
    faces = []
    for j in range(n - 1):
        for i in range(n - 1):
            a, b, c, d = idx[j, i], idx[j, i + 1], idx[j + 1, i + 1], idx[j + 1, i]
            m = cidx[j, i]
            faces += [(a, b, m), (b, c, m), (c, d, m), (d, a, m)]
    return pos, quad_grid_edges(n, n, idx), np.asarray(faces, np.uint32), idx


def tri_grid(n=256, side=1.0, y=0.0, offset=0, flip=False):
    """n x n vertices in XZ, two triangles per quad, edges = quad edges."""
    xs = np.linspace(0.0, side, n, dtype=np.float64)
    pos = np.zeros((n * n, 3), F)
    pos[:, 0] = np.tile(xs, n)
    pos[:, 1] = y
    pos[:, 2] = np.repeat(xs, n)
    idx = np.arange(n * n, dtype=np.int64).reshape(n, n) + offset
    a = idx[:-1, :-1].reshape(-1)
    b = idx[:-1, 1:].reshape(-1)
    c = idx[1:, 1:].reshape(-1)
    d = idx[1:, :-1].reshape(-1)
    if flip:
        f = np.stack([np.stack([a, c, b], 1), np.stack([a, d, c], 1)], 1).reshape(-1, 3)
    else:
        f = np.stack([np.stack([a, b, c], 1), np.stack([a, c, d], 1)], 1).reshape(-1, 3)
    return pos, quad_grid_edges(n, n, idx), f.astype(np.uint32), idx


def icosphere(subdiv=5, radius=0.4, center=(0.0, 0.0, 0.0)):
    """Icosahedron subdivided `subdiv` times (20 * 4^subdiv triangles), outward winding."""
    t = (1.0 + 5 ** 0.5) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    verts = [np.asarray(p, np.float64) / np.linalg.norm(p) for p in v]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
             (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(subdiv):
        cache = {}
        nf = []

        def mid(i, j):
            k = (min(i, j), max(i, j))
            if k not in cache:
                m = verts[i] + verts[j]
                verts.append(m / np.linalg.norm(m))
                cache[k] = len(verts) - 1
            return cache[k]

        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    V = np.asarray(verts) * radius + np.asarray(center)
    Fc = np.asarray(faces)
    return V[Fc].astype(F)  # (T, 3, 3)


def config1(seed=0):
    pos, edges, faces, idx = poke_grid(64, 1.0, seed)
    inv = areal_inv_masses(pos, faces, 0.15)
    n = 64
    top = [int(idx[n - 1, 0]), int(idx[n - 1, n - 1])]  # max z corners
    return dict(
        name="config1_poke_grid_64", positions=pos, edges=edges, faces=faces, inv_masses=inv,
        thickness=0.005, compliance=(1e-8, 1e-8, 1e-6, 1e-5), gravity=(0.0, -9.81, 0.0),
        pins=[(v, pos[v].copy()) for v in top], spheres=[((0.5, -0.3, 0.5), 0.25, 0.3)],
        mesh=None, self_collision=False, dt=1.0 / 60.0, substeps=10, iterations=5, frames=60)


def config2(n=256, seed=0, side=1.0, subdiv=5):
    """Two stacked sheets over an icosphere.  `n` and `subdiv` shrink it for tests."""
    y0 = 0.45
    p0, e0, f0, _ = tri_grid(n, side, y0, 0)
    p1, e1, f1, _ = tri_grid(n, side, y0 + 0.005, n * n)
    pos = np.concatenate([p0, p1]).astype(F)
    rng = np.random.default_rng(seed)
    pos[:, 1] += rng.uniform(-1e-4, 1e-4, len(pos)).astype(F)
    edges = np.concatenate([e0, e1])
    faces = np.concatenate([f0, f1])
    layers = np.concatenate([np.zeros(n * n, np.uint32), np.ones(n * n, np.uint32)])
    inv = areal_inv_masses(pos, faces, 0.15)
    tris = icosphere(subdiv, 0.4, (0.5 * side, 0.0, 0.5 * side))
    return dict(
        name=f"config2_two_sheets_{n}", positions=pos, edges=edges, faces=faces, inv_masses=inv,
        layer_ids=layers, thickness=0.002, compliance=(1e-8, 1e-8, 1e-6, 1e-5), gravity=(0.0, -9.81, 0.0),
        pins=[], spheres=[], mesh=dict(triangles=tris, friction=0.3, thickness=0.01, single_sided=True),
        self_collision=True, dt=1.0 / 60.0, substeps=20, iterations=4, frames=30)


def build(sim_cls, scene, **kw):
    """Construct a simulator (product or oracle) from a scene dict."""
    s = sim_cls(scene["positions"], scene["edges"], scene["faces"], scene["inv_masses"],
                layer_ids=scene.get("layer_ids"), thickness=scene["thickness"], **kw)
    s.set_gravity(*scene["gravity"])
    s.set_compliance_all(*scene["compliance"])
    s.set_enable_self_collision(scene["self_collision"])
    s.set_solver_iterations(scene["iterations"])
    for v, t in scene["pins"]:
        s.set_pin(v, t, 1.0)
    for c, r, f in scene["spheres"]:
        s.add_sphere_collider(c, r, friction=f)
    if scene["mesh"] is not None:
        m = scene["mesh"]
        s.set_mesh_collider_triangles(m["triangles"], friction=m["friction"], thickness=m["thickness"],
                                      single_sided=m["single_sided"])
    return s


def config4(n_instances=64, seed=0, side_range=(32, 192)):
    """Uneven batch: grid sides log-uniform in side_range (1 cm spacing, two
    triangles per quad, edges = quad edges), 2-8 pinned boundary vertices,
    compliance log-uniform in [1e-9, 1e-5], 1-3 sphere / capsule colliders
    below each cloth at seeded poses."""
    rng = np.random.default_rng(seed)
    lo, hi = side_range
    instances = []
    for k in range(n_instances):
        u = rng.uniform()
        side = int(lo * (hi / lo) ** u)
        h = 0.01
        L = (side - 1) * h
        pos, edges, faces, idx = tri_grid(side, L, 0.0)
        pos = pos.astype(F)
        pos[:, 1] += rng.uniform(-1e-4, 1e-4, len(pos)).astype(F)
        inv = areal_inv_masses(pos, faces, 0.15)
        boundary = np.unique(np.concatenate([idx[0], idx[-1], idx[:, 0], idx[:, -1]]))
        pins = rng.choice(boundary, size=int(rng.integers(2, 9)), replace=False)
        c = float(10.0 ** rng.uniform(-9.0, -5.0))
        cols = []
        for _ in range(int(rng.integers(1, 4))):
            r = float(rng.uniform(0.1, 0.3)) * L
            ctr = (float(rng.uniform(0.3, 0.7) * L), float(-r - rng.uniform(0.01, 0.2) * L),
                   float(rng.uniform(0.3, 0.7) * L))
            if rng.uniform() < 0.5:
                cols.append(("sphere", ctr, r, float(rng.uniform(0.1, 0.5))))
            else:
                a = (ctr[0] - 0.3 * L, ctr[1], ctr[2])
                b = (ctr[0] + 0.3 * L, ctr[1], ctr[2] + 0.1 * L)
                cols.append(("capsule", a, b, 0.5 * r, float(rng.uniform(0.1, 0.5))))
        instances.append(dict(positions=pos, edges=edges, faces=faces, inv_masses=inv,
                              compliance=(c, c, c * 100.0, 1e-5), colliders=cols,
                              pins=[(int(v), pos[int(v)].copy()) for v in pins]))
    return dict(name=f"config4_batch_{n_instances}", instances=instances, thickness=0.005,
                gravity=(0.0, -9.81, 0.0), dt=1.0 / 60.0, substeps=10, iterations=5)


def build_batch(scene, device=0):
    from .simulator import BatchedClothSimulator
    s = BatchedClothSimulator(scene["instances"], thickness=scene["thickness"], device=device)
    s.set_gravity(*scene["gravity"])
    s.set_solver_iterations(scene["iterations"])
    for k, inst in enumerate(scene["instances"]):
        for v, t in inst["pins"]:
            s.set_pin(int(s.offsets[k]) + v, t, 1.0)
    return s


def build_instance(sim_cls, scene, k, **kw):
    """One instance of a batch scene as its own simulator (oracle or product)."""
    inst = scene["instances"][k]
    s = sim_cls(inst["positions"], inst["edges"], inst["faces"], inst["inv_masses"], thickness=scene["thickness"],
                layer_ids=np.zeros(len(inst["positions"]), np.uint32), **kw)
    s.set_gravity(*scene["gravity"])
    s.set_compliance_all(*inst["compliance"])
    s.set_enable_self_collision(False)
    s.set_solver_iterations(scene["iterations"])
    for v, t in inst["pins"]:
        s.set_pin(v, t, 1.0)
    for c in inst["colliders"]:
        if c[0] == "sphere":
            s.add_sphere_collider(c[1], c[2], friction=c[3])
        else:
            s.add_capsule_collider(c[1], c[2], c[3], friction=c[4])
    return s
