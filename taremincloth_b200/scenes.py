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


def sewn_garment(n=24, side=0.3, gap=0.06, seed=0):
    """Front and back panels (n x n vertices each, two triangles per quad,
    hanging in XY, `gap` apart in Z) sewn along both side columns into a
    tube; the top corners of each panel pinned; self-collision on."""
    rng = np.random.default_rng(seed)
    ps, es, fs = [], [], []
    for k in range(2):
        p, e, f, idx = tri_grid(n, side, 0.0, k * n * n, flip=k == 1)
        q = np.zeros_like(p)
        q[:, 0] = p[:, 0]
        q[:, 1] = 1.0 - p[:, 2]          # rows hang downwards from y = 1
        q[:, 2] = k * gap
        ps.append(q)
        es.append(e)
        fs.append(f)
    pos = np.concatenate(ps).astype(F)
    pos[:, 2] += rng.uniform(-1e-4, 1e-4, len(pos)).astype(F)
    grid = np.arange(n * n).reshape(n, n)
    sides = np.concatenate([grid[:, 0], grid[:, -1]])
    sewing = np.stack([sides, sides + n * n], 1).astype(np.uint32)
    faces = np.concatenate(fs)
    inv = areal_inv_masses(pos, faces, 0.15)
    pins = []
    for k in range(2):
        for v in (int(grid[0, 0]) + k * n * n, int(grid[0, -1]) + k * n * n):
            pins.append((v, pos[v].copy()))
    return dict(
        name=f"sewn_garment_{n}", positions=pos, edges=np.concatenate(es), faces=faces, inv_masses=inv,
        layer_ids=None, thickness=0.002, compliance=(1e-8, 1e-8, 1e-6, 1e-5), gravity=(0.0, -9.81, 0.0),
        pins=pins, spheres=[], mesh=None, self_collision=True, dt=1.0 / 60.0, substeps=10, iterations=4,
        frames=12, sewing=sewing, sewing_shrink_speed=0.5)


def build(sim_cls, scene, **kw):
    """Construct a simulator (product or oracle) from a scene dict."""
    if scene.get("sewing") is not None:
        kw.setdefault("sewing_springs", scene["sewing"])
        kw.setdefault("sewing_shrink_speed", scene.get("sewing_shrink_speed", 1.0))
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


# ---------------------------------------------------------------------------
# config 3: capsule-chain mannequin with a dynamic bone SDF, cylinder garment
# ---------------------------------------------------------------------------
# (name, parent, start, end, radius): a 20-bone chain, Y up, metres
_BONES = (
    ("pelvis", -1, (0.0, 0.95, 0.0), (0.0, 1.05, 0.0), 0.13),
    ("spine1", 0, (0.0, 1.05, 0.0), (0.0, 1.17, 0.0), 0.12),
    ("spine2", 1, (0.0, 1.17, 0.0), (0.0, 1.29, 0.0), 0.12),
    ("spine3", 2, (0.0, 1.29, 0.0), (0.0, 1.41, 0.0), 0.13),
    ("neck", 3, (0.0, 1.41, 0.0), (0.0, 1.52, 0.0), 0.05),
    ("head", 4, (0.0, 1.52, 0.0), (0.0, 1.72, 0.0), 0.09),
    ("clav_l", 3, (0.03, 1.40, 0.0), (0.18, 1.40, 0.0), 0.05),
    ("uarm_l", 6, (0.18, 1.40, 0.0), (0.45, 1.40, 0.0), 0.05),
    ("farm_l", 7, (0.45, 1.40, 0.0), (0.70, 1.40, 0.0), 0.04),
    ("hand_l", 8, (0.70, 1.40, 0.0), (0.80, 1.40, 0.0), 0.035),
    ("clav_r", 3, (-0.03, 1.40, 0.0), (-0.18, 1.40, 0.0), 0.05),
    ("uarm_r", 10, (-0.18, 1.40, 0.0), (-0.45, 1.40, 0.0), 0.05),
    ("farm_r", 11, (-0.45, 1.40, 0.0), (-0.70, 1.40, 0.0), 0.04),
    ("hand_r", 12, (-0.70, 1.40, 0.0), (-0.80, 1.40, 0.0), 0.035),
    ("thigh_l", 0, (0.09, 0.95, 0.0), (0.09, 0.52, 0.0), 0.07),
    ("shin_l", 14, (0.09, 0.52, 0.0), (0.09, 0.10, 0.0), 0.05),
    ("foot_l", 15, (0.09, 0.10, 0.0), (0.09, 0.05, 0.14), 0.04),
    ("thigh_r", 0, (-0.09, 0.95, 0.0), (-0.09, 0.52, 0.0), 0.07),
    ("shin_r", 17, (-0.09, 0.52, 0.0), (-0.09, 0.10, 0.0), 0.05),
    ("foot_r", 18, (-0.09, 0.10, 0.0), (-0.09, 0.05, 0.14), 0.04),
)


def _bone_frame(a, b):
    """Rest transform (bone local -> world, 4x4 row-major): origin at a, local +y along a->b."""
    a = np.asarray(a, np.float64)
    y = np.asarray(b, np.float64) - a
    y /= np.linalg.norm(y)
    ref = np.array([0.0, 0.0, 1.0]) if abs(y[2]) < 0.9 else np.array([1.0, 0.0, 0.0])
    x = np.cross(y, ref)
    x /= np.linalg.norm(x)
    z = np.cross(x, y)
    T = np.eye(4)
    T[:3, 0], T[:3, 1], T[:3, 2], T[:3, 3] = x, y, z, a
    return T


def _capsule_mesh(radius, length, n_around, n_along, n_cap):
    """Closed capsule around the local +y axis from y=0 to y=length."""
    rings = []
    for k in range(n_cap, 0, -1):  # bottom cap
        phi = 0.5 * np.pi * k / n_cap
        rings.append((-radius * np.sin(phi), radius * np.cos(phi)))
    for k in range(n_along + 1):
        rings.append((length * k / n_along, radius))
    for k in range(1, n_cap + 1):  # top cap
        phi = 0.5 * np.pi * k / n_cap
        rings.append((length + radius * np.sin(phi), radius * np.cos(phi)))
    th = 2.0 * np.pi * np.arange(n_around) / n_around
    verts = [(0.0, -radius, 0.0)]
    for y, r in rings:
        for t in th:
            verts.append((r * np.cos(t), y, r * np.sin(t)))
    verts.append((0.0, length + radius, 0.0))
    V = np.asarray(verts, np.float64)
    tris = []
    nr = len(rings)
    for j in range(n_around):
        tris.append((0, 1 + (j + 1) % n_around, 1 + j))
    for i in range(nr - 1):
        b0, b1 = 1 + i * n_around, 1 + (i + 1) * n_around
        for j in range(n_around):
            j1 = (j + 1) % n_around
            tris.append((b0 + j, b0 + j1, b1 + j))
            tris.append((b0 + j1, b1 + j1, b1 + j))
    top = len(verts) - 1
    last = 1 + (nr - 1) * n_around
    for j in range(n_around):
        tris.append((last + j, last + (j + 1) % n_around, top))
    return V, np.asarray(tris, np.int64)[:, [0, 2, 1]]  # counter-clockwise seen from outside


def mannequin(body_vertices=30000, seed=0):
    """20 capsules (closed meshes), ~body_vertices vertices in total, with 4
    seeded skin weights per vertex (own bone, parent, child, noise).
    Returns verts (N,3) f32, tris (M,3) i32, weights (20, N) f32, bind_inv
    (20,4,4) row-major mesh -> bone local, rest frames (20,4,4), parents."""
    rng = np.random.default_rng(seed)
    nb = len(_BONES)
    lengths = [np.linalg.norm(np.subtract(b[3], b[2])) for b in _BONES]
    areas = np.array([2 * np.pi * b[4] * (L + 2 * b[4]) for b, L in zip(_BONES, lengths)])
    per = np.maximum(areas / areas.sum() * body_vertices, 64)
    V_all, T_all, owner, along = [], [], [], []
    frames = np.zeros((nb, 4, 4))
    off = 0
    for b, (name, parent, a, e, r) in enumerate(_BONES):
        L = lengths[b]
        # spacing h with n_around * (n_along + 2 n_cap) ~ per[b]
        h = np.sqrt(2 * np.pi * r * (L + np.pi * r) / per[b])
        n_around = max(8, int(round(2 * np.pi * r / h)))
        n_along = max(2, int(round(L / h)))
        n_cap = max(2, int(round(0.5 * np.pi * r / h)))
        V, T = _capsule_mesh(r, L, n_around, n_along, n_cap)
        Tf = _bone_frame(a, e)
        frames[b] = Tf
        Vw = (Tf[:3, :3] @ V.T).T + Tf[:3, 3]
        V_all.append(Vw)
        T_all.append(T + off)
        owner.append(np.full(len(V), b))
        along.append(np.clip(V[:, 1] / L, 0.0, 1.0))
        off += len(V)
    verts = np.concatenate(V_all).astype(F)
    tris = np.concatenate(T_all).astype(np.int32)
    owner = np.concatenate(owner)
    along = np.concatenate(along)
    children = [[c for c in range(nb) if _BONES[c][1] == b] for b in range(nb)]
    W = np.zeros((nb, len(verts)), np.float64)
    for i in range(len(verts)):
        b = owner[i]
        w = {b: 1.0}
        p = _BONES[b][1]
        if p >= 0:
            w[p] = w.get(p, 0.0) + max(0.0, 0.5 - along[i]) * 0.8
        for c in children[b][:1]:
            w[c] = w.get(c, 0.0) + max(0.0, along[i] - 0.5) * 0.8
        other = int(rng.integers(0, nb))
        w[other] = w.get(other, 0.0) + float(rng.uniform(0.0, 0.015))  # below the 0.02 AABB threshold
        top = sorted(w.items(), key=lambda kv: -kv[1])[:4]
        s = sum(v for _, v in top)
        for k, v in top:
            W[k, i] = v / s
    bind_inv = np.stack([np.linalg.inv(frames[b]) for b in range(nb)]).astype(F)
    return dict(verts=verts, tris=tris, weights=W.astype(F), bind_inv=bind_inv, frames=frames,
                parents=[b[1] for b in _BONES], names=[b[0] for b in _BONES])


def _rot(axis, ang):
    axis = np.asarray(axis, np.float64) / np.linalg.norm(axis)
    x, y, z = axis
    c, s = np.cos(ang), np.sin(ang)
    C = 1 - c
    R = np.eye(4)
    R[:3, :3] = [[c + x * x * C, x * y * C - z * s, x * z * C + y * s],
                 [y * x * C + z * s, c + y * y * C, y * z * C - x * s],
                 [z * x * C - y * s, z * y * C + x * s, c + z * z * C]]
    return R


# joints driven by the pose cycle: (bone, world axis at rest, phase sign)
_POSE = ((7, (0, 0, 1), 1.0), (11, (0, 0, 1), -1.0), (14, (1, 0, 0), 1.0), (17, (1, 0, 0), -1.0),
         (2, (0, 0, 1), 0.25), (8, (0, 1, 0), 0.5), (12, (0, 1, 0), -0.5))


def pose(body, frame, period=120, amplitude_deg=40.0):
    """World transforms (bone local -> world, row-major) at `frame` of the
    sinusoidal ping-pong cycle: +-amplitude about each driven joint."""
    ang = np.deg2rad(amplitude_deg) * np.sin(2.0 * np.pi * frame / period)
    frames, parents = body["frames"], body["parents"]
    nb = len(parents)
    local = {}
    for b, axis, sign in _POSE:
        a = np.asarray(_BONES[b][2], np.float64)
        Tm, Tp = np.eye(4), np.eye(4)
        Tm[:3, 3], Tp[:3, 3] = -a, a
        local[b] = Tp @ _rot(axis, sign * ang) @ Tm  # rotation about the joint, world axes at rest
    M = np.zeros((nb, 4, 4))
    for b in range(nb):  # parents come first in _BONES
        p = parents[b]
        Pw = np.eye(4) if p < 0 else M[p] @ np.linalg.inv(frames[p])  # parent's world delta
        D = local.get(b, np.eye(4))
        M[b] = Pw @ D @ frames[b]
    return M


def shader_mats(M):
    """(world, inverse world) as the shaders store them: the transposes of the row-major matrices."""
    M = np.asarray(M, np.float64)
    return (np.ascontiguousarray(np.transpose(M, (0, 2, 1))).astype(F),
            np.ascontiguousarray(np.transpose(np.linalg.inv(M), (0, 2, 1))).astype(F))


def bone_tri_sources(body, bake):
    """Per active bone (in the bake's order), the triangles with a weighted
    vertex whose bind-pose bone-local AABB overlaps the bone's padded AABB
    (the static baker's rule, sdf_baker.rs:632-700); (M,4) u32 and (M,3) f32."""
    verts, tris, W, bind = body["verts"], body["tris"], body["weights"], body["bind_inv"]
    src, tw = [], []
    names = body["names"]
    for ob, nm in enumerate(bake["active_bones"]):
        b = names.index(nm)
        info = bake["bone_infos"][ob]
        mn, mx = info[0:3], info[4:7]
        wt = W[b][tris]                                 # (M, 3)
        has = (wt > 0).any(1)
        Pl = (np.c_[verts, np.ones(len(verts), F)] @ bind[b].T.astype(np.float64))[:, :3]
        tp = Pl[tris]                                   # (M, 3, 3)
        tmin, tmax = tp.min(1), tp.max(1)
        ov = (tmin <= mx).all(1) & (tmax >= mn).all(1) & has
        idx = np.nonzero(ov)[0]
        src.append(np.c_[tris[idx], np.full(len(idx), ob)])
        tw.append(wt[idx])
    return np.concatenate(src).astype(np.uint32), np.concatenate(tw).astype(F)


def cylinder_garment(radius=0.18, height=0.7, edge=0.0028, center=(0.0, 0.62, 0.0), seed=0):
    """Open tube around the body's y axis, edge ~`edge`, alternating
    diagonals, seeded jitter (a structured stand-in for an isotropic remesh)."""
    rng = np.random.default_rng(seed)
    na = int(round(2 * np.pi * radius / edge))
    nh = int(round(height / edge)) + 1
    th = 2 * np.pi * np.arange(na) / na
    ys = center[1] + np.linspace(0.0, height, nh)
    pos = np.zeros((nh, na, 3), np.float64)
    pos[:, :, 0] = center[0] + radius * np.cos(th)[None, :]
    pos[:, :, 2] = center[2] + radius * np.sin(th)[None, :]
    pos[:, :, 1] = ys[:, None]
    pos += rng.uniform(-0.1, 0.1, pos.shape) * edge
    idx = np.arange(nh * na).reshape(nh, na)
    faces, edges = [], set()
    for i in range(nh - 1):
        for j in range(na):
            j1 = (j + 1) % na
            a, b, c, d = idx[i, j], idx[i, j1], idx[i + 1, j], idx[i + 1, j1]
            if (i + j) % 2 == 0:
                faces += [(a, b, d), (a, d, c)]
            else:
                faces += [(a, b, c), (b, d, c)]
    faces = np.asarray(faces, np.uint32)
    for f in faces:
        for u, v in ((f[0], f[1]), (f[1], f[2]), (f[2], f[0])):
            edges.add((min(u, v), max(u, v)))
    edges = np.asarray(sorted(edges), np.uint32)
    return pos.reshape(-1, 3).astype(F), edges, faces, idx


def config3(body_vertices=30000, garment_edge=0.0028, resolution=64, seed=0):
    """~100k-vertex tube garment (r 0.18 m, h 0.7 m) around a 20-bone capsule
    mannequin (~30k vertices, 4 weights per vertex) with a dynamic bone SDF
    atlas (per-bone res^3 tiles, fp16 distance + alpha), top ring pinned,
    floor plane; bones follow a +-40 degree sinusoid over 120 frames."""
    body = mannequin(body_vertices, seed)
    pos, edges, faces, idx = cylinder_garment(edge=garment_edge, seed=seed)
    inv = areal_inv_masses(pos, faces, 0.15)
    top = idx[-1]
    return dict(name="config3_garment_bone_sdf", body=body, positions=pos, edges=edges, faces=faces,
                inv_masses=inv, thickness=0.002, compliance=(1e-8, 1e-8, 1e-6, 1e-5), gravity=(0.0, -9.81, 0.0),
                pins=[(int(v), pos[int(v)].copy()) for v in top], resolution=resolution,
                dt=1.0 / 60.0, substeps=10, iterations=4, period=120)


def build_config3(sim_cls, scene, bake=None, device=0):
    """Simulator with the garment, pins, floor, and the dynamic bone SDF set up
    from a GPU bake of the mannequin (returns (sim, bake))."""
    from .simulator import bake_bone_sdf_gpu
    body = scene["body"]
    if bake is None:
        bake = bake_bone_sdf_gpu(body["verts"], body["tris"], body["names"], list(body["weights"]),
                                 body["bind_inv"], resolution=scene["resolution"], device=device)
    s = sim_cls(scene["positions"], scene["edges"], scene["faces"], scene["inv_masses"],
                thickness=scene["thickness"], device=device)
    s.set_gravity(*scene["gravity"])
    s.set_compliance_all(*scene["compliance"])
    s.set_enable_self_collision(False)
    s.set_solver_iterations(scene["iterations"])
    for v, t in scene["pins"]:
        s.set_pin(v, t, 1.0)
    s.add_plane_collider((0.0, 0.0, 0.0), (0.0, 1.0, 0.0), friction=0.5)
    src, tw = bone_tri_sources(body, bake)
    names = body["names"]
    order = [names.index(nm) for nm in bake["active_bones"]]
    W = body["weights"][order]                            # active bones only
    top = np.argsort(-W, axis=0)[:4].T                    # (N, 4) bone slots
    bw = np.take_along_axis(W.T, top, axis=1)
    res = int(bake["bone_infos"][0][7])
    s.setup_dynamic_bone_sdf(bake["width"], bake["height"], bake["depth"], res, bake["bone_infos"],
                             body["verts"], top.astype(np.uint32), bw.astype(F), src, tw,
                             body["bind_inv"][order], update_interval=1)
    return s, bake, order
