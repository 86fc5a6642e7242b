"""The reference's analytic simulator tests, restated as scenarios that run on
any simulator class with the drop-in interface (the CUDA path's
ClothSimulator or the oracle's OracleSim).

Each scenario builds the reference test's mesh with the same constructor
arguments (ClothMesh::from_raw: positions, edges, faces, inv_masses,
layer_ids, thicknesses, default thickness, tension / compression / shear /
bending stiffness), runs the same steps and returns the quantities the
reference asserts on, plus the final positions so that two implementations
can be compared.  Sources (crates/cloth_core/src/simulation/tests.rs unless
named):

  mesh_triangle_collision          :150-203
  mesh_triangle_single_sided       :205-264
  compliant_pin                    :556-634
  self_collision_options           :322-390
  boundary_ee_ccd                  :1124-1205
  one_sided_boundary_ee_ccd        :1207-1297
  vt_ccd_moving_triangle           :1299-1374
  internal_ee_ccd                  :1627-1740
  internal_ee_low_speed_crossover  :1742-1802
  folded_hinge                     :1804-1888
  double_hit_no_dilution           :1890-1948
  discrete_untangling_rotation     :1950-2006
  air_damping                      :2470-2537
  rayleigh_stretch / rayleigh_bend :2539-2670
  static_pin_edge                  :2672-2731
  pair_cache_ee_ccd                :2733-2790
  collision_departure              :2792-2887
  untangle_wrinkled_inner          :3081-3185
  untangle_face_to_face            :3187-3324
  strand_escape                    :3326-3423
  self_collision_symmetry          tests/core/test_self_collision_symmetry.py:63-173
  edge_rest_length_scaling         :266-320
"""
import numpy as np

_f32 = np.float32


def _mk(cls, positions, edges, faces=None, inv_masses=None, layer_ids=None, thicknesses=None, thickness=0.02,
        tension=10000.0, compression=10000.0, shear=5000.0, bending=0.0):
    pos = np.asarray(positions, _f32).reshape(-1, 3)
    e = np.asarray(edges, np.uint32).reshape(-1, 2)
    kw = dict(thickness=thickness, stiffness=tension, compression_stiffness=compression, shear_stiffness=shear,
              bending_stiffness=bending)
    if faces is not None:
        kw["faces"] = np.asarray(faces, np.uint32).reshape(-1, 3)
    if inv_masses is not None:
        kw["inv_masses"] = np.asarray(inv_masses, _f32)
    if layer_ids is not None:
        kw["layer_ids"] = np.asarray(layer_ids, np.uint32)
    if thicknesses is not None:
        kw["thicknesses"] = np.asarray(thicknesses, _f32)
    return cls(pos, e, **kw)


def _pair_cache_off(s):
    if hasattr(s, "set_enable_pair_cache"):
        s.set_enable_pair_cache(False)
    else:
        s.set_pair_cache(False)


def _pair_cache_on(s):
    if hasattr(s, "set_enable_pair_cache"):
        s.set_self_collision_algorithm(1)
        s.set_enable_pair_cache(True)
    else:
        s.set_pair_cache(True)


def _state(s):
    x, _, v = s.get_state()
    return x.astype(np.float64), v.astype(np.float64)


def _tri(p0, p1, p2):
    return np.array([[p0, p1, p2]], _f32)


# --------------------------------------------------------------------------
# mesh-triangle collider (collision.wgsl mesh path)

def mesh_triangle_collision(cls):
    s = _mk(cls, [[0.0, 0.0, 0.5]], np.zeros((0, 2)))
    s.set_mesh_collider_triangles(_tri([-1, -1, 0], [1, -1, 0], [0, 1, 0]), friction=0.2, thickness=0.02,
                                  restitution=0.0, single_sided=False)
    for _ in range(60):
        s.step(1.0 / 60.0, 20)
    x, _ = _state(s)
    return dict(z=x[0, 2], x=x)


def mesh_triangle_single_sided(cls):
    s = _mk(cls, [[0.0, 0.0, -0.1]], np.zeros((0, 2)))
    s.set_mesh_collider_triangles(_tri([-1, -1, 0], [1, -1, 0], [0, 1, 0]), friction=0.2, thickness=0.02,
                                  restitution=0.0, single_sided=True)
    for _ in range(10):
        s.step(1.0 / 60.0, 20)
    x, _ = _state(s)
    return dict(z=x[0, 2], x=x)


def collision_departure(cls):
    """Contact push-out without normal acceleration, then a 1 m jump through a
    small triangle whose both end points lie outside its bounding sphere,
    with and without cluster culling (simulation/tests.rs:2792-2887)."""
    s = _mk(cls, [[0.0, 0.0, 0.005]], np.zeros((0, 2)))
    s.set_gravity(0.0, 0.0, 0.0)
    s.set_damping(0.0)
    s.set_mesh_collider_triangles(_tri([-1, -1, 0], [1, -1, 0], [0, 1, 0]), friction=0.0, thickness=0.02,
                                  restitution=0.0, single_sided=False)
    s.set_positions_and_velocities(np.array([[0.0, 0.0, 0.005]], _f32), np.array([[0.0, 0.0, 1.0]], _f32))
    s.step(1.0 / 60.0, 1)
    x, v = _state(s)
    out = dict(z_dep=x[0, 2], vz_dep=v[0, 2], x=x)
    small = [[-0.1, -0.1, 0.0], [0.1, -0.1, 0.0], [0.0, 0.1, 0.0]]
    far = [[10.0, 10.0, 10.0], [10.1, 10.0, 10.0], [10.0, 10.1, 10.0]]
    for cluster in (False, True):
        s2 = _mk(cls, [[0.0, 0.0, 0.5]], np.zeros((0, 2)), thickness=0.01)
        s2.set_gravity(0.0, 0.0, 0.0)
        s2.set_damping(0.0)
        s2.set_collider_options(cluster, False, 0.0)
        tris = np.array([small] + ([far] * 32 if cluster else []), _f32)
        s2.set_mesh_collider_triangles(tris, friction=0.0, thickness=0.01, restitution=0.0, single_sided=False)
        s2.set_positions_and_velocities(np.array([[0.0, 0.0, 0.5]], _f32), np.array([[0.0, 0.0, -60.0]], _f32))
        s2.step(1.0 / 60.0, 1)
        out[f"z_seg_{int(cluster)}"] = _state(s2)[0][0, 2]
    return out


# --------------------------------------------------------------------------
# pins (pin.wgsl compliant pin)

def compliant_pin(cls, weight, frames):
    s = _mk(cls, [[0, 0, 0], [1, 0, 0], [2, 0, 0]], [[0, 1], [1, 2]], inv_masses=[0.0, 1.0, 0.0],
            thickness=0.005, tension=1000.0, compression=1000.0, shear=5000.0)
    s.set_gravity(0.0, 0.0, 0.0)
    s.set_pin(1, [1.0, 0.5, 0.0], weight)
    for _ in range(frames):
        s.step(1.0 / 60.0, 20)
    x, _ = _state(s)
    return dict(y1=x[1, 1], x=x)


# --------------------------------------------------------------------------
# self-collision (self_collision*.wgsl, direct path)

def self_collision_options(cls):
    pos = [[0, 0, 0], [0.1, 0, 0], [0, 0.1, 0], [0.1, 0.1, 0]]
    s = _mk(cls, pos, [[0, 1], [1, 2], [2, 0], [1, 3], [3, 2]], faces=[[0, 1, 2], [2, 1, 3]], thickness=0.02,
            tension=1000.0, compression=1000.0, shear=1000.0, bending=10.0)
    s.set_gravity(0.0, 0.0, 0.0)
    s.set_enable_self_collision(True)
    s.set_self_collision_options(0.1, 0.2, True, True, 256)
    for _ in range(10):
        s.step(1.0 / 60.0, 10)
    x, _ = _state(s)
    return dict(x=x)


_PANELS = dict(
    positions=[[-0.03, 0.0, 0.0], [-0.03, 0.1, 0.0], [-0.10, 0.05, 0.0],
               [0.03, 0.0, 0.0], [0.03, 0.1, 0.0], [0.10, 0.05, 0.0]],
    edges=[[0, 1], [1, 2], [2, 0], [3, 4], [4, 5], [5, 3]],
    faces=[[0, 1, 2], [3, 4, 5]])


def boundary_ee_ccd(cls):
    s = _mk(cls, _PANELS["positions"], _PANELS["edges"], faces=_PANELS["faces"], thickness=0.01)
    s.set_enable_self_collision(True)
    s.set_gravity(0.0, 0.0, 0.0)
    vel = np.array([[5, 0, 0]] * 3 + [[-5, 0, 0]] * 3, _f32)
    s.set_positions_and_velocities(np.asarray(_PANELS["positions"], _f32), vel)
    s.step(1.0 / 60.0, 10)
    x, _ = _state(s)
    return dict(xa0=x[0, 0], xa1=x[1, 0], xb0=x[3, 0], xb1=x[4, 0], x=x)


def one_sided_boundary_ee_ccd(cls):
    pos = [[-0.03, 0.0, 0.05], [-0.03, 0.1, 0.05], [-0.10, 0.05, 0.05], [0.03, 0.0, 0.05], [0.03, 0.1, 0.05],
           [0.08, 0.05, 0.00], [0.08, 0.05, 0.10]]
    edges = [[0, 1], [1, 2], [2, 0], [3, 4], [4, 5], [5, 3], [3, 6], [6, 4]]
    s = _mk(cls, pos, edges, faces=[[0, 1, 2], [3, 4, 5], [3, 6, 4]], thickness=0.01)
    e, bits = s.get_edges() if hasattr(s, "get_edges") else s.edges()
    k = int(np.nonzero((np.minimum(e[:, 0], e[:, 1]) == 3) & (np.maximum(e[:, 0], e[:, 1]) == 4))[0][0])
    open_34 = bool((int(bits[k >> 5]) >> (k & 31)) & 1)
    s.set_enable_self_collision(True)
    s.set_gravity(0.0, 0.0, 0.0)
    vel = np.array([[5, 0, 0]] * 3 + [[-5, 0, 0]] * 4, _f32)
    s.set_positions_and_velocities(np.asarray(pos, _f32), vel)
    s.step(1.0 / 60.0, 10)
    x, _ = _state(s)
    return dict(open_34=open_34, xa0=x[0, 0], xa1=x[1, 0], xb0=x[3, 0], xb1=x[4, 0], x=x)


def vt_ccd_moving_triangle(cls):
    pos = [[-0.05, -0.05, 0.04], [0.05, -0.05, 0.04], [0.0, 0.05, 0.04], [0.0, 0.0, 0.0], [0.02, 0.0, 0.0]]
    s = _mk(cls, pos, [[0, 1], [1, 2], [2, 0], [3, 4]], faces=[[0, 1, 2]], thickness=0.01)
    s.set_enable_self_collision(True)
    s.set_gravity(0.0, 0.0, 0.0)
    vel = np.array([[0, 0, -4]] * 3 + [[0, 0, 2]] * 2, _f32)
    s.set_positions_and_velocities(np.asarray(pos, _f32), vel)
    s.step(1.0 / 60.0, 10)
    x, _ = _state(s)
    return dict(z_tri=x[:3, 2].mean(), z_pt3=x[3, 2], x=x)


def _roof_pair(z_b):
    """Two orthogonal internal-edge roofs (simulation/tests.rs:1627-1676)."""
    pos = [[-1.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 0.3, -0.5], [0.0, -0.3, -0.5],
           [0.0, -1.0, z_b], [0.0, 1.0, z_b], [0.3, 0.0, z_b + 0.5], [-0.3, 0.0, z_b + 0.5]]
    edges = [[0, 1], [1, 2], [2, 0], [0, 3], [3, 1], [4, 5], [5, 6], [6, 4], [4, 7], [7, 5]]
    faces = [[0, 1, 2], [1, 0, 3], [4, 5, 6], [5, 4, 7]]
    return pos, edges, faces


def _edge_open(s, a, b):
    e, bits = s.get_edges() if hasattr(s, "get_edges") else s.edges()
    k = int(np.nonzero((np.minimum(e[:, 0], e[:, 1]) == a) & (np.maximum(e[:, 0], e[:, 1]) == b))[0][0])
    return bool((int(bits[k >> 5]) >> (k & 31)) & 1)


def _roof_drop(cls, z_b, vz, thickness=0.005, inv_masses=None, pair_cache=False):
    pos, edges, faces = _roof_pair(z_b)
    s = _mk(cls, pos, edges, faces=faces, inv_masses=inv_masses, thickness=thickness)
    opens = (_edge_open(s, 0, 1), _edge_open(s, 4, 5))
    s.set_enable_self_collision(True)
    if pair_cache:
        _pair_cache_on(s)
    else:
        _pair_cache_off(s)
    s.set_gravity(0.0, 0.0, 0.0)
    vel = np.array([[0, 0, 0]] * 4 + [[0, 0, vz]] * 4, _f32)
    s.set_positions_and_velocities(np.asarray(pos, _f32), vel)
    s.step(1.0 / 60.0, 1)
    x, _ = _state(s)
    return dict(opens=opens, z_mid_a=0.5 * (x[0, 2] + x[1, 2]), z_mid_b=0.5 * (x[4, 2] + x[5, 2]), x=x)


def internal_ee_ccd(cls):
    return _roof_drop(cls, 0.008, -1.2)


def internal_ee_low_speed_crossover(cls):
    return _roof_drop(cls, 0.002, -0.24)


def static_pin_edge(cls):
    return _roof_drop(cls, 0.008, -1.2, inv_masses=[0, 0, 0, 0, 1, 1, 1, 1])


def pair_cache_ee_ccd(cls):
    z_b = 0.006
    pos = [[-0.05, 0.0, 0.0], [0.05, 0.0, 0.0], [0.0, 0.03, -0.05], [0.0, -0.03, -0.05],
           [0.0, -0.05, z_b], [0.0, 0.05, z_b], [0.03, 0.0, z_b + 0.05], [-0.03, 0.0, z_b + 0.05]]
    _, edges, faces = _roof_pair(z_b)
    s = _mk(cls, pos, edges, faces=faces, thickness=0.005)
    s.set_enable_self_collision(True)
    _pair_cache_on(s)
    s.set_gravity(0.0, 0.0, 0.0)
    vel = np.array([[0, 0, 0]] * 4 + [[0, 0, -0.9]] * 4, _f32)
    s.set_positions_and_velocities(np.asarray(pos, _f32), vel)
    s.step(1.0 / 60.0, 1)
    x, _ = _state(s)
    return dict(z_mid_a=0.5 * (x[0, 2] + x[1, 2]), z_mid_b=0.5 * (x[4, 2] + x[5, 2]), x=x)


def folded_hinge(cls):
    pos, edges, faces = [], [], []
    for iy in range(3):
        y = iy * 0.05
        pos += [[0.0, y, 0.005], [0.05, y, 0.0], [0.0, y, -0.005]]
    for iy in range(3):
        b = iy * 3
        edges += [[b, b + 1], [b + 1, b + 2]]
        if iy + 1 < 3:
            edges += [[b + ix, b + 3 + ix] for ix in range(3)]
            for ix in range(2):
                a, bb, c, d = b + ix, b + ix + 1, b + 3 + ix + 1, b + 3 + ix
                faces += [[a, bb, c], [a, c, d]]
    s = _mk(cls, pos, edges, faces=faces, thickness=0.004, tension=5000.0, compression=5000.0, shear=2500.0)
    s.set_enable_self_collision(True)
    _pair_cache_off(s)
    s.set_gravity(0.0, 0.0, 0.0)
    for _ in range(20):
        s.step(1.0 / 60.0, 5)
    x, _ = _state(s)
    return dict(max_disp=float(np.linalg.norm(x - np.asarray(pos), axis=1).max()), x=x)


def double_hit_no_dilution(cls):
    z_b = 0.008
    pos = [[-0.02, -0.012, 0.0], [0.02, -0.012, 0.0], [0.0, -0.006, -0.02], [0.0, -0.018, -0.02],
           [-0.02, 0.012, 0.0], [0.02, 0.012, 0.0], [0.0, 0.018, -0.02], [0.0, 0.006, -0.02],
           [0.0, -0.02, z_b], [0.0, 0.02, z_b], [0.006, 0.0, z_b + 0.02], [-0.006, 0.0, z_b + 0.02]]
    edges = [[0, 1], [1, 2], [2, 0], [0, 3], [3, 1], [4, 5], [5, 6], [6, 4], [4, 7], [7, 5],
             [8, 9], [9, 10], [10, 8], [8, 11], [11, 9]]
    faces = [[0, 1, 2], [1, 0, 3], [4, 5, 6], [5, 4, 7], [8, 9, 10], [9, 8, 11]]
    s = _mk(cls, pos, edges, faces=faces, thickness=0.005)
    s.set_enable_self_collision(True)
    _pair_cache_off(s)
    s.set_gravity(0.0, 0.0, 0.0)
    vel = np.array([[0, 0, 0]] * 8 + [[0, 0, -1.5]] * 4, _f32)
    s.set_positions_and_velocities(np.asarray(pos, _f32), vel)
    s.step(1.0 / 60.0, 1)
    x, _ = _state(s)
    return dict(z_a1=0.5 * (x[0, 2] + x[1, 2]), z_a2=0.5 * (x[4, 2] + x[5, 2]), z_b=0.5 * (x[8, 2] + x[9, 2]), x=x)


def discrete_untangling_rotation(cls, rotate):
    pos, edges, faces = _roof_pair(-0.003)
    pos = [[p[0], -p[1], -p[2]] if rotate else p for p in pos]
    s = _mk(cls, pos, edges, faces=faces, layer_ids=[0, 0, 0, 0, 1, 1, 1, 1], thickness=0.005)
    s.set_enable_self_collision(True)
    _pair_cache_off(s)
    s.set_gravity(0.0, 0.0, 0.0)
    s.step(1.0 / 60.0, 1)
    x, _ = _state(s)
    z = 0.5 * (x[4, 2] + x[5, 2])
    return dict(z_outer=-z if rotate else z, x=x)


# --------------------------------------------------------------------------
# damping (predict.wgsl air damping; distance/bending Rayleigh terms)

def air_damping(cls, air, internal):
    s = _mk(cls, [[0, 0, 10], [1, 0, 10]], [[0, 1]], inv_masses=[1.0, 1.0], thickness=0.005, tension=1000.0,
            compression=1000.0, shear=500.0, bending=10.0)
    s.set_gravity(0.0, 0.0, -9.81)
    s.set_damping(air)
    s.set_damping_all(*internal)
    for _ in range(60):
        s.step(1.0 / 60.0, 10)
    x, v = _state(s)
    return dict(vz=v[0, 2], x=x)


def air_damping_expected():
    """The reference's closed form for one air-damping application per
    substep, iterated in f32 (simulation/tests.rs:2495-2499)."""
    dt_sub = _f32(1.0 / 60.0) / _f32(10.0)
    vz = _f32(0.0)
    for _ in range(600):
        vz = vz * max(_f32(1.0) - _f32(2.0) * dt_sub, _f32(0.0)) + _f32(-9.81) * dt_sub
    return float(vz)


def rayleigh_stretch(cls, substeps, damp):
    s = _mk(cls, [[0, 0, 0], [1, 0, 0]], [[0, 1]], inv_masses=[0.0, 50.0], thickness=0.005, tension=200.0,
            compression=200.0, shear=200.0, bending=10.0)
    s.set_gravity(0.0, 0.0, 0.0)
    s.set_damping(0.0)
    s.set_damping_all(damp, damp, 0.0, 0.0)
    s.set_positions_and_velocities(np.array([[0, 0, 0], [1.2, 0, 0]], _f32), None)
    tail = 0.0
    for frame in range(90):
        s.step(1.0 / 60.0, substeps)
        if frame >= 60:
            tail = max(tail, abs(_state(s)[1][1, 0]))
    return dict(tail=tail, x=_state(s)[0])


def rayleigh_bend(cls, damp):
    pos = [[0, 0, 0], [0, 1, 0], [-1, 0.5, 0], [0, 0.5, 1]]
    s = _mk(cls, pos, [[0, 1], [0, 2], [1, 2], [0, 3], [1, 3]], faces=[[0, 1, 2], [1, 0, 3]],
            inv_masses=[0.0, 0.0, 0.0, 500.0], thickness=0.005, tension=5000.0, compression=5000.0, shear=500.0,
            bending=150.0)
    s.set_gravity(0.0, 0.0, 0.0)
    s.set_damping(0.0)
    s.set_damping_all(0.0, 0.0, 0.0, damp)
    phi = _f32(0.35)
    s.set_positions_and_velocities(np.array([[0, 0, 0], [0, 1, 0], [-1, 0.5, 0],
                                             [np.sin(phi), 0.5, np.cos(phi)]], _f32), None)
    tail = 0.0
    for frame in range(90):
        s.step(1.0 / 60.0, 20)
        if frame >= 60:
            tail = max(tail, abs(_state(s)[1][3, 0]))
    return dict(tail=tail, x=_state(s)[0])


# --------------------------------------------------------------------------
# multi-layer untangling (self_collision_untangle.wgsl, layer guards)

def _grid_layer(nx, ny, dx, base, z_of, flip=False, ox=2.0, oy=2.0):
    pos, edges, faces = [], [], []
    for iy in range(ny):
        for ix in range(nx):
            pos.append([(ix - ox) * dx, (iy - oy) * dx, z_of(ix, iy)])
    for iy in range(ny):
        for ix in range(nx):
            v0 = base + iy * nx + ix
            if ix + 1 < nx:
                edges.append([v0, v0 + 1])
            if iy + 1 < ny:
                edges.append([v0, v0 + nx])
            if ix + 1 < nx and iy + 1 < ny:
                v1, v2, v3 = v0 + 1, v0 + nx + 1, v0 + nx
                edges.append([v0, v2])
                faces += [[v0, v2, v1], [v0, v3, v2]] if flip else [[v0, v1, v2], [v0, v2, v3]]
    return pos, edges, faces


def untangle_wrinkled_inner(cls):
    nx = ny = 5
    dx = 0.02
    pos, edges, faces, layers, inv = [], [], [], [], []
    for layer in (0, 1):
        def z_of(ix, iy, layer=layer):
            w = 0.012 if ix == 2 else (0.004 if ix in (1, 3) else 0.0)
            return w + (0.003 if layer == 1 else 0.0)
        p, e, f = _grid_layer(nx, ny, dx, len(pos), z_of)
        for iy in range(ny):
            for ix in range(nx):
                layers.append(layer)
                border = ix in (0, nx - 1) or iy in (0, ny - 1)
                inv.append(0.0 if border else 1.0)
        pos += p
        edges += e
        faces += f
    s = _mk(cls, pos, edges, faces=faces, inv_masses=inv, layer_ids=layers, thickness=0.0014, tension=1500.0,
            compression=150.0, shear=100.0, bending=15.0)
    s.set_gravity(0.0, 0.0, 0.0)
    s.set_damping(2.0)
    s.set_enable_self_collision(True)
    s.set_self_collision_options(1.0, 0.5, True, True, 512)
    for _ in range(10):
        s.step(1.0 / 60.0, 10)
    x, _ = _state(s)
    per = nx * ny
    return dict(z_in=x[:per, 2], z_out=x[per:, 2], z_out0=np.asarray(pos)[per:, 2], x=x)


def _point_in_tri_xy(px, py, a, b, c):
    """Height of the triangle at (px, py) when the point lies inside its XY
    projection, with the reference test's 1e-3 barycentric slack
    (simulation/tests.rs:3274-3294); None otherwise."""
    v0x, v0y = b[0] - a[0], b[1] - a[1]
    v1x, v1y = c[0] - a[0], c[1] - a[1]
    det = v0x * v1y - v1x * v0y
    if abs(det) < 1e-10:
        return None
    qx, qy = px - a[0], py - a[1]
    u = (qx * v1y - v1x * qy) / det
    v = (v0x * qy - qx * v0y) / det
    w = 1.0 - u - v
    if u >= -1e-3 and v >= -1e-3 and w >= -1e-3:
        return w * a[2] + u * b[2] + v * c[2]
    return None


def untangle_face_to_face(cls):
    dx = 0.02
    p0, e0, f0 = _grid_layer(7, 7, dx, 0, lambda ix, iy: 0.0, ox=3.0, oy=3.0)
    base1 = len(p0)
    p1, e1, f1 = _grid_layer(5, 5, dx, base1, lambda ix, iy: 0.006, flip=True)
    inv0 = [0.0 if (ix in (0, 6) or iy in (0, 6)) else 1.0 for iy in range(7) for ix in range(7)]
    pos = p0 + p1
    layers = [0] * base1 + [1] * len(p1)
    inv = inv0 + [1.0] * len(p1)
    vel = np.array([[0, 0, 0]] * base1 + [[0, 0, -0.5]] * len(p1), _f32)
    s = _mk(cls, pos, e0 + e1, faces=f0 + f1, inv_masses=inv, layer_ids=layers, thickness=0.002, tension=1500.0,
            compression=150.0, shear=100.0, bending=15.0)
    s.set_positions_and_velocities(np.asarray(pos, _f32), vel)
    s.set_gravity(0.0, 0.0, -9.81)
    s.set_damping(1.0)
    s.set_enable_self_collision(True)
    s.set_self_collision_options(1.0, 0.5, True, True, 512)
    for _ in range(15):
        s.step(1.0 / 60.0, 15)
    x, _ = _state(s)
    gaps = []
    for i in range(base1, len(pos)):
        tz = None
        for t in f0:
            tz = _point_in_tri_xy(x[i, 0], x[i, 1], x[t[0]], x[t[1]], x[t[2]])
            if tz is not None:
                break
        gaps.append(np.nan if tz is None else x[i, 2] - tz)
    return dict(gaps=np.asarray(gaps), x=x)


def strand_escape(cls):
    nx = ny = 5
    dx = 0.006
    pos, edges, faces = _grid_layer(nx, ny, dx, 0, lambda ix, iy: 0.0)
    layers = [0] * len(pos)
    inv = [0.0 if (ix in (0, nx - 1) or iy in (0, ny - 1)) else 200000.0 for iy in range(ny) for ix in range(nx)]
    thick = [0.0014] * len(pos)
    base = len(pos)
    for i in range(5):
        pos.append([(i - 2.0) * dx, 0.0, 0.0025 if i in (0, 4) else -0.0018])
        layers.append(1)
        inv.append(40000.0)
        thick.append(0.0022)
    edges += [[base + i, base + i + 1] for i in range(4)]
    s = _mk(cls, pos, edges, faces=faces, inv_masses=inv, layer_ids=layers, thicknesses=thick, thickness=0.0014,
            tension=1500.0, compression=150.0, shear=100.0, bending=15.0)
    s.set_gravity(0.0, 0.0, 0.0)
    s.set_damping(2.0)
    s.set_enable_self_collision(True)
    s.set_self_collision_options(1.0, 0.5, True, True, 512)
    for _ in range(5):
        s.step(1.0 / 60.0, 15)
    x, _ = _state(s)
    return dict(z_strand=x[base:, 2], x=x)


# --------------------------------------------------------------------------
# action / reaction (tests/core/test_self_collision_symmetry.py)

def self_collision_symmetry(cls, inv_top, inv_bottom):
    nx = ny = 3
    dx = 0.05
    pos, inv, edges, faces = [], [], [], []
    for z, w in ((-0.01, inv_bottom), (0.01, inv_top)):
        for y in range(ny):
            for x in range(nx):
                pos.append([x * dx, y * dx, z])
                inv.append(w)
    for off in (0, nx * ny):
        for y in range(ny):
            for x in range(nx):
                i = off + y * nx + x
                if x + 1 < nx:
                    edges.append([i, i + 1])
                if y + 1 < ny:
                    edges.append([i, i + nx])
                if x + 1 < nx and y + 1 < ny:
                    faces += [[i, i + 1, i + nx + 1], [i, i + nx + 1, i + nx]]
    s = cls(np.asarray(pos, _f32), np.asarray(edges, np.uint32), faces=np.asarray(faces, np.uint32),
            inv_masses=np.asarray(inv, _f32), layer_id=0, thickness=0.015, stiffness=10000.0)
    s.set_gravity(0.0, 0.0, 0.0)
    s.set_enable_self_collision(True)
    s.set_self_collision_options(relief_factor=1.0, max_displacement_ratio=1.0, exclude_neighbors=True,
                                 enable_normal_untangling=False, max_iterations=128)
    s.step_single_substep(0.005)
    x, _ = _state(s)
    d = x[:, 2] - np.asarray(pos)[:, 2]
    return dict(bottom=float(d[:nx * ny].sum()), top=float(d[nx * ny:].sum()), x=x)


# --------------------------------------------------------------------------
# bone SDF collider (collision.wgsl bone phase; simulation/tests.rs:443-554)

def bone_plane_atlas(size=16):
    """16^3 atlas of one bone over [-0.5, 0.5]^3 whose distance is the texel
    centre's z (f16 distance, f16 alpha 1), and its 20-float bone info
    (AABB, uvw scale with blend 0.05, uvw offset, friction 0.3, thickness
    0.02)."""
    z = -0.5 + (np.arange(size) + 0.5) / size
    d = np.repeat(z.astype(np.float16), size * size).view(np.uint16).astype(np.uint32)
    alpha = np.uint32(np.float16(1.0).view(np.uint16))
    tex = (d | (alpha << np.uint32(16))).astype(np.uint32)
    info = np.array([[-0.5, -0.5, -0.5, 0.0, 0.5, 0.5, 0.5, 0.0, 1.0, 1.0, 1.0, 0.05,
                      0.5, 0.5, 0.5, 0.0, 0.3, 0.02, 0.0, 0.0]], _f32)
    return tex, info


def bone_mats(dz):
    """(world, inverse world) of a bone translated by dz along z, as the
    shaders store them (translation in the last column)."""
    w = np.eye(4, dtype=_f32)[None].copy()
    w[0, 3, 2] = dz
    iw = np.eye(4, dtype=_f32)[None].copy()
    iw[0, 3, 2] = -dz
    return w, iw
