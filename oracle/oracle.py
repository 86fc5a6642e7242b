"""ctypes wrapper around the CPU oracle (``oracle/_build/libtcloth_oracle.so``).

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()``
and the CPU-baseline leg of ``bench.py``.  The product never imports it.

``OracleSim`` mirrors the constructor and setters of the reference's
``taremin_cloth_core.ClothSimulator`` (crates/cloth_py/src/lib.rs:1556-1767)
so parity tests read like the reference's own tests.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libtcloth_oracle.so")
_lib = None

_f = np.float32
_u = np.uint32


def build() -> str:
    """Compile the oracle with its Makefile (gcc, -ffp-contract=off)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        P = C.c_void_p
        fp = np.ctypeslib.ndpointer(dtype=_f, flags="C_CONTIGUOUS")
        up = np.ctypeslib.ndpointer(dtype=_u, flags="C_CONTIGUOUS")
        L.ocl_create.restype = P
        L.ocl_create.argtypes = [P, C.c_int, P, C.c_int, P, C.c_int, P, P, P, C.c_uint32,
                                 C.c_float, C.c_float, C.c_float, C.c_float, C.c_float]
        L.ocl_create_sewn.restype = P
        L.ocl_create_sewn.argtypes = [P, C.c_int, P, C.c_int, P, C.c_int, P, P, P, C.c_uint32,
                                      C.c_float, C.c_float, C.c_float, C.c_float, C.c_float, P, C.c_int, C.c_float]
        L.ocl_set_sewing.argtypes = [P, C.c_float, C.c_int, C.c_float, C.c_float]
        L.ocl_get_sewing.argtypes = [P, P, P, P, P, P, P]
        L.ocl_get_sewing.restype = C.c_int
        L.ocl_get_bending_gate.argtypes = [P, fp]
        L.ocl_bake_mesh_sdf.argtypes = [P, C.c_int, P, C.c_int, C.c_float, C.c_float, C.c_float, C.c_float,
                                         C.c_float, P, P, P]
        L.ocl_bake_mesh_sdf_coarse.argtypes = [P, C.c_int, P, C.c_int, C.c_float, C.c_float, C.c_float, P, P, P, P]
        L.ocl_bake_mesh_sdf_hier.argtypes = [P, C.c_int, P, C.c_int, C.c_float, C.c_float, C.c_float, C.c_float,
                                             C.c_float, P, P, P]
        L.ocl_bake_mesh_sdf_hier.restype = C.c_int
        L.ocl_set_edge_collision.argtypes = [P, C.c_int, C.c_float, C.c_float]
        L.ocl_num_collider_edges.argtypes = [P]
        L.ocl_num_collider_edges.restype = C.c_int
        L.ocl_destroy.argtypes = [P]
        for name, n in [("ocl_set_gravity", 3), ("ocl_set_damping_all", 4), ("ocl_set_compliance_all", 4)]:
            getattr(L, name).argtypes = [P] + [C.c_float] * n
        L.ocl_set_damping.argtypes = [P, C.c_float]
        L.ocl_set_solver_iterations.argtypes = [P, C.c_int]
        L.ocl_set_enable_self_collision.argtypes = [P, C.c_int]
        L.ocl_set_coupled_collider.argtypes = [P, C.c_int]
        L.ocl_set_collider_options.argtypes = [P, C.c_int, C.c_int, C.c_float]
        L.ocl_set_pair_recording.argtypes = [P, C.c_int]
        L.ocl_get_pair_lists.argtypes = [P, P, C.c_size_t, P, C.c_size_t, P]
        L.ocl_set_self_collision_options.argtypes = [P, C.c_float, C.c_float, C.c_int, C.c_int, C.c_int]
        L.ocl_add_sphere.argtypes = [P, fp, C.c_float, C.c_float, C.c_float]
        L.ocl_add_capsule.argtypes = [P, fp, fp, C.c_float, C.c_float, C.c_float]
        L.ocl_add_plane.argtypes = [P, fp, fp, C.c_float, C.c_float]
        L.ocl_set_mesh_triangles.argtypes = [P, fp, C.c_int, C.c_float, C.c_float, C.c_float, C.c_int, P]
        L.ocl_clear_colliders.argtypes = [P]
        L.ocl_set_pin.argtypes = [P, C.c_uint32, fp, C.c_float]
        L.ocl_clear_pins.argtypes = [P]
        L.ocl_step.argtypes = [P, C.c_float, C.c_int]
        L.ocl_num_vertices.argtypes = [P]
        L.ocl_num_vertices.restype = C.c_int
        L.ocl_get_positions.argtypes = [P, fp]
        L.ocl_get_state.argtypes = [P, P, P, P]
        L.ocl_set_state.argtypes = [P, fp, P]
        L.ocl_counts.argtypes = [P, np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")]
        L.ocl_get_distance.argtypes = [P, up, fp, fp, fp, up]
        L.ocl_get_bending.argtypes = [P, up, fp, fp, fp]
        L.ocl_get_dist_colors.argtypes = [P, up, up]
        L.ocl_get_bend_colors.argtypes = [P, up, up]
        L.ocl_get_edges.argtypes = [P, up, up]
        L.ocl_topology_sizes.argtypes = [P, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.ocl_topology_sizes.restype = C.c_int
        L.ocl_get_topology.argtypes = [P, up, up, up, up, fp, fp, up, up, up, up]
        L.ocl_cell_size.argtypes = [P]
        L.ocl_cell_size.restype = C.c_float
        L.ocl_build_hash.argtypes = [P, C.c_int, up, up]
        L.ocl_get_mesh_triangles.argtypes = [P, fp]
        L.ocl_half_roundtrip.argtypes = [P, C.c_int, P, P]
        L.ocl_set_self_collision_intervals.argtypes = [P, C.c_int, C.c_int]
        L.ocl_set_pair_cache.argtypes = [P, C.c_int, C.c_int]
        L.ocl_set_pair_cache_options.argtypes = [P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_float, C.c_float,
                                                 C.c_float]
        L.ocl_get_active_pairs.argtypes = [P, up, P, C.c_size_t, P, C.c_size_t]
        L.ocl_bone_skin_mats.argtypes = [C.c_int, P, P, P]
        L.ocl_bone_skin.argtypes = [C.c_int, P, P, P, P, P]
        L.ocl_bone_prep.argtypes = [C.c_int, P, P, P, P, P]
        L.ocl_bone_bake.argtypes = [C.c_int, P, P, P]
        L.ocl_set_bone_sdf.argtypes = [P, C.c_uint32, C.c_uint32, C.c_uint32, P, C.c_int, P, P]
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class OracleSim:
    """Sequential CPU restatement of GpuClothSimulator (test oracle)."""

    def __init__(self, positions, edges, faces=None, inv_masses=None, layer_ids=None,
                 thicknesses=None, layer_id=0, thickness=0.005, stiffness=1000.0,
                 bending_stiffness=10.0, compression_stiffness=None, shear_stiffness=None,
                 sewing_springs=None, sewing_shrink_speed=1.0):
        L = lib()
        self._keep = []
        pos = np.ascontiguousarray(positions, dtype=_f).reshape(-1, 3)
        e = np.ascontiguousarray(edges, dtype=_u).reshape(-1, 2)
        f = None if faces is None else np.ascontiguousarray(faces, dtype=_u).reshape(-1, 3)
        im = None if inv_masses is None else np.ascontiguousarray(inv_masses, dtype=_f)
        li = None if layer_ids is None else np.ascontiguousarray(layer_ids, dtype=_u)
        th = None if thicknesses is None else np.ascontiguousarray(thicknesses, dtype=_f)
        comp = stiffness if compression_stiffness is None else compression_stiffness
        shear = stiffness * 0.5 if shear_stiffness is None else shear_stiffness
        self.n = pos.shape[0]
        sew = None if sewing_springs is None else np.ascontiguousarray(sewing_springs, dtype=_u).reshape(-1, 2)
        self._h = L.ocl_create_sewn(_ptr(pos), pos.shape[0], _ptr(e), e.shape[0], _ptr(f),
                                    0 if f is None else f.shape[0], _ptr(im), _ptr(li), _ptr(th),
                                    layer_id, thickness, stiffness, comp, shear, bending_stiffness,
                                    _ptr(sew), 0 if sew is None else sew.shape[0], sewing_shrink_speed)

    def __del__(self):
        try:
            if self._h:
                lib().ocl_destroy(self._h)
                self._h = None
        except Exception:
            pass

    # --- setters -----------------------------------------------------
    def set_gravity(self, gx, gy, gz):
        lib().ocl_set_gravity(self._h, gx, gy, gz)

    def set_damping(self, d):
        lib().ocl_set_damping(self._h, d)

    def set_damping_all(self, t, c, s, b):
        lib().ocl_set_damping_all(self._h, t, c, s, b)

    def set_solver_iterations(self, n):
        lib().ocl_set_solver_iterations(self._h, int(n))

    def set_enable_self_collision(self, on):
        lib().ocl_set_enable_self_collision(self._h, int(bool(on)))

    def set_coupled_collider(self, on):
        lib().ocl_set_coupled_collider(self._h, int(bool(on)))

    def set_self_collision_options(self, relief_factor=0.2, max_displacement_ratio=0.2,
                                   exclude_neighbors=True, enable_normal_untangling=True,
                                   max_iterations=128):
        lib().ocl_set_self_collision_options(self._h, relief_factor, max_displacement_ratio,
                                             int(exclude_neighbors), int(enable_normal_untangling),
                                             int(max_iterations))

    def set_compliance_all(self, tension, compression, shear, bending):
        lib().ocl_set_compliance_all(self._h, tension, compression, shear, bending)

    def set_collider_options(self, enable_cluster_culling=False, enable_single_sided_recovery=True,
                             sweep_margin=0.05):
        lib().ocl_set_collider_options(self._h, int(enable_cluster_culling), int(enable_single_sided_recovery),
                                       sweep_margin)

    def add_sphere_collider(self, center, radius, friction=0.0, restitution=0.0):
        lib().ocl_add_sphere(self._h, np.asarray(center, _f), radius, friction, restitution)

    def add_capsule_collider(self, point_a, point_b, radius, friction=0.0, restitution=0.0):
        lib().ocl_add_capsule(self._h, np.asarray(point_a, _f), np.asarray(point_b, _f), radius,
                              friction, restitution)

    def add_plane_collider(self, point, normal, friction=0.0, restitution=0.0):
        lib().ocl_add_plane(self._h, np.asarray(point, _f), np.asarray(normal, _f), friction,
                            restitution)

    def set_mesh_collider_triangles(self, triangles, friction=0.3, thickness=0.01, restitution=0.0,
                                    single_sided=True, attributes=None):
        t = np.ascontiguousarray(triangles, dtype=_f).reshape(-1, 9)
        a = None if attributes is None else np.ascontiguousarray(attributes, dtype=_f)
        self._keep = [t, a]
        lib().ocl_set_mesh_triangles(self._h, t, t.shape[0], friction, thickness, restitution,
                                     int(single_sided), _ptr(a))

    def clear_colliders(self):
        lib().ocl_clear_colliders(self._h)

    def set_pin(self, vertex_idx, target_pos, weight=1.0):
        lib().ocl_set_pin(self._h, int(vertex_idx), np.asarray(target_pos, _f), weight)

    def clear_pins(self):
        lib().ocl_clear_pins(self._h)

    # --- stepping / state -----------------------------------------------
    def step(self, dt=1.0 / 60.0, substeps=None, solver_iterations=None):
        if solver_iterations is not None:
            self.set_solver_iterations(solver_iterations)
        lib().ocl_step(self._h, dt, 0 if substeps is None else int(substeps))
        return 20 if substeps is None else int(substeps)

    def get_positions(self, out=None):
        o = np.empty(self.n * 3, _f) if out is None else out
        lib().ocl_get_positions(self._h, o)
        return o

    def get_state(self):
        x = np.empty((self.n, 3), _f)
        p = np.empty((self.n, 3), _f)
        v = np.empty((self.n, 3), _f)
        lib().ocl_get_state(self._h, _ptr(x), _ptr(p), _ptr(v))
        return x, p, v

    def set_positions_and_velocities(self, positions, velocities=None):
        self.set_state(positions, velocities)

    def step_single_substep(self, dt_sub):
        lib().ocl_step(self._h, dt_sub, 1)

    def set_state(self, x, v=None):
        x = np.ascontiguousarray(x, _f).reshape(-1)
        vv = None if v is None else np.ascontiguousarray(v, _f).reshape(-1)
        lib().ocl_set_state(self._h, x, _ptr(vv))

    # --- introspection --------------------------------------------------
    def counts(self):
        o = np.zeros(8, np.int32)
        lib().ocl_counts(self._h, o)
        keys = ["nd", "nb", "n_dist_colors", "n_bend_colors", "n_edges", "table_size",
                "num_virtual", "multi_layer"]
        return dict(zip(keys, (int(v) for v in o)))

    def distance_constraints(self):
        c = self.counts()
        nd = c["nd"]
        v = np.zeros(2 * max(nd, 1), _u)
        r, tc, cc = (np.zeros(max(nd, 1), _f) for _ in range(3))
        ty = np.zeros(max(nd, 1), _u)
        lib().ocl_get_distance(self._h, v, r, tc, cc, ty)
        return dict(v=v[:2 * nd].reshape(-1, 2), rest=r[:nd], tc=tc[:nd], cc=cc[:nd], type=ty[:nd])

    def bending_constraints(self):
        nb = self.counts()["nb"]
        v = np.zeros(4 * max(nb, 1), _u)
        r, cp, p0, p1 = (np.zeros(max(nb, 1), _f) for _ in range(4))
        lib().ocl_get_bending(self._h, v, r, cp, p0)
        lib().ocl_get_bending_gate(self._h, p1)
        return dict(v=v[:4 * nb].reshape(-1, 4), rest=r[:nb], comp=cp[:nb], pad0=p0[:nb], pad1=p1[:nb])

    # --- contact-pair cache ---------------------------------------------
    def set_pair_cache(self, enable=True, final_fallback=True):
        lib().ocl_set_pair_cache(self._h, int(bool(enable)), int(bool(final_fallback)))

    def set_pair_cache_options(self, max_vt_pairs=65536, max_ee_pairs=65536, margin_mode=1, safety_margin=0.005,
                               horizon_scale=1.3, max_horizon=0.02):
        lib().ocl_set_pair_cache_options(self._h, int(max_vt_pairs), int(max_ee_pairs), int(margin_mode),
                                         safety_margin, horizon_scale, max_horizon)

    def active_pairs(self):
        """(vt_accepted, ee_accepted, vt_pairs (k x 4), ee_pairs (k x 4)) of the latest broad phase."""
        c = np.zeros(4, _u)
        lib().ocl_get_active_pairs(self._h, c, None, 0, None, 0)
        vt = np.zeros((max(int(c[2]), 1), 4), _u)
        ee = np.zeros((max(int(c[3]), 1), 4), _u)
        lib().ocl_get_active_pairs(self._h, c, vt.ctypes.data, int(c[2]), ee.ctypes.data, int(c[3]))
        return int(c[0]), int(c[1]), vt[:int(c[2])], ee[:int(c[3])]

    # --- edge colliders -------------------------------------------------
    def set_pair_recording(self, enable=True):
        lib().ocl_set_pair_recording(self._h, int(bool(enable)))

    def get_pair_lists(self):
        cnt = np.zeros(2, _u)
        lib().ocl_get_pair_lists(self._h, None, 0, None, 0, _ptr(cnt))
        vt = np.zeros((max(int(cnt[0]), 1), 4), _u)
        ee = np.zeros((max(int(cnt[1]), 1), 2), _u)
        lib().ocl_get_pair_lists(self._h, _ptr(vt), vt.shape[0], _ptr(ee), ee.shape[0], _ptr(cnt))
        return dict(vt=vt[:int(cnt[0])], ee=ee[:int(cnt[1])])

    def set_edge_collision(self, enable=True, margin_scale=1.0, margin_offset=0.0):
        lib().ocl_set_edge_collision(self._h, int(bool(enable)), margin_scale, margin_offset)

    def num_collider_edges(self):
        return lib().ocl_num_collider_edges(self._h)

    # --- sewing --------------------------------------------------------
    def set_sewing(self, stiffness=10000.0, lock=True, lock_distance=0.02, shrink_speed=1.0):
        lib().ocl_set_sewing(self._h, stiffness, int(bool(lock)), lock_distance, shrink_speed)

    def sewing(self):
        """Sewing constraints in colour order: vertex pairs, current rest
        lengths, colour offsets / counts and the sewing group of each vertex."""
        L = lib()
        nc = C.c_int()
        k = L.ocl_get_sewing(self._h, C.byref(nc), None, None, None, None, None)
        v = np.zeros(2 * max(k, 1), _u)
        cur = np.zeros(max(k, 1), _f)
        off, cnt = np.zeros(max(nc.value, 1), _u), np.zeros(max(nc.value, 1), _u)
        rep = np.zeros(max(self.n, 1), _u)
        L.ocl_get_sewing(self._h, None, _ptr(v), _ptr(cur), _ptr(off), _ptr(cnt), _ptr(rep))
        return dict(v=v[:2 * k].reshape(-1, 2), cur=cur[:k], off=off[:nc.value], cnt=cnt[:nc.value],
                    rep=rep[:self.n])

    def colors(self):
        c = self.counts()
        do, dc = np.zeros(max(c["n_dist_colors"], 1), _u), np.zeros(max(c["n_dist_colors"], 1), _u)
        bo, bc = np.zeros(max(c["n_bend_colors"], 1), _u), np.zeros(max(c["n_bend_colors"], 1), _u)
        lib().ocl_get_dist_colors(self._h, do, dc)
        lib().ocl_get_bend_colors(self._h, bo, bc)
        k, m = c["n_dist_colors"], c["n_bend_colors"]
        return dict(dist_off=do[:k], dist_cnt=dc[:k], bend_off=bo[:m], bend_cnt=bc[:m])

    def edges(self):
        ne = self.counts()["n_edges"]
        e = np.zeros(2 * max(ne, 1), _u)
        b = np.zeros(max((ne + 31) // 32, 1), _u)
        lib().ocl_get_edges(self._h, e, b)
        return e[:2 * ne].reshape(-1, 2), b[:(ne + 31) // 32]

    def topology(self):
        a, t, s = C.c_int(), C.c_int(), C.c_int()
        n = lib().ocl_topology_sizes(self._h, C.byref(a), C.byref(t), C.byref(s))
        out = dict(adj_off=np.zeros(n + 1, _u), adj_idx=np.zeros(max(a.value, 1), _u),
                   th_off=np.zeros(n + 1, _u), th_idx=np.zeros(max(t.value, 1), _u),
                   th_rest=np.zeros(max(t.value, 1), _f), local_len=np.zeros(max(n, 1), _f),
                   star_off=np.zeros(n + 1, _u), star_idx=np.zeros(2 * max(s.value, 1), _u),
                   island=np.zeros(max(n, 1), _u), layer=np.zeros(max(n, 1), _u))
        lib().ocl_get_topology(self._h, out["adj_off"], out["adj_idx"], out["th_off"], out["th_idx"],
                               out["th_rest"], out["local_len"], out["star_off"], out["star_idx"],
                               out["island"], out["layer"])
        out["adj_idx"] = out["adj_idx"][:a.value]
        out["th_idx"] = out["th_idx"][:t.value]
        out["th_rest"] = out["th_rest"][:t.value]
        out["star_idx"] = out["star_idx"][:2 * s.value].reshape(-1, 2)
        return out

    def cell_size(self):
        return float(lib().ocl_cell_size(self._h))

    def build_hash(self, which=0):
        c = self.counts()
        T = c["table_size"]
        cnt = self.n if which == 0 else c["n_edges"]
        cs = np.zeros(T + 1, _u)
        srt = np.zeros(max(cnt, 1), _u)
        lib().ocl_build_hash(self._h, which, cs, srt)
        return cs, srt[:cnt]


# --- bone SDF (skinning.wgsl, prep_bone_triangles.wgsl, bake_sdf.wgsl) -----
def half_roundtrip(x):
    """(binary16 bits, value back in float32) with round to nearest even."""
    x = np.ascontiguousarray(x, _f).ravel()
    bits = np.zeros(x.size, np.uint16)
    out = np.zeros(x.size, _f)
    lib().ocl_half_roundtrip(_ptr(x), x.size, _ptr(bits), _ptr(out))
    return bits, out


def bone_skin_mats(world, bind_inv):
    """S = M_world B_bind per bone (column-major out), as the host does before skinning.
    world: (N, 4, 4) as stored for the shaders; bind_inv: (N, 4, 4) row-major."""
    w = np.ascontiguousarray(world, _f).reshape(-1, 16)
    x = np.zeros((w.shape[0], 32), _f)
    x[:, :16] = w
    b = np.ascontiguousarray(bind_inv, _f).reshape(-1, 16)
    out = np.zeros((w.shape[0], 16), _f)
    lib().ocl_bone_skin_mats(w.shape[0], _ptr(x), _ptr(b), _ptr(out))
    return out


def bone_skin(rest, bidx, bw, skin_mats):
    nv = rest.shape[0]
    r4 = np.zeros((nv, 4), _f)
    r4[:, :3] = rest[:, :3]
    out = np.zeros((nv, 4), _f)
    lib().ocl_bone_skin(nv, _ptr(r4), _ptr(np.ascontiguousarray(bidx, _u)), _ptr(np.ascontiguousarray(bw, _f)),
                        _ptr(np.ascontiguousarray(skin_mats, _f)), _ptr(out))
    return out


def bone_prep(skinned4, inv_mats, src4, srcw4):
    nt = src4.shape[0]
    out = np.zeros((nt, 16), _f)
    lib().ocl_bone_prep(nt, _ptr(np.ascontiguousarray(skinned4, _f)), _ptr(np.ascontiguousarray(inv_mats, _f)),
                        _ptr(np.ascontiguousarray(src4, _u)), _ptr(np.ascontiguousarray(srcw4, _f)), _ptr(out))
    return out


def bone_bake(params16, tris16, dims):
    """params16: (P, 16) uint32 words of the bake parameters; returns the atlas texels."""
    W, H, D = dims
    atlas = np.zeros(W * H * D, _u)
    p = np.ascontiguousarray(params16, _u)
    lib().ocl_bone_bake(p.shape[0], _ptr(p), _ptr(np.ascontiguousarray(tris16, _f)), _ptr(atlas))
    return atlas


def bake_params_words(lmin, tri_start, lmax, tri_count, col, row, layer, res, W, H, D, pitch=0):
    w = np.zeros(16, _u)
    w[0:3] = np.asarray(lmin, _f).view(_u)
    w[3] = tri_start
    w[4:7] = np.asarray(lmax, _f).view(_u)
    w[7] = tri_count
    w[8:16] = [col, row, layer, res, W, H, D, pitch]
    return w


def _set_bone_sdf(self, dims, atlas, infos, xforms32):
    W, H, D = dims
    a = np.ascontiguousarray(atlas, _u)
    i = np.ascontiguousarray(infos, _f).reshape(-1, 20)
    x = np.ascontiguousarray(xforms32, _f).reshape(-1, 32)
    self._keep_bone = (a, i, x)
    lib().ocl_set_bone_sdf(self._h, W, H, D, _ptr(a), i.shape[0], _ptr(i), _ptr(x))


OracleSim.set_bone_sdf = _set_bone_sdf


def _set_sc_interval(self, interval):
    self._sc_iv = max(int(interval), 1)
    lib().ocl_set_self_collision_intervals(self._h, self._sc_iv, getattr(self, "_ee_iv", 1))


def _set_ee_interval(self, interval):
    self._ee_iv = int(interval)
    lib().ocl_set_self_collision_intervals(self._h, getattr(self, "_sc_iv", 1), self._ee_iv)


OracleSim.set_self_collision_substep_interval = _set_sc_interval
OracleSim.set_self_collision_ee_substep_interval = _set_ee_interval


def bake_mesh_sdf(verts, tris, voxel_size=0.004, margin=0.02, friction=0.5, thickness=0.005, restitution=0.0):
    """Single-mesh SDF of a closed mesh: (dims (3,), info (20,), texels (d, h, w) uint32)."""
    L = lib()
    v = np.ascontiguousarray(verts, dtype=_f).reshape(-1, 3)
    t = np.ascontiguousarray(tris, dtype=np.int32).reshape(-1, 3)
    dims = np.zeros(3, _u)
    info = np.zeros(20, _f)
    L.ocl_bake_mesh_sdf(_ptr(v), v.shape[0], _ptr(t), t.shape[0], voxel_size, margin, friction, thickness,
                        restitution, _ptr(dims), _ptr(info), None)
    tex = np.zeros(int(dims[0]) * int(dims[1]) * int(dims[2]), _u)
    L.ocl_bake_mesh_sdf(_ptr(v), v.shape[0], _ptr(t), t.shape[0], voxel_size, margin, friction, thickness,
                        restitution, _ptr(dims), _ptr(info), _ptr(tex))
    return dims, info, tex.reshape(int(dims[2]), int(dims[1]), int(dims[0]))


def bake_mesh_sdf_coarse(verts, tris, voxel_size=0.004, margin=0.02, thickness=0.005):
    """Coarse pass of the hierarchical bake of a closed mesh:
    (dims (3,), coarse_voxel, dist (d, h, w) uint32, nearest (d, h, w, 8) uint32)."""
    L = lib()
    v = np.ascontiguousarray(verts, dtype=_f).reshape(-1, 3)
    t = np.ascontiguousarray(tris, dtype=np.int32).reshape(-1, 3)
    dims = np.zeros(3, _u)
    cv = np.zeros(1, _f)
    L.ocl_bake_mesh_sdf_coarse(_ptr(v), v.shape[0], _ptr(t), t.shape[0], voxel_size, margin, thickness, _ptr(dims),
                               _ptr(cv), None, None)
    n = int(dims[0]) * int(dims[1]) * int(dims[2])
    dist = np.zeros(n, _u)
    near = np.zeros(n * 8, _u)
    L.ocl_bake_mesh_sdf_coarse(_ptr(v), v.shape[0], _ptr(t), t.shape[0], voxel_size, margin, thickness, _ptr(dims),
                               _ptr(cv), _ptr(dist), _ptr(near))
    shape = (int(dims[2]), int(dims[1]), int(dims[0]))
    return dims, float(cv[0]), dist.reshape(shape), near.reshape(shape + (8,))


def bake_mesh_sdf_hierarchical(verts, tris, voxel_size=0.004, margin=0.02, friction=0.5, thickness=0.005,
                               restitution=0.0):
    """Hierarchical bake of a closed mesh: (dims, info, texels (d, h, w)); raises
    RuntimeError when the band is wider than two coarse cells."""
    L = lib()
    v = np.ascontiguousarray(verts, dtype=_f).reshape(-1, 3)
    t = np.ascontiguousarray(tris, dtype=np.int32).reshape(-1, 3)
    dims = np.zeros(3, _u)
    info = np.zeros(20, _f)
    if L.ocl_bake_mesh_sdf_hier(_ptr(v), v.shape[0], _ptr(t), t.shape[0], voxel_size, margin, friction, thickness,
                                restitution, _ptr(dims), _ptr(info), None):
        raise RuntimeError("band wider than two coarse cells")
    tex = np.zeros(int(dims[0]) * int(dims[1]) * int(dims[2]), _u)
    L.ocl_bake_mesh_sdf_hier(_ptr(v), v.shape[0], _ptr(t), t.shape[0], voxel_size, margin, friction, thickness,
                             restitution, _ptr(dims), _ptr(info), _ptr(tex))
    return dims, info, tex.reshape(int(dims[2]), int(dims[1]), int(dims[0]))
