"""``ClothSimulator``: the reference's PyO3 class, re-homed on the C ABI.

Mirrors ``taremin_cloth_core.ClothSimulator`` (crates/cloth_py/src/lib.rs:1549-3100)
for the XPBD substep: same constructor arguments and defaults, same setter
names, same exceptions (``ValueError`` for bad shapes or indices,
``RuntimeError`` when the GPU cannot be initialised).  All work runs in
``libtcloth.so`` on the GPU.
"""
from __future__ import annotations

import ctypes as C
import json

import numpy as np

from . import _lib

_f32 = np.float32
_u32 = np.uint32


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _arr(a, dtype, cols=None, name="array"):
    if a is None:
        return None
    x = np.ascontiguousarray(np.asarray(a), dtype=dtype)
    if cols is not None:
        if x.ndim != 2 or x.shape[1] != cols:
            raise ValueError(f"{name} must have shape (N, {cols}), got {tuple(x.shape)}")
    return x


def bake_bone_sdf_gpu(mesh_verts, mesh_tris, bone_names, bone_weights, bone_bind_matrices, resolution=64,
                      margin=0.2, weight_threshold=0.02, blend_k=0.05, friction=0.5, thickness=0.005,
                      restitution=0.0, close_open_boundaries=True, device=0):
    """Bone-local SDF atlas of a skinned mesh on the GPU (lib.rs:1186-1350).
    Returns dict(texture_bytes, width, height, depth, bone_infos (N, 20),
    active_bones, bind_matrices (N, 4, 4))."""
    if resolution == 0:
        raise ValueError("resolution must be >= 1")
    v = np.ascontiguousarray(np.asarray(mesh_verts, _f32))
    if v.ndim != 2 or v.shape[1] < 3:
        raise ValueError("mesh_verts must have shape (N, 3)")
    v = np.ascontiguousarray(v[:, :3])
    t = np.ascontiguousarray(np.asarray(mesh_tris, np.int32))
    if t.ndim != 2 or t.shape[1] < 3:
        raise ValueError("mesh_tris must have shape (M, 3)")
    t = np.ascontiguousarray(t[:, :3])
    names = list(bone_names)
    if len(bone_weights) != len(names):
        raise ValueError("bone_names and bone_weights differ in length")
    w = np.zeros((len(names), v.shape[0]), _f32)
    for b, wb in enumerate(bone_weights):
        wb = np.asarray(wb, _f32).ravel()
        if wb.size != v.shape[0]:
            raise ValueError(f"bone_weights[{b}] has {wb.size} entries for {v.shape[0]} vertices")
        w[b] = wb
    m = np.ascontiguousarray(np.asarray(bone_bind_matrices, _f32))
    if m.ndim != 3 or m.shape[0] < len(names) or m.shape[1:] != (4, 4):
        raise ValueError("bone_bind_matrices must have shape (N_bones, 4, 4)")
    L = _lib.load()
    h = C.c_void_p()
    _lib.check(L.tc_bake_bone_sdf(_ptr(v), v.shape[0], _ptr(t), t.shape[0], len(names), _ptr(w), _ptr(m),
                                  int(resolution), float(margin), float(weight_threshold), float(blend_k),
                                  float(friction), float(thickness), float(restitution),
                                  int(bool(close_open_boundaries)), int(device), C.byref(h)))
    try:
        dims = np.zeros(4, _u32)
        _lib.check(L.tc_bake_dims(h, _ptr(dims)))
        W, H, D, na = (int(x) for x in dims)
        tex = np.zeros(W * H * D, _u32)
        infos = np.zeros((na, 20), _f32)
        active = np.zeros(na, _u32)
        bind = np.zeros((na, 4, 4), _f32)
        _lib.check(L.tc_bake_get(h, _ptr(tex), _ptr(infos), _ptr(active), _ptr(bind)))
    finally:
        L.tc_bake_destroy(h)
    return {"texture_bytes": tex.tobytes(), "width": W, "height": H, "depth": D, "bone_infos": infos,
            "active_bones": [names[int(i)] for i in active], "bind_matrices": bind}


def bake_mesh_sdf_gpu(mesh_verts, mesh_tris, voxel_size=0.004, margin=0.02, friction=0.5, thickness=0.005,
                      restitution=0.0, close_open_boundaries=True, device=0):
    """Signed distance field of one mesh on the GPU (lib.rs:1349-1416).
    Returns dict(texture_bytes, width, height, depth, bone_info (20,))."""
    v = np.ascontiguousarray(np.asarray(mesh_verts, _f32))
    if v.ndim != 2 or v.shape[1] < 3:
        raise ValueError("mesh_verts must have shape (N, 3)")
    v = np.ascontiguousarray(v[:, :3])
    t = np.ascontiguousarray(np.asarray(mesh_tris, np.int32))
    if t.ndim != 2 or t.shape[1] < 3:
        raise ValueError("mesh_tris must have shape (M, 3)")
    t = np.ascontiguousarray(t[:, :3])
    L = _lib.load()
    h = C.c_void_p()
    _lib.check(L.tc_bake_mesh_sdf(_ptr(v), v.shape[0], _ptr(t), t.shape[0], float(voxel_size), float(margin),
                                  float(friction), float(thickness), float(restitution),
                                  int(bool(close_open_boundaries)), int(device), C.byref(h)))
    try:
        dims = np.zeros(4, _u32)
        _lib.check(L.tc_bake_dims(h, _ptr(dims)))
        W, H, D = (int(x) for x in dims[:3])
        tex = np.zeros(W * H * D, _u32)
        info = np.zeros(20, _f32)
        _lib.check(L.tc_bake_get(h, _ptr(tex), _ptr(info), None, None))
    finally:
        L.tc_bake_destroy(h)
    return {"texture_bytes": tex.tobytes(), "width": W, "height": H, "depth": D, "bone_info": info}


def _rows(a, width, dtype, name):
    if a is None:
        return None
    x = np.asarray(a)
    if x.size == 0:
        return None
    if x.ndim != 2 or x.shape[1] < width:
        raise ValueError(f"{name} must have shape (M, {width})")
    return np.ascontiguousarray(x[:, :width], dtype=dtype)


def compute_combined_inv_masses(positions, faces=None, strand_edges=None, pin_weights=None, areal_density=0.15,
                                linear_density=0.0):
    """Inverse masses from areal and linear density (lib.rs:553-611, mesh.rs:237-312); host only."""
    pos = np.asarray(positions, _f32)
    if pos.ndim != 2 or pos.shape[1] != 3:
        raise ValueError("each vertex of positions must have 3 coordinates")
    pos = np.ascontiguousarray(pos)
    f = _rows(faces, 3, _u32, "faces")
    st = _rows(strand_edges, 2, _u32, "strand_edges")
    pw = None if pin_weights is None else np.ascontiguousarray(np.asarray(pin_weights, _f32).reshape(-1))
    out = np.zeros(pos.shape[0], _f32)
    L = _lib.load()
    _lib.check(L.tc_compute_combined_inv_masses(_ptr(pos), pos.shape[0], _ptr(f), 0 if f is None else f.shape[0],
                                                _ptr(st), 0 if st is None else st.shape[0], _ptr(pw),
                                                0 if pw is None else pw.size, float(areal_density),
                                                float(linear_density), _ptr(out)))
    return out


def compute_areal_inv_masses(positions, faces=None, pin_weights=None, areal_density=0.15, strand_edges=None,
                             linear_density=0.0):
    """The same with the reference's older argument order (lib.rs:613-640)."""
    return compute_combined_inv_masses(positions, faces, strand_edges, pin_weights, areal_density, linear_density)


def color_edge_pairs(num_vertices, edges):
    """Welsh-Powell colour per vertex pair (lib.rs:642-652, coloring.rs:180-233); host only."""
    e = _rows(edges, 2, _u32, "edges")
    if e is None:
        return []
    out = np.zeros(e.shape[0], _u32)
    L = _lib.load()
    _lib.check(L.tc_color_edge_pairs(int(num_vertices), _ptr(e), e.shape[0], _ptr(out)))
    return [int(c) for c in out]


def mark_device_lost(device=0):
    """Mark a device's context lost (context.rs:131-134); the next simulator
    created on it re-initialises the context, older simulators refuse calls."""
    _lib.check(_lib.load().tc_mark_device_lost(int(device)))


def device_status(device=0):
    """(lost, epoch) of a device's context (context.rs:126-129)."""
    lost, epoch = C.c_int(0), C.c_uint64(0)
    _lib.check(_lib.load().tc_device_status(int(device), C.byref(lost), C.byref(epoch)))
    return bool(lost.value), int(epoch.value)


# SimConfig::default (crates/cloth_core/src/config.rs:3-37, :142-196): the
# value of every field a settings JSON record leaves out
CONFIG_DEFAULTS = {
    "version": 1, "gravity": [0.0, 0.0, -9.81], "damping": 1.0, "tension_damping": 5.0,
    "compression_damping": 5.0, "shear_damping": 5.0, "bending_damping": 0.5, "tension_stiffness": 1500.0,
    "compression_stiffness": 150.0, "shear_stiffness": 100.0, "bending_stiffness": 15.0, "solver_iterations": 2,
    "solver_mode": 0, "workgroup_size": 32, "enable_self_collision": False, "relief_factor": 1.0,
    "max_displacement_ratio": 0.5, "exclude_neighbors": True, "enable_normal_untangling": True,
    "self_collision_max_iterations": 256, "coupled_mode": 0, "coupled_collider": False, "post_relaxation_iters": 2,
    "substep_interval": 1, "ee_substep_interval": 1, "self_collision_algorithm": 0, "enable_pair_cache": False,
    "pair_margin_mode": 1, "pair_safety_margin": 0.005, "pair_horizon_scale": 1.3, "pair_max_horizon": 0.02,
    "pair_max_pairs": 65536, "enable_pair_final_fallback": True, "enable_edge_collision": False,
    "edge_margin_scale": 1.0, "edge_margin_offset": 0.0, "sewing_stiffness": 10000.0, "sewing_shrink_speed": 1.0,
    "enable_sewing_lock": True, "sewing_lock_distance": 0.02, "sewing_priority_enabled": False,
    "sewing_priority_threshold": 0.9, "sewing_priority_merge_dist": 0.005, "sewing_priority_ramp_frames": 3,
    "sewing_priority_max_frames": 600, "areal_density": 0.15, "enable_adaptive_substep": False, "min_substeps": 4,
    "max_substeps": 64, "auto_coupled_on_low_substeps": True, "auto_compensate_iterations": True,
    "enable_strain_adaptive": True, "strain_tolerance": 0.008,
}


def find_triangle_intersections(positions, faces, ignore_adjacent=True, cell_size=None, sewing_springs=None):
    """Self-intersecting face pairs [(f0, f1), ...], f0 < f1 ascending
    (lib.rs:856-879, geometry.rs:506-633); host only, no GPU needed."""
    pos = _arr(positions, _f32, 3, "positions")
    f = _rows(faces, 3, _u32, "faces")
    if f is None:
        return []
    sew = _rows(sewing_springs, 2, _u32, "sewing_springs") if sewing_springs is not None else None
    L = _lib.load()
    cnt = C.c_uint32(0)
    cap = max(64, f.shape[0])
    while True:
        out = np.zeros(2 * cap, _u32)
        _lib.check(L.tc_find_triangle_intersections(_ptr(pos), pos.shape[0], _ptr(f), f.shape[0],
                                                    int(bool(ignore_adjacent)),
                                                    float(cell_size) if cell_size else 0.0, _ptr(sew),
                                                    0 if sew is None else sew.shape[0], _ptr(out), cap,
                                                    C.byref(cnt)))
        if cnt.value <= cap:
            return [(int(a), int(b)) for a, b in out[:2 * cnt.value].reshape(-1, 2)]
        cap = cnt.value


def _mesh_arrays(mesh_verts, mesh_tris):
    v = np.ascontiguousarray(np.asarray(mesh_verts, _f32))
    if v.ndim != 2 or v.shape[1] < 3:
        raise ValueError("mesh_verts must have shape (N, 3)")
    t = np.ascontiguousarray(np.asarray(mesh_tris, np.int32))
    if t.ndim != 2 or t.shape[1] < 3:
        raise ValueError("mesh_tris must have shape (M, 3)")
    return np.ascontiguousarray(v[:, :3]), np.ascontiguousarray(t[:, :3])


def bake_mesh_sdf_hierarchical_gpu(mesh_verts, mesh_tris, voxel_size=0.004, margin=0.02, friction=0.5,
                                   thickness=0.005, restitution=0.0, close_open_boundaries=True, device=0):
    """Two-pass (coarse grid, then fine grid) mesh SDF (lib.rs:1418-1488).
    Returns dict(texture_bytes, width, height, depth, bone_info (20,))."""
    v, t = _mesh_arrays(mesh_verts, mesh_tris)
    L = _lib.load()
    h = C.c_void_p()
    _lib.check(L.tc_bake_mesh_sdf_hierarchical(_ptr(v), v.shape[0], _ptr(t), t.shape[0], float(voxel_size),
                                               float(margin), float(friction), float(thickness), float(restitution),
                                               int(bool(close_open_boundaries)), int(device), C.byref(h)))
    try:
        dims = np.zeros(4, _u32)
        _lib.check(L.tc_bake_dims(h, _ptr(dims)))
        W, H, D = (int(x) for x in dims[:3])
        tex = np.zeros(W * H * D, _u32)
        info = np.zeros(20, _f32)
        _lib.check(L.tc_bake_get(h, _ptr(tex), _ptr(info), None, None))
    finally:
        L.tc_bake_destroy(h)
    return {"texture_bytes": tex.tobytes(), "width": W, "height": H, "depth": D, "bone_info": info}


def bake_mesh_sdf_coarse_gpu(mesh_verts, mesh_tris, voxel_size=0.004, margin=0.02, friction=0.5, thickness=0.005,
                             restitution=0.0, device=0):
    """Coarse pass of the hierarchical bake (lib.rs:1490-1540).  Returns
    dict(dist_packed (uint32 per coarse voxel), nearest_tri (8 per voxel),
    width, height, depth, coarse_voxel)."""
    v, t = _mesh_arrays(mesh_verts, mesh_tris)
    L = _lib.load()
    h = C.c_void_p()
    _lib.check(L.tc_bake_mesh_sdf_coarse(_ptr(v), v.shape[0], _ptr(t), t.shape[0], float(voxel_size), float(margin),
                                         float(friction), float(thickness), float(restitution), int(device),
                                         C.byref(h)))
    try:
        dims = np.zeros(4, _u32)
        _lib.check(L.tc_bake_dims(h, _ptr(dims)))
        W, H, D = (int(x) for x in dims[:3])
        dist = np.zeros(W * H * D, _u32)
        near = np.zeros(W * H * D * 8, _u32)
        cv = C.c_float()
        _lib.check(L.tc_bake_get(h, _ptr(dist), None, None, None))
        _lib.check(L.tc_bake_get_nearest(h, _ptr(near), C.byref(cv)))
    finally:
        L.tc_bake_destroy(h)
    return {"dist_packed": dist, "nearest_tri": near, "width": W, "height": H, "depth": D, "coarse_voxel": cv.value}


def is_gpu_available() -> bool:
    try:
        return bool(_lib.load().tc_gpu_available())
    except RuntimeError:
        return False


def get_gpu_device_name(device: int = 0) -> str:
    buf = C.create_string_buffer(256)
    _lib.check(_lib.load().tc_device_name(device, buf, 256))
    return buf.value.decode()


class ClothSimulator:
    """GPU XPBD cloth simulator (drop-in for the reference's ClothSimulator)."""

    def __init__(self, positions, edges, faces=None, inv_masses=None, sewing_springs=None, layer_ids=None,
                 thicknesses=None, layer_id=0, thickness=0.005, stiffness=1000.0, bending_stiffness=10.0,
                 sewing_shrink_speed=1.0, sewing_stiffness=None, enable_sewing_lock=None,
                 sewing_lock_distance=None, compression_stiffness=None, shear_stiffness=None, workgroup_size=32,
                 solver_mode=0, enable_compact_readback=None, enable_pair_cache=None, areal_density=None,
                 enable_coarse_constraints=None, self_collision_algorithm=None, device=0):
        L = _lib.load()
        self._h = None
        pos = _arr(positions, _f32, 3, "positions")
        e = _arr(edges, _u32, 2, "edges")
        sew = None
        if sewing_springs is not None:
            sa = np.asarray(sewing_springs)
            if sa.ndim != 2 or sa.shape[1] != 2:
                raise ValueError("each sewing_springs row must be a vertex pair (v0, v1)")
            sew = np.ascontiguousarray(sa, dtype=_u32)
            if sew.size and int(sew.max()) >= pos.shape[0]:
                bad = sew[(sew >= pos.shape[0]).any(axis=1)][0]
                raise ValueError(f"sewing_springs contains an index >= the vertex count ({pos.shape[0]}): "
                                 f"[{bad[0]}, {bad[1]}]")
        if solver_mode not in (0,):
            raise NotImplementedError("only the graph-coloured solver (solver_mode=0) is built")
        f = _arr(faces, _u32, 3, "faces") if faces is not None else None
        n = pos.shape[0]

        def per_vertex(a, dtype, name):
            if a is None:
                return None
            x = np.ascontiguousarray(np.asarray(a).reshape(-1), dtype=dtype)
            if x.shape[0] != n:
                raise ValueError(f"{name} length ({x.shape[0]}) does not match the vertex count ({n})")
            return x

        im = per_vertex(inv_masses, _f32, "inv_masses")
        li = per_vertex(layer_ids, _u32, "layer_ids")
        th = per_vertex(thicknesses, _f32, "thicknesses")
        comp = stiffness if compression_stiffness is None else compression_stiffness
        shear = stiffness * 0.5 if shear_stiffness is None else shear_stiffness
        h = C.c_void_p()
        nf = 0 if f is None else f.shape[0]
        nsew = 0 if sew is None else sew.shape[0]
        _lib.check(L.tc_create_sewn(C.byref(h), _ptr(pos), n, _ptr(e), e.shape[0], _ptr(f), nf, _ptr(im), _ptr(li),
                                    _ptr(th), int(layer_id), float(thickness), float(stiffness), float(comp),
                                    float(shear), float(bending_stiffness), _ptr(sew), nsew,
                                    float(sewing_shrink_speed),
                                    float("nan") if sewing_stiffness is None else float(sewing_stiffness),
                                    1 if enable_sewing_lock is None else int(bool(enable_sewing_lock)),
                                    float("nan") if sewing_lock_distance is None else float(sewing_lock_distance),
                                    int(device)))
        self._h = h
        self._L = L
        self._n = n
        self._solver_iterations = 2
        if enable_pair_cache is not None:
            self.set_enable_pair_cache(enable_pair_cache)
        if self_collision_algorithm is not None:
            self.set_self_collision_algorithm(self_collision_algorithm)

    def __del__(self):
        if getattr(self, "_h", None):
            try:
                self._L.tc_destroy(self._h)
            except Exception:
                pass
            self._h = None

    def _c(self, status):
        _lib.check(status)

    # ---------------- stepping
    def step(self, dt=0.016666667, substeps=None, solver_iterations=None):
        if solver_iterations is not None:
            self.set_solver_iterations(solver_iterations)
        eff = C.c_uint32()
        self._c(self._L.tc_step(self._h, float(dt), 0 if substeps is None else int(substeps), C.byref(eff)))
        return eff.value

    def step_async(self, dt=0.016666667, substeps=None, solver_iterations=None):
        if solver_iterations is not None:
            self.set_solver_iterations(solver_iterations)
        self._c(self._L.tc_step_async(self._h, float(dt), 0 if substeps is None else int(substeps)))

    def fetch_positions(self, out_array):
        out = self._out(out_array)
        ok = C.c_int()
        self._c(self._L.tc_fetch_positions(self._h, _ptr(out), out.size, C.byref(ok)))
        return bool(ok.value)

    def step_buffered(self, dt=0.016666667, substeps=None, solver_iterations=None):
        """One frame into the device ring (8 slots); returns the frames held."""
        if solver_iterations is not None:
            self.set_solver_iterations(solver_iterations)
        c = C.c_uint32()
        self._c(self._L.tc_step_buffered(self._h, float(dt), 0 if substeps is None else int(substeps), C.byref(c)))
        return c.value

    def fetch_buffered_positions(self, out_array):
        """Every held frame (frames x N x 3 floats, as much as fits) into
        out_array in one copy; returns the frame count and empties the ring."""
        if not isinstance(out_array, np.ndarray) or out_array.dtype != _f32 or not out_array.flags.c_contiguous \
                or not out_array.flags.writeable:
            raise ValueError("out_array must be a writable, contiguous float32 NumPy array")
        c = C.c_uint32()
        self._c(self._L.tc_fetch_buffered_positions(self._h, _ptr(out_array), out_array.size, C.byref(c)))
        return c.value

    def get_buffered_frame_count(self):
        c = C.c_uint32()
        self._c(self._L.tc_get_buffered_frame_count(self._h, C.byref(c)))
        return c.value

    def clear_frame_buffer(self):
        self._c(self._L.tc_clear_frame_buffer(self._h))

    def _out(self, out_array):
        if not isinstance(out_array, np.ndarray) or out_array.dtype != _f32 or not out_array.flags.c_contiguous \
                or not out_array.flags.writeable:
            raise ValueError("out_array must be a writable, contiguous float32 NumPy array")
        if out_array.size < self._n * 3:
            raise ValueError(f"out_array needs at least {self._n * 3} elements")
        return out_array

    def get_positions(self, out_array):
        out = self._out(out_array)
        self._c(self._L.tc_get_positions(self._h, _ptr(out), out.size))

    # ---------------- settings the CUDA path has no use for, kept for the API
    # (lib.rs:1898-1906, :1935-1937, :2828-2836, :2030-2060)
    def set_workgroup_size(self, wg_size):
        self._wg = 64 if int(wg_size) == 64 else 32
        self._c(self._L.tc_set_workgroup_size(self._h, int(wg_size)))

    def get_workgroup_size(self):
        return getattr(self, "_wg", 32)

    def get_solver_mode(self):
        return 0

    def set_solver_mode(self, mode):
        if int(mode) != 0:
            raise NotImplementedError("only the graph-coloured solver (solver_mode=0) is built")

    def set_coupled_self_collision_options(self, mode, relaxation_iters=0):
        """mode 0 (self-collision once per substep after the final pins) is the one built."""
        if int(mode) != 0:
            raise NotImplementedError("coupled self-collision modes 1-3 are not built")
        self._c(self._L.tc_set_coupled_self_collision_options(self._h, 0, int(relaxation_iters)))

    def set_nonfinite_check(self, enable=True):
        """Make position read-backs raise FloatingPointError on NaN / Inf."""
        self._c(self._L.tc_set_nonfinite_check(self._h, int(bool(enable))))

    def set_launch_block(self, threads=256):
        """Threads per block of the per-colour constraint launches (same results)."""
        self._c(self._L.tc_set_launch_block(self._h, int(threads)))

    def set_hash_cell_size(self, cell=None):
        """Spatial-hash cell; None restores the reference formula's value."""
        self._c(self._L.tc_set_hash_cell_size(self._h, 0.0 if cell is None else float(cell)))

    def set_self_collision_variant(self, ee_variant=0):
        """Edge-edge kernel shape (same results): 0 warp per edge with the counted
        pairs worked one lane each (default), 1 grouped by cell, 2 warp per edge
        with the contact work in the edge's warp."""
        self._c(self._L.tc_set_self_collision_variant(self._h, int(ee_variant)))

    def set_ee_pair_list_capacity(self, entries=0):
        """Capacity of the E-E pair list of variant 0 (0 = 24 per edge + 1024);
        pairs past it are worked by the search kernel, with the same results."""
        self._c(self._L.tc_set_ee_pair_list_capacity(self._h, int(entries)))

    # ---------------- narrow-phase pair lists (parity instrumentation)
    def set_pair_recording(self, enable=True, max_vt_pairs=1 << 20, max_ee_pairs=1 << 20):
        """Record, at every self-collision pass, the direct pass's V-T pairs that
        reach the contact math and its E-E pairs counted within max_search."""
        self._c(self._L.tc_set_pair_recording(self._h, int(bool(enable)), int(max_vt_pairs), int(max_ee_pairs)))

    def get_pair_lists(self):
        """dict(vt=(k, 4) uint32 rows (vertex, a < b < c), ee=(m, 2) rows (e0 < e1)),
        sorted, of the latest self-collision pass."""
        cnt = np.zeros(2, _u32)
        self._c(self._L.tc_get_pair_lists(self._h, None, 0, None, 0, _ptr(cnt)))
        vt = np.zeros((max(int(cnt[0]), 1), 4), _u32)
        ee = np.zeros((max(int(cnt[1]), 1), 2), _u32)
        self._c(self._L.tc_get_pair_lists(self._h, _ptr(vt), vt.shape[0], _ptr(ee), ee.shape[0], _ptr(cnt)))
        return dict(vt=vt[:int(cnt[0])], ee=ee[:int(cnt[1])])

    # ---------------- settings record (lib.rs:3029-3047, config_impl.rs:16-160)
    def get_config_json(self):
        """Every settable parameter as the reference's SimConfig JSON text."""
        n = C.c_size_t(0)
        self._c(self._L.tc_get_config_json(self._h, None, 0, C.byref(n)))
        buf = C.create_string_buffer(n.value + 1)
        self._c(self._L.tc_get_config_json(self._h, buf, n.value + 1, C.byref(n)))
        return buf.value.decode("ascii")

    def get_config_hash(self):
        """64-bit FNV-1a of get_config_json() (change detection between frames)."""
        h = C.c_uint64(0)
        self._c(self._L.tc_get_config_hash(self._h, C.byref(h)))
        return h.value

    def apply_config_json(self, json_str):
        """Apply a SimConfig JSON record through the setters, in the reference's
        order (config_impl.rs:80-155); absent fields take SimConfig's defaults
        (config.rs:142-196), unknown fields are ignored; malformed text or
        mistyped fields raise ValueError before anything is applied."""
        try:
            d = json.loads(json_str)
        except (TypeError, ValueError) as e:
            raise ValueError(f"could not parse the settings JSON: {e}") from None
        if not isinstance(d, dict):
            raise ValueError("the settings JSON must be an object")
        c = dict(CONFIG_DEFAULTS)
        for k, v in d.items():
            if k not in c:
                continue
            want = type(CONFIG_DEFAULTS[k])
            if want is bool:
                ok = isinstance(v, bool)
            elif want is int:
                ok = isinstance(v, int) and not isinstance(v, bool) and 0 <= v <= 0xFFFFFFFF
            elif want is float:
                ok = isinstance(v, (int, float)) and not isinstance(v, bool)
            else:
                ok = isinstance(v, list) and len(v) == 3 and all(
                    isinstance(x, (int, float)) and not isinstance(x, bool) for x in v)
            if not ok:
                raise ValueError(f"settings field {k!r} has an invalid value {v!r}")
            c[k] = v
        self.set_gravity(*c["gravity"])
        self.set_damping(c["damping"])
        self.set_damping_all(c["tension_damping"], c["compression_damping"], c["shear_damping"],
                             c["bending_damping"])
        self.set_stiffness_all(c["tension_stiffness"], c["compression_stiffness"], c["shear_stiffness"],
                               c["bending_stiffness"])
        self.set_solver_iterations(c["solver_iterations"])
        self.set_solver_mode(c["solver_mode"])
        self.set_workgroup_size(c["workgroup_size"])
        self.set_enable_self_collision(c["enable_self_collision"])
        self.set_self_collision_options(c["relief_factor"], c["max_displacement_ratio"], c["exclude_neighbors"],
                                        c["enable_normal_untangling"], c["self_collision_max_iterations"])
        self.set_coupled_self_collision_options(c["coupled_mode"], c["post_relaxation_iters"])
        self.set_coupled_collider(c["coupled_collider"])
        self.set_auto_coupled_on_low_substeps(c["auto_coupled_on_low_substeps"])
        self.set_self_collision_substep_interval(max(c["substep_interval"], 1))
        self.set_self_collision_ee_substep_interval(c["ee_substep_interval"])
        self.set_self_collision_algorithm(c["self_collision_algorithm"])
        self.set_enable_pair_cache(c["enable_pair_cache"])
        self.set_pair_cache_options(c["pair_max_pairs"], c["pair_max_pairs"], c["pair_margin_mode"],
                                    c["pair_safety_margin"], c["pair_horizon_scale"], c["pair_max_horizon"])
        self.set_enable_pair_cache_final_fallback(c["enable_pair_final_fallback"])
        self.set_enable_edge_collision(c["enable_edge_collision"])
        self.set_edge_margin_scale(c["edge_margin_scale"])
        self.set_edge_margin_offset(c["edge_margin_offset"])
        self.set_sewing_stiffness(c["sewing_stiffness"])
        self.set_sewing_shrink_speed(c["sewing_shrink_speed"])
        self.set_enable_sewing_lock(c["enable_sewing_lock"])
        self.set_sewing_lock_distance(c["sewing_lock_distance"])
        self.set_areal_density(c["areal_density"])
        self.set_sewing_priority_options(c["sewing_priority_enabled"], c["sewing_priority_threshold"],
                                         c["sewing_priority_merge_dist"], c["sewing_priority_ramp_frames"],
                                         c["sewing_priority_max_frames"])
        self.set_adaptive_substep_options(c["enable_adaptive_substep"], c["min_substeps"], c["max_substeps"])
        self.set_auto_compensate_iterations(c["auto_compensate_iterations"])
        self.set_strain_adaptive_options(c["enable_strain_adaptive"], c["strain_tolerance"])

    def set_areal_density(self, density):
        d = float(density)
        if np.isfinite(d):
            self._areal_density = min(max(d, 0.0), 100.0)
        self._c(self._L.tc_set_areal_density(self._h, d))

    def set_enable_compact_readback(self, enable):
        self._compact = bool(enable)

    def get_enable_compact_readback(self):
        return getattr(self, "_compact", False)

    def get_effective_normal_untangling(self):
        return getattr(self, "_untangle", True) and bool(self._counts()[7])

    def get_num_virtual_vertices(self):
        v = C.c_uint32()
        self._c(self._L.tc_get_num_virtual_vertices(self._h, C.byref(v)))
        return v.value

    def step_single_substep(self, dt_sub):
        self._c(self._L.tc_step_single_substep(self._h, float(dt_sub)))

    # ---------------- contact-pair cache (lib.rs:2029-2105)
    def set_enable_pair_cache(self, enable):
        self._c(self._L.tc_set_enable_pair_cache(self._h, int(bool(enable))))

    def set_pair_cache_enabled(self, enabled):
        self.set_enable_pair_cache(enabled)

    def get_enable_pair_cache(self):
        v = C.c_int()
        self._c(self._L.tc_get_enable_pair_cache(self._h, C.byref(v)))
        return bool(v.value)

    def set_self_collision_algorithm(self, algo):
        """0: direct, 1: contact-pair cache; 2 (virtual particles) is not built."""
        if int(algo) == 2:
            raise NotImplementedError("self-collision algorithm 2 (virtual-particle vertex-vertex) is not built")
        self._c(self._L.tc_set_self_collision_algorithm(self._h, int(algo)))

    def get_self_collision_algorithm(self):
        v = C.c_uint32()
        self._c(self._L.tc_get_self_collision_algorithm(self._h, C.byref(v)))
        return v.value

    def set_pair_cache_options(self, max_vt_pairs=65536, max_ee_pairs=65536, margin_mode=1, safety_margin=0.005,
                               horizon_scale=1.3, max_horizon=0.02):
        self._c(self._L.tc_set_pair_cache_options(self._h, int(max_vt_pairs), int(max_ee_pairs), int(margin_mode),
                                                  float(safety_margin), float(horizon_scale), float(max_horizon)))

    def set_enable_pair_cache_final_fallback(self, enable):
        self._c(self._L.tc_set_enable_pair_cache_final_fallback(self._h, int(bool(enable))))

    def get_enable_pair_cache_final_fallback(self):
        v = C.c_int()
        self._c(self._L.tc_get_enable_pair_cache_final_fallback(self._h, C.byref(v)))
        return bool(v.value)

    def get_pair_cache_stats(self):
        """(vt_count, ee_count, max_vt_pairs, max_ee_pairs) of the latest broad phase."""
        out = np.zeros(4, _u32)
        self._c(self._L.tc_get_pair_cache_stats(self._h, _ptr(out)))
        return tuple(int(x) for x in out)

    def get_active_pairs(self):
        """(vt_count, ee_count, V-T pairs, E-E pairs): the stored pairs as lists of four vertex ids."""
        c = np.zeros(4, _u32)
        self._c(self._L.tc_get_active_pairs(self._h, _ptr(c), None, 0, None, 0))
        vt = np.zeros((max(int(c[2]), 1), 4), _u32)
        ee = np.zeros((max(int(c[3]), 1), 4), _u32)
        self._c(self._L.tc_get_active_pairs(self._h, _ptr(c), _ptr(vt), int(c[2]), _ptr(ee), int(c[3])))
        return (int(c[0]), int(c[1]), vt[:int(c[2])].tolist(), ee[:int(c[3])].tolist())

    # ---------------- edge colliders (lib.rs:2736-2749)
    def set_enable_edge_collision(self, enable):
        self._c(self._L.tc_set_enable_edge_collision(self._h, int(bool(enable))))

    def set_edge_margin_scale(self, scale):
        self._c(self._L.tc_set_edge_margin_scale(self._h, float(scale)))

    def set_edge_margin_offset(self, offset):
        self._c(self._L.tc_set_edge_margin_offset(self._h, float(offset)))

    def get_num_collider_edges(self):
        v = C.c_uint32()
        self._c(self._L.tc_get_num_collider_edges(self._h, C.byref(v)))
        return v.value

    # ---------------- sewing (lib.rs:2798-2925)
    def get_num_sewing_constraints(self):
        v = C.c_uint32()
        self._c(self._L.tc_get_num_sewing_constraints(self._h, C.byref(v)))
        return v.value

    def set_sewing_stiffness(self, stiffness=10000.0):
        self._c(self._L.tc_set_sewing_stiffness(self._h, float(stiffness)))

    def set_sewing_shrink_speed(self, speed=1.0):
        self._c(self._L.tc_set_sewing_shrink_speed(self._h, float(speed)))

    def get_sewing_shrink_speed(self):
        v = C.c_float()
        self._c(self._L.tc_get_sewing_shrink_speed(self._h, C.byref(v)))
        return v.value

    def set_enable_sewing_lock(self, enabled=True):
        self._c(self._L.tc_set_enable_sewing_lock(self._h, int(bool(enabled))))

    def set_sewing_lock_distance(self, distance=0.02):
        self._c(self._L.tc_set_sewing_lock_distance(self._h, float(distance)))

    def get_sewing_lock_distance(self):
        v = C.c_float()
        self._c(self._L.tc_get_sewing_lock_distance(self._h, C.byref(v)))
        return v.value

    def get_sewing_current_rest_lengths(self):
        out = np.zeros(self.get_num_sewing_constraints(), _f32)
        self._c(self._L.tc_get_sewing_current_rest_lengths(self._h, _ptr(out), out.size))
        return [float(x) for x in out]

    def set_sewing_current_rest_lengths(self, values):
        v = np.ascontiguousarray(np.asarray(values, dtype=_f32).reshape(-1))
        self._c(self._L.tc_set_sewing_current_rest_lengths(self._h, _ptr(v), v.size))

    def set_sewing_priority_options(self, enabled, threshold=0.9, merge_dist=0.005, ramp_frames=3, max_frames=600):
        self._c(self._L.tc_set_sewing_priority_options(self._h, int(bool(enabled)), float(threshold),
                                                        float(merge_dist), int(ramp_frames), int(max_frames)))

    def set_sewing_priority_state(self, latched, frame, ramp_t, ratio):
        self._c(self._L.tc_set_sewing_priority_state(self._h, int(bool(latched)), int(frame), float(ramp_t),
                                                      float(ratio)))

    def update_sewing_priority(self, positions):
        """(closure ratio, gravity scale, latched) from host positions (N x 3)."""
        p = _arr(positions, _f32, 3, "positions")
        out = np.zeros(3, _f32)
        self._c(self._L.tc_update_sewing_priority(self._h, _ptr(p), p.shape[0], _ptr(out)))
        return float(out[0]), float(out[1]), bool(out[2] > 0.5)

    def _sewing_priority(self):
        out = np.zeros(4, _f32)
        self._c(self._L.tc_get_sewing_priority(self._h, _ptr(out)))
        return out

    def get_sewing_priority_scale(self):
        return float(self._sewing_priority()[0])

    def get_sewing_closure_ratio(self):
        return float(self._sewing_priority()[1])

    def is_sewing_priority_active(self):
        return bool(self._sewing_priority()[2] > 0.5)

    def set_positions_and_velocities(self, positions, velocities=None):
        p = _arr(positions, _f32, 3, "positions")
        v = None if velocities is None else _arr(velocities, _f32, 3, "velocities")
        self._c(self._L.tc_set_positions_and_velocities(self._h, _ptr(p), _ptr(v), p.shape[0]))

    def reset(self):
        self._c(self._L.tc_reset(self._h))

    # ---------------- parameters
    def set_gravity(self, gx, gy, gz):
        self._c(self._L.tc_set_gravity(self._h, gx, gy, gz))

    def set_damping(self, damping):
        self._c(self._L.tc_set_damping(self._h, damping))

    def set_damping_all(self, tension_damp, compression_damp, shear_damp, bending_damp):
        self._c(self._L.tc_set_damping_all(self._h, tension_damp, compression_damp, shear_damp, bending_damp))

    def set_solver_iterations(self, iterations):
        self._solver_iterations = max(int(iterations), 1)
        self._c(self._L.tc_set_solver_iterations(self._h, int(iterations)))

    def get_effective_solver_iterations(self):
        return self._solver_iterations

    def set_stiffness(self, stretch_stiffness, bending_stiffness):
        self.set_stiffness_all(stretch_stiffness, stretch_stiffness, stretch_stiffness * 0.5, bending_stiffness)

    def set_stiffness_all(self, tension_stiffness, compression_stiffness, shear_stiffness, bending_stiffness):
        self._c(self._L.tc_set_stiffness_all(self._h, tension_stiffness, compression_stiffness, shear_stiffness,
                                             bending_stiffness))

    def set_compliance_all(self, tension, compression, shear, bending):
        """Set XPBD compliances (m/N) directly (no stiffness mapping)."""
        self._c(self._L.tc_set_compliance_all(self._h, tension, compression, shear, bending))

    def reset_edge_stiffness_multipliers(self):
        self._c(self._L.tc_reset_edge_stiffness_multipliers(self._h))

    # ---------------- rest lengths per input edge (lib.rs:2684-2733)
    def set_edge_rest_length_scales(self, edge_indices, scales):
        i = np.ascontiguousarray(edge_indices, _u32).reshape(-1)
        m = np.ascontiguousarray(scales, _f32).reshape(-1)
        self._c(self._L.tc_set_edge_rest_length_scales(self._h, _ptr(i), _ptr(m), min(i.size, m.size)))

    def reset_edge_rest_lengths(self):
        self._c(self._L.tc_reset_edge_rest_lengths(self._h))

    def _edge_constraint(self, edge_idx):
        out = np.zeros(3, _f32)
        self._c(self._L.tc_get_edge_constraint(self._h, int(edge_idx), _ptr(out)))
        return out

    def get_edge_rest_length(self, edge_idx):
        return float(self._edge_constraint(edge_idx)[0])

    def get_edge_initial_rest_length(self, edge_idx):
        return float(self._edge_constraint(edge_idx)[1])

    def get_edge_tension_compliance(self, edge_idx):
        return float(self._edge_constraint(edge_idx)[2])

    def set_edge_stiffness_multipliers(self, edge_indices, multipliers):
        i = np.ascontiguousarray(edge_indices, _u32)
        m = np.ascontiguousarray(multipliers, _f32)
        k = min(i.size, m.size)
        self._c(self._L.tc_set_edge_stiffness_multipliers(self._h, _ptr(i), _ptr(m), k))

    def set_enable_self_collision(self, enable):
        self._c(self._L.tc_set_enable_self_collision(self._h, int(bool(enable))))

    def set_self_collision_options(self, relief_factor=0.2, max_displacement_ratio=0.2, exclude_neighbors=True,
                                   enable_normal_untangling=True, max_iterations=128):
        self._c(self._L.tc_set_self_collision_options(self._h, relief_factor, max_displacement_ratio,
                                                      int(exclude_neighbors), int(enable_normal_untangling),
                                                      int(max_iterations)))
        self._untangle = bool(enable_normal_untangling)

    def set_coupled_collider(self, enabled):
        self._c(self._L.tc_set_coupled_collider(self._h, int(bool(enabled))))

    def set_auto_coupled_on_low_substeps(self, enabled):
        self._c(self._L.tc_set_auto_coupled_on_low_substeps(self._h, int(bool(enabled))))

    def set_collider_options(self, enable_cluster_culling=False, enable_single_sided_recovery=True,
                             sweep_margin=0.05):
        self._c(self._L.tc_set_collider_options(self._h, int(enable_cluster_culling),
                                                int(enable_single_sided_recovery), sweep_margin))

    # ---------------- colliders
    def add_sphere_collider(self, center, radius, friction=0.0, restitution=0.0):
        self._c(self._L.tc_add_sphere_collider(self._h, _ptr(np.asarray(center, _f32)), radius, friction,
                                               restitution))

    def add_capsule_collider(self, point_a, point_b, radius, friction=0.0, restitution=0.0):
        self._c(self._L.tc_add_capsule_collider(self._h, _ptr(np.asarray(point_a, _f32)),
                                                _ptr(np.asarray(point_b, _f32)), radius, friction, restitution))

    def add_plane_collider(self, point, normal, friction=0.0, restitution=0.0):
        self._c(self._L.tc_add_plane_collider(self._h, _ptr(np.asarray(point, _f32)), _ptr(np.asarray(normal, _f32)),
                                              friction, restitution))

    def set_mesh_collider_triangles(self, triangles, friction=0.3, thickness=0.01, restitution=0.0,
                                    single_sided=True, attributes=None):
        t = np.ascontiguousarray(triangles, _f32)
        if t.ndim != 3 or t.shape[1:] != (3, 3):
            raise ValueError("each triangle must have shape [3, 3]")
        a = None
        if attributes is not None:
            a = np.ascontiguousarray(attributes, _f32)
            if a.ndim != 2 or a.shape[0] < t.shape[0] or a.shape[1] < 4:
                raise ValueError("attributes must have shape (N_triangles, >=4)")
            a = np.ascontiguousarray(a[:, :4])
        self._c(self._L.tc_set_mesh_collider_triangles(self._h, _ptr(t), t.shape[0], friction, thickness,
                                                       restitution, int(bool(single_sided)), _ptr(a)))

    def clear_colliders(self):
        self._c(self._L.tc_clear_colliders(self._h))

    # ---------------- pins
    def set_pin(self, vertex_idx, target_pos, weight=1.0):
        self._c(self._L.tc_set_pin(self._h, int(vertex_idx), _ptr(np.asarray(target_pos, _f32)), weight))

    def set_pins_batch(self, indices, targets, weights):
        i = np.ascontiguousarray(indices, _u32)
        t = _arr(targets, _f32, 3, "targets")
        w = np.ascontiguousarray(weights, _f32)
        k = min(i.size, t.shape[0], w.size)
        self._c(self._L.tc_set_pins_batch(self._h, _ptr(i), _ptr(t), _ptr(w), k))

    def release_pin(self, vertex_idx):
        self._c(self._L.tc_release_pin(self._h, int(vertex_idx)))

    def release_pins_batch(self, indices):
        for v in indices:
            self.release_pin(v)

    def clear_pins(self):
        self._c(self._L.tc_clear_pins(self._h))

    def set_vertex_inv_masses(self, indices, inv_masses):
        i = np.ascontiguousarray(indices, _u32)
        w = np.ascontiguousarray(inv_masses, _f32)
        self._c(self._L.tc_set_vertex_inv_masses(self._h, _ptr(i), _ptr(w), min(i.size, w.size)))

    def get_vertex_inv_masses(self):
        o = np.empty(self._n, _f32)
        self._c(self._L.tc_get_vertex_inv_masses(self._h, _ptr(o), self._n))
        return o

    # ---------------- counts / introspection
    def _counts(self):
        o = np.zeros(8, _u32)
        self._c(self._L.tc_get_counts(self._h, _ptr(o)))
        return o

    def get_num_vertices(self):
        return int(self._counts()[0])

    def get_num_distance_constraints(self):
        return int(self._counts()[1])

    def get_num_bending_constraints(self):
        return int(self._counts()[2])

    def get_has_multiple_layers(self):
        return bool(self._counts()[7])

    def get_counts(self):
        c = self._counts()
        keys = ["n", "nd", "nb", "n_edges", "n_dist_colors", "n_bend_colors", "table_size", "multi_layer"]
        return dict(zip(keys, (int(v) for v in c)))

    def get_cell_size(self):
        v = C.c_float()
        self._c(self._L.tc_get_cell_size(self._h, C.byref(v)))
        return v.value

    def get_state(self):
        x, p, v = (np.empty((self._n, 3), _f32) for _ in range(3))
        self._c(self._L.tc_get_state(self._h, _ptr(x), _ptr(p), _ptr(v)))
        return x, p, v

    def get_coloring(self):
        c = self.get_counts()
        dv = np.zeros((max(c["nd"], 1), 2), _u32)
        dp = np.zeros((max(c["nd"], 1), 4), _f32)
        do, dc = np.zeros(max(c["n_dist_colors"], 1), _u32), np.zeros(max(c["n_dist_colors"], 1), _u32)
        self._c(self._L.tc_get_distance_constraints(self._h, _ptr(dv), _ptr(dp), _ptr(do), _ptr(dc)))
        bv = np.zeros((max(c["nb"], 1), 4), _u32)
        bp = np.zeros((max(c["nb"], 1), 4), _f32)
        bo, bc = np.zeros(max(c["n_bend_colors"], 1), _u32), np.zeros(max(c["n_bend_colors"], 1), _u32)
        self._c(self._L.tc_get_bending_constraints(self._h, _ptr(bv), _ptr(bp), _ptr(bo), _ptr(bc)))
        k, m = c["n_dist_colors"], c["n_bend_colors"]
        return dict(dist_v=dv[:c["nd"]], dist_par=dp[:c["nd"]], dist_off=do[:k], dist_cnt=dc[:k],
                    bend_v=bv[:c["nb"]], bend_par=bp[:c["nb"]], bend_off=bo[:m], bend_cnt=bc[:m])

    def get_hash_state(self, which=0):
        c = self.get_counts()
        cs = np.zeros(c["table_size"] + 1, _u32)
        cnt = self._n if which == 0 else c["n_edges"]
        srt = np.zeros(max(cnt, 1), _u32)
        self._c(self._L.tc_get_hash_state(self._h, int(which), _ptr(cs), _ptr(srt)))
        return cs, srt[:cnt]

    def get_edges(self):
        ne = self.get_counts()["n_edges"]
        e = np.zeros((max(ne, 1), 2), _u32)
        b = np.zeros(max((ne + 31) // 32, 1), _u32)
        self._c(self._L.tc_get_edges(self._h, _ptr(e), _ptr(b)))
        return e[:ne], b[:(ne + 31) // 32]

    def set_residual_tracking(self, enable=True):
        self._c(self._L.tc_set_residual_tracking(self._h, int(bool(enable))))

    def get_residuals(self):
        c = self.get_counts()
        k, m = max(c["n_dist_colors"], 1), max(c["n_bend_colors"], 1)
        dr, dm, br, bm = np.zeros(k, _f32), np.zeros(k, _f32), np.zeros(m, _f32), np.zeros(m, _f32)
        tot = np.zeros(4, _f32)
        self._c(self._L.tc_get_residuals(self._h, _ptr(dr), _ptr(dm), _ptr(br), _ptr(bm), _ptr(tot)))
        return dict(dist_rms=dr[:c["n_dist_colors"]], dist_max=dm[:c["n_dist_colors"]],
                    bend_rms=br[:c["n_bend_colors"]], bend_max=bm[:c["n_bend_colors"]],
                    dist_rms_total=float(tot[0]), dist_max_total=float(tot[1]),
                    bend_rms_total=float(tot[2]), bend_max_total=float(tot[3]))

    def get_predicted_residual(self):
        """With residual tracking: RMS |C| of the last substep's predicted
        positions (before any iteration)."""
        v = C.c_float()
        self._c(self._L.tc_get_predicted_residual(self._h, C.byref(v)))
        return v.value

    def set_profiling_enabled(self, enable):
        self._c(self._L.tc_set_profiling_enabled(self._h, int(bool(enable))))
        return bool(enable)

    def take_profile(self):
        """[(pass name, total ms, launch groups)] since the last call."""
        buf = C.create_string_buffer(4096)
        ms = np.zeros(64, _f32)
        cnt = np.zeros(64, _u32)
        k = C.c_uint32()
        self._c(self._L.tc_take_profile(self._h, buf, 4096, _ptr(ms), _ptr(cnt), 64, C.byref(k)))
        names = buf.value.decode().split("\n")[:k.value]
        return [(nm, float(ms[i]), int(cnt[i])) for i, nm in enumerate(names)]

    def set_persistent_solver(self, enable=True):
        """One cooperative launch per substep (per frame without self-collision)
        with bounded grid barriers between colours; off = one launch per colour."""
        self._c(self._L.tc_set_persistent_solver(self._h, int(bool(enable))))

    def set_launch_config(self, persistent=True, blocks_per_sm=4):
        """persistent: False = one launch per colour, True = persistent cooperative
        solver with `blocks_per_sm`, 2 = cluster solver (batched instances),
        3 = staged cluster solver (batched instances, vertex records in the
        clusters' shared memory)."""
        mode = int(persistent) if persistent in (2, 3) and persistent is not True else int(bool(persistent))
        self._c(self._L.tc_set_launch_config(self._h, mode, int(blocks_per_sm)))

    def get_launch_limits(self):
        a, b = C.c_uint32(), C.c_uint32()
        self._c(self._L.tc_get_launch_limits(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def check_barrier_timeout(self, spin_limit=1000):
        """Run a barrier that can never be released; raises BarrierTimeout."""
        self._c(self._L.tc_check_barrier_timeout(self._h, int(spin_limit)))

    def frame_kernel_count(self):
        """Kernel launches in the recorded frame graph."""
        v = C.c_uint32()
        self._c(self._L.tc_frame_kernel_count(self._h, C.byref(v)))
        return v.value

    def last_frame_ms(self):
        v = C.c_float()
        self._c(self._L.tc_last_frame_ms(self._h, C.byref(v)))
        return v.value

    def get_ccd_queue(self):
        """(edge pairs deferred to the CCD kernel in the latest self-collision pass, capacity)"""
        out = np.zeros(2, _u32)
        self._c(self._L.tc_get_ccd_queue(self._h, _ptr(out)))
        return int(out[0]), int(out[1])

    # ---- adaptive substeps and iterations (lib.rs:1788-1805, :1950-1965)
    def set_adaptive_substep_options(self, enabled, min_substeps=4, max_substeps=64):
        self._c(self._L.tc_set_adaptive_substep_options(self._h, int(bool(enabled)), int(min_substeps),
                                                        int(max_substeps)))

    def set_auto_compensate_iterations(self, enabled):
        self._c(self._L.tc_set_auto_compensate_iterations(self._h, int(bool(enabled))))

    def set_strain_adaptive_options(self, enabled, tolerance=0.008):
        self._c(self._L.tc_set_strain_adaptive_options(self._h, int(bool(enabled)), float(tolerance)))

    def note_external_displacement(self, disp):
        self._c(self._L.tc_note_external_displacement(self._h, float(disp)))

    def _adaptive(self):
        out = np.zeros(6, _f32)
        self._c(self._L.tc_get_adaptive_state(self._h, _ptr(out)))
        return out

    def get_effective_substeps(self):
        return int(self._adaptive()[0])

    def get_effective_solver_iterations(self):
        return int(self._adaptive()[1])

    def get_last_step_max_strain(self):
        return float(self._adaptive()[2])

    # ---- self-collision substep intervals (lib.rs:1966-2000)
    def set_self_collision_substep_interval(self, interval):
        self._c(self._L.tc_set_self_collision_substep_interval(self._h, int(interval)))

    def set_self_collision_ee_substep_interval(self, interval):
        self._c(self._L.tc_set_self_collision_ee_substep_interval(self._h, int(interval)))

    def _intervals(self):
        out = np.zeros(2, _u32)
        self._c(self._L.tc_get_self_collision_intervals(self._h, _ptr(out)))
        return out

    def get_self_collision_substep_interval(self):
        return int(self._intervals()[0])

    def get_self_collision_ee_substep_interval(self):
        return int(self._intervals()[1])

    # ---- bone SDF colliders (lib.rs:2245-2600)
    @staticmethod
    def _mats(a, name):
        m = np.ascontiguousarray(np.asarray(a, _f32))
        if m.ndim != 3 or m.shape[1:] != (4, 4):
            raise ValueError(f"{name} must have shape (N, 4, 4)")
        return m

    @staticmethod
    def _dirty(d):
        if d is None:
            return None, -1
        x = np.ascontiguousarray(np.asarray(d, _u32).ravel())
        return x, x.size

    def set_bone_sdf_colliders(self, width, height, depth, texture_bytes, bone_infos):
        """Static atlas: Rg16Float texture bytes (width x height x depth x 4) and
        bone_infos of shape (N, 20)."""
        tex = np.frombuffer(bytes(texture_bytes), dtype=np.uint32)
        info = np.ascontiguousarray(np.asarray(bone_infos, _f32))
        if info.ndim != 2 or (info.size and info.shape[1] < 20):
            raise ValueError("bone_infos rows need at least 20 elements")
        info = np.ascontiguousarray(info[:, :20]) if info.size else np.zeros((0, 20), _f32)
        self._c(self._L.tc_set_bone_sdf_colliders(self._h, int(width), int(height), int(depth), _ptr(tex),
                                                  tex.size, _ptr(info), info.shape[0]))

    def update_bone_transforms(self, world_matrices, inv_world_matrices, dirty_bone_indices=None):
        w = self._mats(world_matrices, "world_matrices")
        iw = self._mats(inv_world_matrices, "inv_world_matrices")
        if iw.shape[0] != w.shape[0]:
            raise ValueError("world_matrices and inv_world_matrices need the same shape (N, 4, 4)")
        d, nd = self._dirty(dirty_bone_indices)
        self._c(self._L.tc_update_bone_transforms(self._h, _ptr(w), _ptr(iw), w.shape[0], _ptr(d), nd))

    def set_dynamic_bone_sdf_dirty_bones(self, dirty_bone_indices=None):
        d, nd = self._dirty(dirty_bone_indices)
        self._c(self._L.tc_set_dynamic_bone_sdf_dirty_bones(self._h, _ptr(d), nd))

    def clear_bone_sdf_colliders(self):
        self._c(self._L.tc_clear_bone_sdf_colliders(self._h))

    def setup_dynamic_bone_sdf(self, width, height, depth, res, bone_infos, rest_verts, bone_indices, bone_weights,
                               tri_sources, tri_weights, bone_bind_inv_matrices, update_interval=1):
        if res == 0 or width == 0 or height == 0 or depth == 0:
            raise ValueError("width, height, depth and res must be >= 1")
        info = np.ascontiguousarray(np.asarray(bone_infos, _f32))
        if info.ndim != 2 or info.shape[1] < 20:
            raise ValueError("bone_infos rows need at least 20 elements")
        info = np.ascontiguousarray(info[:, :20])
        rv = np.ascontiguousarray(np.asarray(rest_verts, _f32))
        bi = np.ascontiguousarray(np.asarray(bone_indices, _u32))
        bw = np.ascontiguousarray(np.asarray(bone_weights, _f32))
        if rv.ndim != 2 or rv.shape[1] < 3 or bi.ndim != 2 or bi.shape[1] < 4 or bw.ndim != 2 or bw.shape[1] < 4:
            raise ValueError("rest_verts needs >= 3 columns, bone_indices / bone_weights >= 4")
        if bi.shape[0] != rv.shape[0] or bw.shape[0] != rv.shape[0]:
            raise ValueError("rest_verts, bone_indices and bone_weights need the same vertex count")
        bi = np.ascontiguousarray(bi[:, :4])
        bw = np.ascontiguousarray(bw[:, :4])
        ts = np.ascontiguousarray(np.asarray(tri_sources, _u32))
        tw = np.ascontiguousarray(np.asarray(tri_weights, _f32))
        if ts.ndim != 2 or ts.shape[1] < 4 or tw.ndim != 2 or tw.shape[1] < 3 or tw.shape[0] != ts.shape[0]:
            raise ValueError("tri_sources (M, 4) and tri_weights (M, 3) are required")
        ts = np.ascontiguousarray(ts[:, :4])
        tw = np.ascontiguousarray(tw[:, :3])
        inv = self._mats(bone_bind_inv_matrices, "bone_bind_inv_matrices")
        self._c(self._L.tc_setup_dynamic_bone_sdf(
            self._h, int(width), int(height), int(depth), int(res), _ptr(info), info.shape[0], _ptr(rv), rv.shape[1],
            _ptr(bi), _ptr(bw), rv.shape[0], _ptr(ts), _ptr(tw), ts.shape[0], _ptr(inv), inv.shape[0],
            int(update_interval)))

    def set_dynamic_bone_sdf_enabled(self, enabled):
        self._c(self._L.tc_set_dynamic_bone_sdf_enabled(self._h, int(bool(enabled))))

    def set_dynamic_bone_sdf_update_interval(self, interval):
        self._c(self._L.tc_set_dynamic_bone_sdf_update_interval(self._h, int(interval)))

    def get_bone_sdf_atlas(self):
        """(width, height, depth), uint32 texels (packed half2: distance, alpha)."""
        dims = np.zeros(3, _u32)
        self._c(self._L.tc_get_bone_sdf_atlas(self._h, None, 0, _ptr(dims)))
        out = np.zeros(int(dims[0]) * int(dims[1]) * int(dims[2]), _u32)
        self._c(self._L.tc_get_bone_sdf_atlas(self._h, _ptr(out), out.size, _ptr(dims)))
        return tuple(int(x) for x in dims), out

    def get_bone_infos(self):
        n = C.c_uint32()
        self._c(self._L.tc_get_bone_infos(self._h, None, 0, C.byref(n)))
        out = np.zeros((n.value, 20), _f32)
        self._c(self._L.tc_get_bone_infos(self._h, _ptr(out), out.size, C.byref(n)))
        return out

    # ---- learned warm start (new; no counterpart in the reference)
    def ws_enable(self, k_replaced=1, res_thresh=float("inf")):
        """Warm-start every substep with the graph MLP, run iterations - k
        plain iterations, and the k others when the max residual is above
        res_thresh (the plain solver's residual)."""
        self._c(self._L.tc_ws_enable(self._h, 1, int(k_replaced), float(res_thresh)))

    def ws_disable(self):
        self._c(self._L.tc_ws_enable(self._h, 0, 0, 0.0))

    def ws_set_kernel(self, kind=0):
        """Tensor-core path of the network's message-passing layers (inference
        and training): 0 tcgen05 (default), 1 warp-level mma.sync."""
        self._c(self._L.tc_ws_set_kernel(self._h, int(kind)))

    def ws_record(self, capacity, every=1):
        """Record `capacity` training snapshots, one every `every` substeps,
        during the following plain frames."""
        self._c(self._L.tc_ws_record(self._h, int(capacity), int(every)))

    def ws_recorded(self):
        v = C.c_uint32()
        self._c(self._L.tc_ws_recorded(self._h, C.byref(v)))
        return v.value

    def ws_train(self, epochs=50, lr=1e-3, seed=0):
        """Adam on the recorded snapshots; (mean loss of the first epoch, of the last)."""
        a, b = C.c_float(), C.c_float()
        self._c(self._L.tc_ws_train(self._h, int(epochs), float(lr), int(seed), C.byref(a), C.byref(b)))
        return a.value, b.value

    def ws_params(self):
        out = np.zeros(self._L.tc_ws_param_count(), _f32)
        self._c(self._L.tc_ws_get_params(self._h, _ptr(out), out.size))
        return out

    def ws_set_params(self, params):
        p = _arr(params, _f32).ravel()
        self._c(self._L.tc_ws_set_params(self._h, _ptr(p), p.size))

    def ws_stats(self):
        """{'substeps', 'fallbacks', 'last_residual', 'threshold'}"""
        out = np.zeros(4, np.float64)
        self._c(self._L.tc_ws_stats(self._h, _ptr(out)))
        return {"substeps": int(out[0]), "fallbacks": int(out[1]), "last_residual": float(out[2]),
                "threshold": float(out[3])}

    def ws_set_relative_threshold(self, ratio):
        """ratio > 0: a warm-started substep falls back when its residual is
        above ratio x the residual of its predicted positions; 0 returns to
        the absolute threshold of ws_enable."""
        self._c(self._L.tc_ws_set_relative_threshold(self._h, float(ratio)))

    def ws_reset_stats(self):
        self._c(self._L.tc_ws_reset_stats(self._h))


class BatchedClothSimulator(ClothSimulator):
    """Many independent cloths in one simulator (one persistent launch per frame).

    ``instances`` is a list of dicts with ``positions`` (N_k x 3), ``edges``,
    ``faces``, optional ``inv_masses``, ``compliance`` = (tension,
    compression, shear, bending) and ``colliders`` = list of
    ``("sphere", center, radius, friction)`` or
    ``("capsule", a, b, radius, friction)``.  Vertex ``v`` of instance ``k``
    is simulator vertex ``offsets[k] + v``.  Each instance evolves exactly as
    it would in its own ``ClothSimulator``.
    """

    def __init__(self, instances, thickness=0.005, device=0):
        L = _lib.load()
        self._h = None
        pos, edges, faces, inv, comp, pcnt, prims = [], [], [], [], [], [], []
        vc, ec, fc = [], [], []
        for inst in instances:
            p = _arr(inst["positions"], _f32, 3, "positions")
            e = _arr(inst["edges"], _u32, 2, "edges")
            f = _arr(inst.get("faces", np.zeros((0, 3), _u32)), _u32, 3, "faces")
            pos.append(p); edges.append(e); faces.append(f)
            vc.append(p.shape[0]); ec.append(e.shape[0]); fc.append(f.shape[0])
            im = inst.get("inv_masses")
            inv.append(np.ones(p.shape[0], _f32) if im is None else np.asarray(im, _f32).reshape(-1))
            comp.append(np.asarray(inst["compliance"], _f32).reshape(4))
            cols = inst.get("colliders", [])
            pcnt.append(len(cols))
            for c in cols:
                if c[0] == "sphere":
                    _, ctr, r, fr = c
                    prims.append([0, fr, 0.0, r, *ctr, 0.0, 0.0, 0.0])
                elif c[0] == "capsule":
                    _, a, b, r, fr = c
                    prims.append([1, fr, 0.0, r, *a, *b])
                else:
                    raise ValueError(f"unknown collider kind {c[0]!r}")
        P = np.ascontiguousarray(np.concatenate(pos), _f32)
        E = np.ascontiguousarray(np.concatenate(edges), _u32)
        Fa = np.ascontiguousarray(np.concatenate(faces), _u32)
        I = np.ascontiguousarray(np.concatenate(inv), _f32)
        Cm = np.ascontiguousarray(np.stack(comp), _f32)
        Pr = np.ascontiguousarray(np.asarray(prims, _f32).reshape(-1, 10))
        arrs = [np.asarray(x, _u32) for x in (vc, ec, fc, pcnt)]
        h = C.c_void_p()
        _lib.check(L.tc_batch_create(C.byref(h), len(instances), _ptr(arrs[0]), _ptr(arrs[1]), _ptr(arrs[2]),
                                     _ptr(P), _ptr(E), _ptr(Fa), _ptr(I), float(thickness), _ptr(Cm), _ptr(arrs[3]),
                                     _ptr(Pr), int(device)))
        self._h = h
        self._L = L
        self._n = P.shape[0]
        self._solver_iterations = 2
        self.offsets = np.concatenate([[0], np.cumsum(vc)]).astype(np.int64)
