"""Loader for the in-tree CUDA library ``libtcloth.so`` (C ABI in include/tcloth.h).

There is no CPU fallback: importing works without a GPU (so the C ABI can be
inspected), but creating a simulator fails with ``RuntimeError`` when the
library is missing or no CUDA device is visible.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtcloth.so")

TC_OK, TC_ERR_INVALID, TC_ERR_CUDA, TC_ERR_NOMEM, TC_ERR_TIMEOUT, TC_ERR_NONFINITE = range(6)

_P = C.c_void_p
_U = C.c_uint32
_F = C.c_float
_I = C.c_int

# name -> argtypes (all return tc_status unless listed in _RESTYPES)
SIGNATURES = {
    "tc_last_error": [],
    "tc_gpu_available": [],
    "tc_device_name": [_I, C.c_char_p, C.c_size_t],
    "tc_create": [C.POINTER(_P), _P, _U, _P, _U, _P, _U, _P, _P, _P, _U, _F, _F, _F, _F, _F, _I],
    "tc_create_sewn": [C.POINTER(_P), _P, _U, _P, _U, _P, _U, _P, _P, _P, _U, _F, _F, _F, _F, _F, _P, _U, _F, _F, _I,
                       _F, _I],
    "tc_destroy": [_P],
    "tc_batch_create": [C.POINTER(_P), _U, _P, _P, _P, _P, _P, _P, _P, _F, _P, _P, _P, _I],
    "tc_batch_instance_offsets": [_P, _P, _U, C.POINTER(_U)],
    "tc_step": [_P, _F, _U, C.POINTER(_U)],
    "tc_step_async": [_P, _F, _U],
    "tc_fetch_positions": [_P, _P, C.c_size_t, C.POINTER(_I)],
    "tc_step_buffered": [_P, _F, _U, C.POINTER(_U)],
    "tc_fetch_buffered_positions": [_P, _P, C.c_size_t, C.POINTER(_U)],
    "tc_get_buffered_frame_count": [_P, C.POINTER(_U)],
    "tc_clear_frame_buffer": [_P],
    "tc_get_positions": [_P, _P, C.c_size_t],
    "tc_set_positions_and_velocities": [_P, _P, _P, _U],
    "tc_reset": [_P],
    "tc_set_gravity": [_P, _F, _F, _F],
    "tc_set_enable_edge_collision": [_P, _I],
    "tc_compute_combined_inv_masses": [_P, _U, _P, _U, _P, _U, _P, _U, _F, _F, _P],
    "tc_color_edge_pairs": [_U, _P, _U, _P],
    "tc_set_pair_recording": [_P, _I, _U, _U],
    "tc_set_self_collision_variant": [_P, _U],
    "tc_set_ee_pair_list_capacity": [_P, C.c_uint64],
    "tc_set_launch_block": [_P, _U],
    "tc_set_hash_cell_size": [_P, _F],
    "tc_mark_device_lost": [_I],
    "tc_device_status": [_I, C.POINTER(_I), C.POINTER(C.c_uint64)],
    "tc_set_nonfinite_check": [_P, _I],
    "tc_get_pair_lists": [_P, _P, _U, _P, _U, _P],
    "tc_get_config_json": [_P, C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)],
    "tc_get_config_hash": [_P, C.POINTER(C.c_uint64)],
    "tc_set_workgroup_size": [_P, _U],
    "tc_set_areal_density": [_P, _F],
    "tc_set_coupled_self_collision_options": [_P, _U, _U],
    "tc_find_triangle_intersections": [_P, _U, _P, _U, _I, _F, _P, _U, _P, _U, C.POINTER(_U)],
    "tc_reset_edge_stiffness_multipliers": [_P],
    "tc_set_edge_rest_length_scales": [_P, _P, _P, _U],
    "tc_reset_edge_rest_lengths": [_P],
    "tc_get_edge_constraint": [_P, _U, _P],
    "tc_step_single_substep": [_P, _F],
    "tc_get_num_virtual_vertices": [_P, C.POINTER(_U)],
    "tc_set_enable_pair_cache": [_P, _I],
    "tc_get_enable_pair_cache": [_P, C.POINTER(_I)],
    "tc_set_self_collision_algorithm": [_P, _U],
    "tc_get_self_collision_algorithm": [_P, C.POINTER(_U)],
    "tc_set_pair_cache_options": [_P, _U, _U, _U, _F, _F, _F],
    "tc_set_enable_pair_cache_final_fallback": [_P, _I],
    "tc_get_enable_pair_cache_final_fallback": [_P, C.POINTER(_I)],
    "tc_get_pair_cache_stats": [_P, _P],
    "tc_get_active_pairs": [_P, _P, _P, C.c_size_t, _P, C.c_size_t],
    "tc_set_edge_margin_scale": [_P, _F],
    "tc_set_edge_margin_offset": [_P, _F],
    "tc_get_num_collider_edges": [_P, C.POINTER(_U)],
    "tc_get_num_sewing_constraints": [_P, C.POINTER(_U)],
    "tc_set_sewing_stiffness": [_P, _F],
    "tc_set_sewing_shrink_speed": [_P, _F],
    "tc_get_sewing_shrink_speed": [_P, C.POINTER(_F)],
    "tc_set_enable_sewing_lock": [_P, _I],
    "tc_set_sewing_lock_distance": [_P, _F],
    "tc_get_sewing_lock_distance": [_P, C.POINTER(_F)],
    "tc_get_sewing_current_rest_lengths": [_P, _P, C.c_size_t],
    "tc_set_sewing_current_rest_lengths": [_P, _P, C.c_size_t],
    "tc_set_sewing_priority_options": [_P, _I, _F, _F, _U, _U],
    "tc_set_sewing_priority_state": [_P, _I, _U, _F, _F],
    "tc_update_sewing_priority": [_P, _P, _U, _P],
    "tc_get_sewing_priority": [_P, _P],
    "tc_set_damping": [_P, _F],
    "tc_set_damping_all": [_P, _F, _F, _F, _F],
    "tc_set_solver_iterations": [_P, _U],
    "tc_set_stiffness_all": [_P, _F, _F, _F, _F],
    "tc_set_compliance_all": [_P, _F, _F, _F, _F],
    "tc_set_edge_stiffness_multipliers": [_P, _P, _P, _U],
    "tc_set_enable_self_collision": [_P, _I],
    "tc_set_self_collision_options": [_P, _F, _F, _I, _I, _U],
    "tc_set_coupled_collider": [_P, _I],
    "tc_set_auto_coupled_on_low_substeps": [_P, _I],
    "tc_set_collider_options": [_P, _I, _I, _F],
    "tc_add_sphere_collider": [_P, _P, _F, _F, _F],
    "tc_add_capsule_collider": [_P, _P, _P, _F, _F, _F],
    "tc_add_plane_collider": [_P, _P, _P, _F, _F],
    "tc_set_mesh_collider_triangles": [_P, _P, _U, _F, _F, _F, _I, _P],
    "tc_clear_colliders": [_P],
    "tc_set_pin": [_P, _U, _P, _F],
    "tc_set_pins_batch": [_P, _P, _P, _P, _U],
    "tc_release_pin": [_P, _U],
    "tc_clear_pins": [_P],
    "tc_set_vertex_inv_masses": [_P, _P, _P, _U],
    "tc_get_vertex_inv_masses": [_P, _P, _U],
    "tc_get_counts": [_P, _P],
    "tc_get_cell_size": [_P, C.POINTER(_F)],
    "tc_get_state": [_P, _P, _P, _P],
    "tc_get_distance_constraints": [_P, _P, _P, _P, _P],
    "tc_get_bending_constraints": [_P, _P, _P, _P, _P],
    "tc_get_hash_state": [_P, _I, _P, _P],
    "tc_get_edges": [_P, _P, _P],
    "tc_set_residual_tracking": [_P, _I],
    "tc_get_residuals": [_P, _P, _P, _P, _P, _P],
    "tc_last_frame_ms": [_P, C.POINTER(_F)],
    "tc_set_profiling_enabled": [_P, _I],
    "tc_frame_kernel_count": [_P, C.POINTER(_U)],
    "tc_set_persistent_solver": [_P, _I],
    "tc_set_launch_config": [_P, _I, _U],
    "tc_get_launch_limits": [_P, C.POINTER(_U), C.POINTER(_U)],
    "tc_check_barrier_timeout": [_P, _U],
    "tc_hash_build_static": [_P, _U, _F, _U, _P, _P, _P],
    "tc_take_profile": [_P, C.c_char_p, C.c_size_t, _P, _P, _U, C.POINTER(_U)],
    "tc_get_ccd_queue": [_P, _P],
    "tc_set_adaptive_substep_options": [_P, _I, _U, _U],
    "tc_set_auto_compensate_iterations": [_P, _I],
    "tc_set_strain_adaptive_options": [_P, _I, _F],
    "tc_note_external_displacement": [_P, _F],
    "tc_get_adaptive_state": [_P, _P],
    "tc_adaptive_eval": [_F, _U, _U, _P, _P],
    "tc_set_self_collision_substep_interval": [_P, _U],
    "tc_set_self_collision_ee_substep_interval": [_P, _U],
    "tc_get_self_collision_intervals": [_P, _P],
    "tc_set_bone_sdf_colliders": [_P, _U, _U, _U, _P, C.c_size_t, _P, _U],
    "tc_update_bone_transforms": [_P, _P, _P, _U, _P, C.c_int64],
    "tc_set_dynamic_bone_sdf_dirty_bones": [_P, _P, C.c_int64],
    "tc_clear_bone_sdf_colliders": [_P],
    "tc_setup_dynamic_bone_sdf": [_P, _U, _U, _U, _U, _P, _U, _P, _U, _P, _P, _U, _P, _P, _U, _P, _U, _U],
    "tc_set_dynamic_bone_sdf_enabled": [_P, _I],
    "tc_set_dynamic_bone_sdf_update_interval": [_P, _U],
    "tc_get_bone_sdf_atlas": [_P, _P, C.c_size_t, _P],
    "tc_get_bone_infos": [_P, _P, C.c_size_t, C.POINTER(_U)],
    "tc_bake_bone_sdf": [_P, _U, _P, _U, _U, _P, _P, _U, _F, _F, _F, _F, _F, _F, _I, _I, C.POINTER(_P)],
    "tc_bake_mesh_sdf": [_P, _U, _P, _U, _F, _F, _F, _F, _F, _I, _I, C.POINTER(_P)],
    "tc_bake_mesh_sdf_hierarchical": [_P, _U, _P, _U, _F, _F, _F, _F, _F, _I, _I, C.POINTER(_P)],
    "tc_bake_mesh_sdf_coarse": [_P, _U, _P, _U, _F, _F, _F, _F, _F, _I, C.POINTER(_P)],
    "tc_bake_get_nearest": [_P, _P, C.POINTER(_F)],
    "tc_bake_dims": [_P, _P],
    "tc_bake_get": [_P, _P, _P, _P, _P],
    "tc_bake_destroy": [_P],
    "tc_ws_param_count": [],
    "tc_ws_enable": [_P, _I, _U, _F],
    "tc_ws_set_kernel": [_P, _U],
    "tc_ws_record": [_P, _U, _U],
    "tc_ws_recorded": [_P, C.POINTER(_U)],
    "tc_ws_train": [_P, _U, _F, C.c_uint64, C.POINTER(_F), C.POINTER(_F)],
    "tc_ws_get_params": [_P, _P, C.c_size_t],
    "tc_ws_set_params": [_P, _P, C.c_size_t],
    "tc_ws_stats": [_P, _P],
    "tc_ws_set_relative_threshold": [_P, _F],
    "tc_get_predicted_residual": [_P, _P],
    "tc_ws_reset_stats": [_P],
    "tc_mlp_grad": [_U, _P, _P, _P, _P, _P, _P, C.POINTER(_F), _P, _P, _P, _I],
    "tc_mesh_build": [C.POINTER(_P), _P, _U, _P, _U, _P, _U, _P, _P, _P, _U, _F, _F, _F, _F, _F],
    "tc_mesh_build_sewn": [C.POINTER(_P), _P, _U, _P, _U, _P, _U, _P, _P, _P, _U, _F, _F, _F, _F, _F, _P, _U, _F, _F,
                           _I],
    "tc_mesh_sewing": [_P, C.POINTER(_U), C.POINTER(_U), _P, _P, _P, _P, _P],
    "tc_mesh_destroy": [_P],
    "tc_mesh_counts": [_P, _P, C.POINTER(_F)],
    "tc_mesh_constraints": [_P, _P, _P, _P, _P, _P, _P, _P, _P],
    "tc_mesh_topology_sizes": [_P, C.POINTER(_U), C.POINTER(_U), C.POINTER(_U)],
    "tc_mesh_topology": [_P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P],
}
_RESTYPES = {"tc_last_error": C.c_char_p, "tc_gpu_available": _I, "tc_ws_param_count": _U}

_lib = None


def load(path: str = LIB_PATH):
    """Load libtcloth.so and bind every declared symbol (raises if absent)."""
    global _lib
    if _lib is not None and path == LIB_PATH:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(
            f"libtcloth.so not found at {path}; build it with `python -c 'import __graft_entry__ as g; g.build()'`")
    L = C.CDLL(path)
    for name, args in SIGNATURES.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = _RESTYPES.get(name, _I)
    if path == LIB_PATH:
        _lib = L
    return L


class BarrierTimeout(RuntimeError):
    """A bounded grid-barrier wait of the persistent solver gave up."""


def check(status: int) -> None:
    """Map a tc_status to the reference's Python exceptions."""
    if status == TC_OK:
        return
    msg = load().tc_last_error().decode("utf-8", "replace")
    if status == TC_ERR_INVALID:
        raise ValueError(msg)
    if status == TC_ERR_TIMEOUT:
        raise BarrierTimeout(msg)
    if status == TC_ERR_NOMEM:
        raise MemoryError(msg)
    if status == TC_ERR_NONFINITE:
        raise FloatingPointError(msg)
    raise RuntimeError(msg)
