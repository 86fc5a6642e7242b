/*
 * tcloth.h -- C ABI of the B200 XPBD cloth substep (libtcloth.so).
 *
 * Drop-in replacement for the device half of Taremin/TareminCloth's
 * cloth_core: the entry points are what the crate's FFI (cloth_py's
 * ClothSimulator, crates/cloth_py/src/lib.rs:1549-3100, over
 * GpuClothSimulator, crates/cloth_core/src/simulation/mod.rs:57-355) binds.
 * Plain pointers and sizes only.  Every function returns a tc_status; on a
 * non-zero status tc_last_error() returns a thread-local message.
 * Input arrays are copied during the call; output arrays are caller-owned.
 * A tc_sim is used from one host thread at a time.
 */
#ifndef TCLOTH_H
#define TCLOTH_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  TC_OK = 0,
  TC_ERR_INVALID = 1, /* bad shape / index / argument (PyO3 ValueError)  */
  TC_ERR_CUDA = 2,    /* device unavailable or CUDA failure (RuntimeError) */
  TC_ERR_NOMEM = 3,   /* device or host allocation failed                 */
  TC_ERR_TIMEOUT = 4, /* a bounded device-side wait gave up               */
  TC_ERR_NONFINITE = 5 /* a checked read-back found NaN or Inf             */
} tc_status;

typedef struct tc_sim tc_sim;

/* Last error message of this thread ("" when none). */
const char *tc_last_error(void);
/* 1 when a CUDA device of compute capability 10.x is visible. */
int tc_gpu_available(void);
/* Device name of `device` into buf (nul-terminated). */
tc_status tc_device_name(int device, char *buf, size_t len);

/* ClothSimulator::new (crates/cloth_py/src/lib.rs:1556-1767) with
 * ClothMesh::from_raw_with_opts (crates/cloth_core/src/mesh.rs:407-1377).
 * faces, inv_masses, layer_ids, thicknesses may be NULL.  Stiffness in N/m
 * maps to compliance 1/k (k >= 5000 -> 0, k <= 0 -> 1e10).  Indices out of
 * range return TC_ERR_INVALID, like the reference's ValueError. */
tc_status tc_create(tc_sim **out, const float *positions, uint32_t n, const uint32_t *edges, uint32_t ne,
                    const uint32_t *faces, uint32_t nf, const float *inv_masses, const uint32_t *layer_ids,
                    const float *thicknesses, uint32_t layer_id, float thickness, float tension_stiffness,
                    float compression_stiffness, float shear_stiffness, float bending_stiffness, int device);
/* tc_create with the sewing arguments of ClothSimulator::new
 * (lib.rs:1557-1573, 1643-1665; mesh.rs:706-947): nsew sewing springs
 * (pairs of vertices; an index out of range returns TC_ERR_INVALID),
 * sewing_shrink_speed (m/s), sewing_stiffness (NaN: default 10000) and
 * enable_sewing_lock, which only fill the per-constraint fields as the
 * reference does (the solve reads tc_set_sewing_stiffness /
 * tc_set_enable_sewing_lock, default 10000 and on), sewing_lock_distance
 * (NaN: default 0.02 m).  The springs also add seam-gated bending across
 * sewn boundary edges and contract the self-collision topology. */
tc_status tc_create_sewn(tc_sim **out, const float *positions, uint32_t n, const uint32_t *edges, uint32_t ne,
                         const uint32_t *faces, uint32_t nf, const float *inv_masses, const uint32_t *layer_ids,
                         const float *thicknesses, uint32_t layer_id, float thickness, float tension_stiffness,
                         float compression_stiffness, float shear_stiffness, float bending_stiffness,
                         const uint32_t *sewing, uint32_t nsew, float sewing_shrink_speed, float sewing_stiffness,
                         int enable_sewing_lock, float sewing_lock_distance, int device);
tc_status tc_destroy(tc_sim *s);

/* Batched instances (new; the reference runs one cloth per simulator): one
 * simulator over `ninst` independent cloths.  Per instance k: vcount[k]
 * vertices, ecount[k] edges, fcount[k] faces (arrays concatenated, indices
 * local to the instance), compliance[4k..4k+3] = tension, compression,
 * shear, bending compliance, prim_count[k] primitive colliders of 10 floats
 * each in `prims` (type 0 sphere / 1 capsule / 2 plane, friction,
 * restitution, radius, a.xyz, b.xyz).  Vertex v of instance k is simulator
 * vertex offsets[k] + v (tc_batch_instance_offsets); pins use these indices.
 * Each instance evolves bit for bit as it would in its own simulator.
 * Self-collision is off. */
tc_status tc_batch_create(tc_sim **out, uint32_t ninst, const uint32_t *vcount, const uint32_t *ecount,
                          const uint32_t *fcount, const float *positions, const uint32_t *edges, const uint32_t *faces,
                          const float *inv_masses, float thickness, const float *compliance,
                          const uint32_t *prim_count, const float *prims, int device);
tc_status tc_batch_instance_offsets(tc_sim *s, uint32_t *offsets, uint32_t max_entries, uint32_t *n_instances);

/* GpuClothSimulator::step (crates/cloth_core/src/simulation/dispatch.rs:610-671):
 * one frame of `substeps` substeps (0 -> 20), synchronous.  The frame is
 * recorded once into a CUDA graph and replayed while parameters are unchanged. */
tc_status tc_step(tc_sim *s, float dt, uint32_t substeps, uint32_t *effective_substeps);
/* step_single_substep (dispatch.rs:674-688): one substep of dt_sub,
 * synchronous, without adaptive planning or displacement feedback. */
tc_status tc_step_single_substep(tc_sim *s, float dt_sub);
/* step_async (dispatch.rs:740-806): enqueue a frame on the simulator's stream
 * and return; fetch_positions (lib.rs:1834-1846) waits and copies. */
tc_status tc_step_async(tc_sim *s, float dt, uint32_t substeps);
tc_status tc_fetch_positions(tc_sim *s, float *out, size_t out_len, int *ok);
/* step_buffered / fetch_buffered_positions / get_buffered_frame_count /
 * clear_frame_buffer (dispatch.rs:1293-1408, lib.rs:1845-1881): a frame
 * whose positions go to the next of 8 device slots (the last slot once all
 * are full) with no wait, count = frames held; a fetch copies every held
 * frame (frames x n x 3 floats, as much as fits in out) in one transfer,
 * returns their count and empties the ring; tc_reset empties it too. */
tc_status tc_step_buffered(tc_sim *s, float dt, uint32_t substeps, uint32_t *count);
tc_status tc_fetch_buffered_positions(tc_sim *s, float *out, size_t out_len, uint32_t *count);
tc_status tc_get_buffered_frame_count(tc_sim *s, uint32_t *count);
tc_status tc_clear_frame_buffer(tc_sim *s);
/* get_positions (lib.rs:2110-2120): out holds n*3 floats. */
tc_status tc_get_positions(tc_sim *s, float *out, size_t out_len);
/* set_positions_and_velocities (dispatch.rs:953-988); vel may be NULL. */
tc_status tc_set_positions_and_velocities(tc_sim *s, const float *pos, const float *vel, uint32_t n);
/* reset (dispatch.rs:1411-1427) */
tc_status tc_reset(tc_sim *s);

/* parameters (simulation/mod.rs:1091-1106, :1429-1449, lib.rs:2751-2800) */
tc_status tc_set_gravity(tc_sim *s, float gx, float gy, float gz);
/* Edge colliders (edge_collision.wgsl; simulation/mod.rs:1007-1025,
 * lib.rs:2736-2749), off by default: after the final pins of each substep,
 * every cloth edge is tested against the edges of the mesh-collider
 * triangles near its midpoint (contact distance = thickness sum x scale +
 * offset, scale >= 1, offset >= 0) and pushed out through the pin channel
 * of the self-collision accumulator, applied before self-collision.  The
 * collider edges are extracted when the triangles are set. */
tc_status tc_set_enable_edge_collision(tc_sim *s, int enable);
tc_status tc_set_edge_margin_scale(tc_sim *s, float scale);
tc_status tc_set_edge_margin_offset(tc_sim *s, float offset);
tc_status tc_get_num_collider_edges(tc_sim *s, uint32_t *count);
/* Sewing (simulation/mod.rs:1211-1420, lib.rs:2798-2925).  Each substep
 * shrinks every spring's current rest length towards 0 at the shrink speed
 * (sewing_shrink.wgsl), projects the springs per colour after the distance
 * constraints of every iteration and once more before the velocity update
 * (sewing.wgsl; dispatch.rs:119-337).  Stiffness >= 5000 gives a hard
 * constraint, else compliance 1 / max(k, 1); with the lock on, a pair
 * closer than max(thickness sum, lock distance) latches to rest 0. */
tc_status tc_get_num_sewing_constraints(tc_sim *s, uint32_t *count);
tc_status tc_set_sewing_stiffness(tc_sim *s, float stiffness);
tc_status tc_set_sewing_shrink_speed(tc_sim *s, float speed);
tc_status tc_get_sewing_shrink_speed(tc_sim *s, float *speed);
tc_status tc_set_enable_sewing_lock(tc_sim *s, int enabled);
tc_status tc_set_sewing_lock_distance(tc_sim *s, float distance);
tc_status tc_get_sewing_lock_distance(tc_sim *s, float *distance);
/* current rest length of every spring, in the simulator's (colour) order;
 * a set with len != the spring count is ignored, as in the reference */
tc_status tc_get_sewing_current_rest_lengths(tc_sim *s, float *out, size_t len);
tc_status tc_set_sewing_current_rest_lengths(tc_sim *s, const float *values, size_t len);
/* Sewing priority: gravity is held at 0 until the share of springs closed
 * within merge_dist reaches threshold (or max_frames pass), then ramps back
 * with smoothstep over ramp_frames frames.  tc_update_sewing_priority takes
 * host positions (n x 3) and returns (ratio, gravity scale, latched);
 * tc_get_sewing_priority gives (gravity scale, ratio, held, latched). */
tc_status tc_set_sewing_priority_options(tc_sim *s, int enabled, float threshold, float merge_dist,
                                         uint32_t ramp_frames, uint32_t max_frames);
tc_status tc_set_sewing_priority_state(tc_sim *s, int latched, uint32_t frame, float ramp_t, float ratio);
tc_status tc_update_sewing_priority(tc_sim *s, const float *positions, uint32_t n, float out[3]);
tc_status tc_get_sewing_priority(tc_sim *s, float out[4]);
tc_status tc_set_damping(tc_sim *s, float damping);
tc_status tc_set_damping_all(tc_sim *s, float tension, float compression, float shear, float bending);
tc_status tc_set_solver_iterations(tc_sim *s, uint32_t iterations);
tc_status tc_set_stiffness_all(tc_sim *s, float tension, float compression, float shear, float bending);
/* Sets compliances directly (m/N); no stiffness mapping.  New entry point:
 * the reference reaches compliance only through stiffness. */
tc_status tc_set_compliance_all(tc_sim *s, float tension, float compression, float shear, float bending);
tc_status tc_set_edge_stiffness_multipliers(tc_sim *s, const uint32_t *edge_idx, const float *mult, uint32_t count);
/* reset_edge_stiffness_multipliers (simulation/mod.rs:1526-1532) */
tc_status tc_reset_edge_stiffness_multipliers(tc_sim *s);
/* set_edge_rest_length_scales / reset_edge_rest_lengths (simulation/mod.rs:1450-1491):
 * the distance constraint of input edge idx[i] gets rest = initial rest x
 * max(scales[i], 0.01); edges without one are skipped. */
tc_status tc_set_edge_rest_length_scales(tc_sim *s, const uint32_t *idx, const float *scales, uint32_t count);
tc_status tc_reset_edge_rest_lengths(tc_sim *s);
/* get_edge_rest_length, get_edge_initial_rest_length, get_edge_tension_compliance
 * (simulation/mod.rs:1535-1568): out = (rest, initial rest, tension compliance)
 * of input edge edge_idx, zeros when it has no distance constraint. */
tc_status tc_get_edge_constraint(tc_sim *s, uint32_t edge_idx, float out[3]);
tc_status tc_set_enable_self_collision(tc_sim *s, int enable);
/* set_self_collision_options (simulation/mod.rs:920-950) */
tc_status tc_set_self_collision_options(tc_sim *s, float relief_factor, float max_displacement_ratio,
                                        int exclude_neighbors, int enable_normal_untangling, uint32_t max_iterations);
/* Contact-pair cache ("Active Pair Caching", self-collision algorithm 1;
 * simulation/mod.rs:36-41, :582-600, :703-715, :799-893; dispatch.rs:1111-1132,
 * :1249-1290, :1540-1670; lib.rs:2029-2105), off by default.  At the first
 * substep of a frame one pass over the vertex hash keeps, per vertex, the
 * quota nearest vertex-triangle and edge-edge candidates within the
 * thickness plus the safety margin plus (margin_mode 1) a velocity horizon
 * min(|v| dt_frame horizon_scale, max_horizon); every substep then solves
 * only those pairs.  quota = clamp(max_pairs / vertices, 1, 8).  With the
 * final fallback on (default) the last substep of a frame runs the direct
 * pass on a fresh hash.  set_self_collision_algorithm: 0 direct, 1 pair
 * cache; 2 (virtual particles) returns TC_ERR_INVALID. */
tc_status tc_set_enable_pair_cache(tc_sim *s, int enable);
tc_status tc_get_enable_pair_cache(tc_sim *s, int *enabled);
tc_status tc_set_self_collision_algorithm(tc_sim *s, uint32_t algo);
tc_status tc_get_self_collision_algorithm(tc_sim *s, uint32_t *algo);
/* max pairs clamped to [64, 262144], margin_mode 0 fixed / else velocity
 * horizon, safety_margin to [0, 0.05], horizon_scale to [0, 4], max_horizon
 * to [0, 0.1] (set_pair_cache_options, simulation/mod.rs:826-848) */
tc_status tc_set_pair_cache_options(tc_sim *s, uint32_t max_vt_pairs, uint32_t max_ee_pairs, uint32_t margin_mode,
                                    float safety_margin, float horizon_scale, float max_horizon);
tc_status tc_set_enable_pair_cache_final_fallback(tc_sim *s, int enable);
tc_status tc_get_enable_pair_cache_final_fallback(tc_sim *s, int *enabled);
/* out = (V-T candidates accepted, E-E candidates accepted, max_vt_pairs,
 * max_ee_pairs) of the latest broad phase (get_pair_cache_stats) */
tc_status tc_get_pair_cache_stats(tc_sim *s, uint32_t out[4]);
/* get_active_pairs (dispatch.rs:1249-1290): counts = (V-T accepted, E-E
 * accepted, stored V-T pairs, stored E-E pairs); the stored pairs, four
 * vertex ids each in slot order, go to vt_pairs / ee_pairs up to the given
 * capacities in pairs (NULL to query the counts only). */
tc_status tc_get_active_pairs(tc_sim *s, uint32_t counts[4], uint32_t *vt_pairs, size_t vt_capacity,
                              uint32_t *ee_pairs, size_t ee_capacity);
tc_status tc_set_coupled_collider(tc_sim *s, int enable);
tc_status tc_set_auto_coupled_on_low_substeps(tc_sim *s, int enable);
tc_status tc_set_collider_options(tc_sim *s, int enable_cluster_culling, int enable_single_sided_recovery,
                                  float sweep_margin);

/* colliders (simulation/mod.rs:1571-1628, lib.rs:2157-2240) */
tc_status tc_add_sphere_collider(tc_sim *s, const float center[3], float radius, float friction, float restitution);
tc_status tc_add_capsule_collider(tc_sim *s, const float a[3], const float b[3], float radius, float friction,
                                  float restitution);
tc_status tc_add_plane_collider(tc_sim *s, const float point[3], const float normal[3], float friction,
                                float restitution);
/* triangles: T x 3 x 3 floats; attributes (nullable): T x 4 (friction,
 * thickness, restitution, flags).  The floats are copied into pinned host
 * memory before the call returns; the Morton order and the culling spheres
 * are computed on the device ahead of the next step. */
tc_status tc_set_mesh_collider_triangles(tc_sim *s, const float *triangles, uint32_t T, float friction,
                                         float thickness, float restitution, int single_sided, const float *attributes);
tc_status tc_clear_colliders(tc_sim *s);
/* Self-collision every `interval` substeps and on the last (>= 1), and the
 * edge-edge pass every `interval` substeps and on the last (0 = never,
 * 1 = always): dispatch.rs:105-114, mod.rs:1071-1088.  Defaults 1 / 1.
 * out = (self-collision interval, E-E interval). */
tc_status tc_set_self_collision_substep_interval(tc_sim *s, uint32_t interval);
tc_status tc_set_self_collision_ee_substep_interval(tc_sim *s, uint32_t interval);
tc_status tc_get_self_collision_intervals(tc_sim *s, uint32_t out[2]);
/* Adaptive substeps and iterations (set_adaptive_substep_options etc.,
 * simulation/mod.rs:723-790; decisions dispatch.rs:477-607).  Off by default.
 * When on, tc_step's substep count is chosen from the previous frames'
 * maximum vertex displacement (CFL), the free-fall floor and the P95 tensile
 * strain of a 2048-constraint sample, with hysteresis; iterations are
 * compensated toward a propagation budget.  The feedback is reduced on the
 * GPU after each frame (no position readback).
 * out = effective substeps, effective iterations, last P95 strain, last max
 * displacement, CFL characteristic length, mesh diameter in hops. */
tc_status tc_set_adaptive_substep_options(tc_sim *s, int enabled, uint32_t min_substeps, uint32_t max_substeps);
tc_status tc_set_auto_compensate_iterations(tc_sim *s, int enabled);
tc_status tc_set_strain_adaptive_options(tc_sim *s, int enabled, float tolerance);
tc_status tc_note_external_displacement(tc_sim *s, float disp);
tc_status tc_get_adaptive_state(tc_sim *s, float out[6]);
/* The decision rules alone (no simulator), for tests; in[18] is documented
 * beside the definition order: enabled, min, max, base substeps, previous
 * effective substeps, characteristic length, thickness, gx, gy, gz, max
 * displacement, external displacement, strain adaptive, tolerance, last
 * strain, auto compensate, solver iterations, diameter hops.  out = substeps,
 * iterations for iter_substeps substeps (0 = for the substeps chosen). */
tc_status tc_adaptive_eval(float dt, uint32_t requested, uint32_t iter_substeps, const float in[18], uint32_t out[2]);

/* Bone SDF colliders (lib.rs:2245-2600, simulation/mod.rs:1630-2464).  The
 * atlas is width x height x depth texels of packed half2 (distance in the low
 * 16 bits, alpha in the high 16), z-major then y then x: the reference's
 * Rg16Float texture bytes read as uint32.  bone_infos: n_bones rows of 20
 * floats (aabb_min 4, aabb_max 4, uvw_scale 4, uvw_offset 4, friction,
 * thickness, restitution, weight threshold).  Matrices: 16 floats per bone in
 * the reference's GpuBoneTransform order (column-major: row j, column k at
 * [k*4 + j]).  Sampling is trilinear with clamp-to-edge in fp32. */
tc_status tc_set_bone_sdf_colliders(tc_sim *s, uint32_t width, uint32_t height, uint32_t depth,
                                    const uint32_t *texels, size_t n_texels, const float *bone_infos,
                                    uint32_t n_bones);
/* dirty: bones to rebake at the next dynamic update; n_dirty < 0 = all
 * (None), 0 = none (the reference skips the rebake) */
tc_status tc_update_bone_transforms(tc_sim *s, const float *world, const float *inv_world, uint32_t n_bones,
                                    const uint32_t *dirty, int64_t n_dirty);
tc_status tc_set_dynamic_bone_sdf_dirty_bones(tc_sim *s, const uint32_t *dirty, int64_t n_dirty);
tc_status tc_clear_bone_sdf_colliders(tc_sim *s);
/* Dynamic bone SDF: before a frame (every update_interval frames) skin the
 * body (4 bone indices / weights per vertex, rest_cols >= 3 floats per rest
 * vertex), move each source triangle (i0, i1, i2, bone; weights w0, w1, w2)
 * into its bone's frame and rebake the bones' res^3 tiles on the GPU.
 * bind_inv: row-major, as lib.rs:2550-2562.  Indices must be in range
 * (TC_ERR_INVALID), where the reference reads out of its buffers. */
tc_status tc_setup_dynamic_bone_sdf(tc_sim *s, uint32_t width, uint32_t height, uint32_t depth, uint32_t res,
                                    const float *bone_infos, uint32_t n_bones, const float *rest_verts,
                                    uint32_t rest_cols, const uint32_t *bone_indices, const float *bone_weights,
                                    uint32_t n_verts, const uint32_t *tri_sources, const float *tri_weights,
                                    uint32_t n_tris, const float *bind_inv, uint32_t n_bind,
                                    uint32_t update_interval);
tc_status tc_set_dynamic_bone_sdf_enabled(tc_sim *s, int enable);
tc_status tc_set_dynamic_bone_sdf_update_interval(tc_sim *s, uint32_t interval);
/* Read back the atlas (dims = width, height, depth; out may be NULL) and the
 * bone infos including the world bounding spheres in their .w slots. */
tc_status tc_get_bone_sdf_atlas(tc_sim *s, uint32_t *out, size_t len, uint32_t dims[3]);
tc_status tc_get_bone_infos(tc_sim *s, float *out, size_t len, uint32_t *n_bones);

/* bake_bone_sdf_gpu (lib.rs:1186-1350, sdf_baker.rs:465-940): bone-local SDF
 * atlas of a skinned mesh.  bone_weights: n_bones rows of n_verts;
 * bind_matrices: n_bones row-major 4x4 (mesh -> bone local).  Fails with
 * TC_ERR_CUDA (RuntimeError) when no bone has a weight above the threshold. */
typedef struct tc_bake tc_bake;
tc_status tc_bake_bone_sdf(const float *mesh_verts, uint32_t n_verts, const int32_t *mesh_tris, uint32_t n_tris,
                           uint32_t n_bones, const float *bone_weights, const float *bind_matrices,
                           uint32_t resolution, float margin, float weight_threshold, float blend_k, float friction,
                           float thickness, float restitution, int close_open_boundaries, int device, tc_bake **out);
/* out = width, height, depth, number of active bones */
/* bake_mesh_sdf_gpu (lib.rs:1349-1416; sdf_baker.rs:939-1060, :1114-1326):
 * the signed distance field of one mesh (open boundary loops capped first
 * when close_open_boundaries) over its bounding box padded by
 * max(size x margin, 0.04) + thickness + 0.02 per axis, at voxel_size
 * (8..2048 voxels per axis): per voxel the distance to the nearest triangle
 * (the first of equal distances), negative behind its normal, packed as
 * fp16 (distance, 1).  tc_bake_get gives the texels and infos[20] = local
 * min, 0, local max, width, uvw scale (4), uvw offset (4), friction,
 * thickness, restitution, 0; no active bones.  No vertices:
 * TC_ERR_CUDA, like the reference's error. */
tc_status tc_bake_mesh_sdf(const float *mesh_verts, uint32_t nv, const int32_t *mesh_tris, uint32_t nt,
                           float voxel_size, float margin, float friction, float thickness, float restitution,
                           int close_open_boundaries, int device, tc_bake **out);
/* bake_mesh_sdf_hierarchical_gpu (lib.rs:1418-1488; sdf_baker.rs:1603-1900,
 * bake_mesh_sdf_hier_*.wgsl): the same field in two passes.  The coarse
 * pass keeps, per cell of max(voxel x 4, 0.001), the 8 nearest triangles.
 * A fine voxel whose parent cell is at least band + half a cell diagonal
 * from the surface copies the parent's value (band = 4 fine voxels); the
 * others take the nearest of the candidates of the 5 x 5 x 5 cells around
 * the parent, rescanning every triangle when the best two are within
 * 0.2 mm with opposite signs.  A band wider than two coarse cells, or no
 * vertices: TC_ERR_CUDA, like the reference's errors. */
tc_status tc_bake_mesh_sdf_hierarchical(const float *mesh_verts, uint32_t nv, const int32_t *mesh_tris, uint32_t nt,
                                        float voxel_size, float margin, float friction, float thickness,
                                        float restitution, int close_open_boundaries, int device, tc_bake **out);
/* bake_mesh_sdf_coarse_gpu (lib.rs:1490-1540; sdf_baker.rs:1328-1600), the
 * coarse pass alone (open loops always capped): texels = packed distance per
 * coarse voxel; tc_bake_get_nearest gives the 8 nearest triangle indices per
 * voxel (voxel * 8 + k, nearest first) and the coarse voxel size. */
tc_status tc_bake_mesh_sdf_coarse(const float *mesh_verts, uint32_t nv, const int32_t *mesh_tris, uint32_t nt,
                                  float voxel_size, float margin, float friction, float thickness, float restitution,
                                  int device, tc_bake **out);
tc_status tc_bake_get_nearest(tc_bake *b, uint32_t *nearest, float *coarse_voxel);
/* compute_combined_inv_masses / compute_areal_inv_masses (mesh.rs:237-312,
 * lib.rs:553-640), host only: a third of each valid triangle's area x
 * areal_density to its corners and half of each strand edge's length x
 * linear_density to its ends; out[i] = 0 for pin >= 1, else
 * (1 - pin) / max(mass, 1e-9) with pin clamped to [0, 1] (entries past npin:
 * 0).  faces, strand_edges and pin_weights may be NULL. */
tc_status tc_compute_combined_inv_masses(const float *positions, uint32_t n, const uint32_t *faces, uint32_t nf,
                                         const uint32_t *strand_edges, uint32_t ns, const float *pin_weights,
                                         uint32_t npin, float areal_density, float linear_density, float *out);
/* color_edge_pairs (coloring.rs:180-233, lib.rs:642-652), host only:
 * Welsh-Powell colours of vertex pairs, order (-degree, index). */
tc_status tc_color_edge_pairs(uint32_t num_vertices, const uint32_t *pairs, uint32_t np, uint32_t *colors);
/* Device health (crates/cloth_core/src/context.rs:101-140, test :499): a
 * per-device lost flag and context epoch.  tc_mark_device_lost marks the
 * device lost (anomaly handling, tests; host-side only).  The next
 * simulator creation on that device re-initialises it (synchronise, epoch
 * + 1, flag cleared; TC_ERR_CUDA when the device does not answer, which
 * needs a fresh process).  Simulators created in an older epoch refuse every
 * call with TC_ERR_CUDA; destroying them still works. */
tc_status tc_mark_device_lost(int device);
tc_status tc_device_status(int device, int *lost, uint64_t *epoch);
/* Read-back sentinel (the NaN / Inf invariant of docs/architecture.md
 * section 5): when on, tc_get_positions, tc_fetch_positions and
 * tc_fetch_buffered_positions return TC_ERR_NONFINITE if the copied
 * positions hold NaN or Inf (the copy is still written).  Off by default, as
 * in the reference, whose read-backs return whatever the GPU holds. */
tc_status tc_set_nonfinite_check(tc_sim *s, int enable);
/* Autotuned settings (new).  tc_set_launch_block: threads per block of the
 * one-launch-per-colour constraint kernels (64 .. 1024, powers of two);
 * results do not change.  tc_set_hash_cell_size: the spatial-hash cell of
 * the self-collision passes; cell <= 0 restores the reference formula's
 * value (pipelines.rs:898-912), which is the parity setting.  Another cell
 * changes which neighbours are seen, so it is a physics setting: the
 * autotuner keeps one only when positions and residual stay within stated
 * bounds of the reference cell's. */
tc_status tc_set_launch_block(tc_sim *s, uint32_t threads);
tc_status tc_set_hash_cell_size(tc_sim *s, float cell);
/* Kernel shape of the direct pass's edge-edge search (new; results and pair
 * lists do not change): 0 (default) = one warp per edge over the 27
 * neighbour cells, the counted pairs listed and their contact work done one
 * lane per pair by a second kernel; 1 = one lane per edge, a warp taking 32
 * edges of the hash-sorted order and building each distinct cell's
 * candidate list once in shared memory; 2 = as 0 with the contact work done
 * by the edge's own warp. */
tc_status tc_set_self_collision_variant(tc_sim *s, uint32_t ee_variant);
/* Capacity, in (edge, edge) pairs, of the list through which variant 0
 * hands its counted pairs to the contact kernel (new; 0 = the default,
 * 24 per edge + 1024).  The list is split evenly among 256 segments; pairs
 * past their segment's share are worked by the search kernel itself, so
 * results do not depend on it. */
tc_status tc_set_ee_pair_list_capacity(tc_sim *s, uint64_t entries);
/* Narrow-phase pair lists of the direct self-collision pass, for parity
 * (no counterpart in the reference's API; the passes are
 * shaders/self_collision.wgsl:317-681 and
 * shaders/self_collision_ee_direct.wgsl:266-776).  With recording on, every
 * self-collision pass clears and refills two lists: the (vertex, triangle)
 * pairs that pass the cheap tests of the vertex-triangle search (triangle
 * ownership, swept bounds, two-hop exclusion) and reach the contact math,
 * and the (edge, edge) pairs counted within max_search.  The pair-cache
 * pass records none.  tc_get_pair_lists returns the latest pass's lists,
 * canonical and sorted: V-T rows (vertex, a, b, c) with a < b < c the
 * triangle's vertices, E-E rows (e0, e1) with e0 < e1; counts[0..1] are the
 * list lengths.  A list longer than its recording capacity is
 * TC_ERR_INVALID, as is an output array smaller than the list.  Recording
 * adds one atomic per recorded pair. */
tc_status tc_set_pair_recording(tc_sim *s, int enable, uint32_t max_vt_pairs, uint32_t max_ee_pairs);
tc_status tc_get_pair_lists(tc_sim *s, uint32_t *vt, uint32_t vt_capacity, uint32_t *ee, uint32_t ee_capacity,
                            uint32_t counts[2]);
/* The settings record of the reference (SimConfig,
 * crates/cloth_core/src/config.rs:40-140, written by
 * simulation/config_impl.rs:16-78; cloth_py lib.rs:3029-3042).
 * tc_get_config_json writes the compact JSON text (fields in the record's
 * order, floats as the shortest f32 digits) into buf when capacity > 0,
 * truncated to capacity - 1 bytes and NUL-terminated, and its full length in
 * *length.  tc_get_config_hash is the 64-bit FNV-1a of that text
 * (config.rs:205-214, lib.rs:3044-3047).  Applying a record is the host's
 * job: parse it and call the setters in config_impl.rs:80-155's order. */
tc_status tc_get_config_json(tc_sim *s, char *buf, size_t capacity, size_t *length);
tc_status tc_get_config_hash(tc_sim *s, uint64_t *hash);
/* set_workgroup_size (mod.rs:2987-2994): 64 or else 32, stored for the
 * record; the CUDA path's launch shapes do not depend on it. */
tc_status tc_set_workgroup_size(tc_sim *s, uint32_t wg_size);
/* set_areal_density (mod.rs:1241-1245): finite values clamped to [0, 100]. */
tc_status tc_set_areal_density(tc_sim *s, float density);
/* set_coupled_self_collision_options (mod.rs:1055-1058): mode 0 only (the
 * others are TC_ERR_INVALID); the relaxation count is stored. */
tc_status tc_set_coupled_self_collision_options(tc_sim *s, uint32_t mode, uint32_t relaxation_iters);
/* find_triangle_intersections (crates/cloth_core/src/geometry.rs:506-633,
 * crates/cloth_py/src/lib.rs:856-879), host only: face pairs (f0 < f1,
 * ascending) whose triangles share a point; with ignore_adjacent, pairs that
 * share a vertex (or a vertex cluster joined by the optional sewing springs)
 * are skipped; faces with repeated or out-of-range indices are skipped.
 * cell_size <= 0 picks the broad-phase cell.  Writes min(count, capacity)
 * pairs (2 words each) and the total in *count. */
tc_status tc_find_triangle_intersections(const float *positions, uint32_t n, const uint32_t *faces, uint32_t nf,
                                         int ignore_adjacent, float cell_size, const uint32_t *sewing, uint32_t nsew,
                                         uint32_t *pairs, uint32_t capacity, uint32_t *count);
tc_status tc_bake_dims(tc_bake *b, uint32_t out[4]);
/* texels (w*h*d), infos (n_active x 20), active (source bone index per
 * active bone), bind (n_active x 16); any may be NULL */
tc_status tc_bake_get(tc_bake *b, uint32_t *texels, float *infos, uint32_t *active, float *bind);
tc_status tc_bake_destroy(tc_bake *b);

/* pins (simulation/mod.rs:2768-2860) */
tc_status tc_set_pin(tc_sim *s, uint32_t vertex, const float target[3], float weight);
tc_status tc_set_pins_batch(tc_sim *s, const uint32_t *idx, const float *targets, const float *weights, uint32_t count);
tc_status tc_release_pin(tc_sim *s, uint32_t vertex);
tc_status tc_clear_pins(tc_sim *s);
tc_status tc_set_vertex_inv_masses(tc_sim *s, const uint32_t *idx, const float *inv_masses, uint32_t count);
tc_status tc_get_vertex_inv_masses(tc_sim *s, float *out, uint32_t n);

/* counts (lib.rs:2928-2950): out[8] = n, distance, bending, edges,
 * distance colours, bending colours, hash table size, multi-layer flag */
/* get_num_virtual_vertices (lib.rs:2045-2048): the virtual-particle count of
 * the mesh (pipelines.rs:170-185, capped at 150,000); the particles
 * themselves (self-collision algorithm 2) are not built. */
tc_status tc_get_num_virtual_vertices(tc_sim *s, uint32_t *count);
tc_status tc_get_counts(tc_sim *s, uint32_t out[8]);
tc_status tc_get_cell_size(tc_sim *s, float *cell);

/* ---- parity introspection (new; no reference counterpart) ---- */
/* x, p, v: n*3 each (any may be NULL) */
tc_status tc_get_state(tc_sim *s, float *x, float *p, float *v);
/* colour-sorted constraints: v01 (nd*2), par (nd*4: rest, tc, cc, type),
 * off/cnt per colour */
tc_status tc_get_distance_constraints(tc_sim *s, uint32_t *v01, float *par, uint32_t *off, uint32_t *cnt);
tc_status tc_get_bending_constraints(tc_sim *s, uint32_t *v0123, float *par, uint32_t *off, uint32_t *cnt);
/* Build the spatial hash from the current predicted positions on the device
 * (which = 0 vertices, 1 edges) and copy cell_starts (table+1) and sorted. */
tc_status tc_get_hash_state(tc_sim *s, int which, uint32_t *cell_starts, uint32_t *sorted);
/* Sorted unique edges (ne*2) and open-boundary bits ((ne+31)/32). */
tc_status tc_get_edges(tc_sim *s, uint32_t *edges, uint32_t *bits);
/* Per-colour residual |C(x) + alpha~ lambda| after the last iteration of the
 * last substep of the latest frame, when tracking is on.  rms/max arrays are
 * sized by the colour counts; totals[4] = dist rms, dist max, bend rms, bend max. */
tc_status tc_set_residual_tracking(tc_sim *s, int enable);
/* With residual tracking: RMS residual |C| over all distance and bending
 * constraints at the predicted positions of the latest frame's last substep
 * (before any iteration, lambda = 0). */
tc_status tc_get_predicted_residual(tc_sim *s, float *rms);
tc_status tc_get_residuals(tc_sim *s, float *dist_rms, float *dist_max, float *bend_rms, float *bend_max,
                           float totals[4]);
/* ---- host-only topology build (no device needed) ----
 * Runs the same constraint / colouring / topology builder that tc_create
 * uses, so the host half of the path can be checked without a GPU. */
typedef struct tc_mesh tc_mesh;
tc_status tc_mesh_build(tc_mesh **out, const float *positions, uint32_t n, const uint32_t *edges, uint32_t ne,
                        const uint32_t *faces, uint32_t nf, const float *inv_masses, const uint32_t *layer_ids,
                        const float *thicknesses, uint32_t layer_id, float thickness, float tension_stiffness,
                        float compression_stiffness, float shear_stiffness, float bending_stiffness);
/* tc_mesh_build with sewing springs (arguments as tc_create_sewn) */
tc_status tc_mesh_build_sewn(tc_mesh **out, const float *positions, uint32_t n, const uint32_t *edges, uint32_t ne,
                             const uint32_t *faces, uint32_t nf, const float *inv_masses, const uint32_t *layer_ids,
                             const float *thicknesses, uint32_t layer_id, float thickness, float tension_stiffness,
                             float compression_stiffness, float shear_stiffness, float bending_stiffness,
                             const uint32_t *sewing, uint32_t nsew, float sewing_shrink_speed, float sewing_stiffness,
                             int enable_sewing_lock);
tc_status tc_mesh_destroy(tc_mesh *m);
/* Sewing constraints (colour-sorted, coloring.rs:236-300): count, colours,
 * vertex pairs, par[5] = current rest, target rest, shrink speed,
 * compliance, lock flag; colour offsets / counts; rep[n] = sewing group of
 * each vertex (its smallest member).  Any output may be NULL. */
tc_status tc_mesh_sewing(tc_mesh *m, uint32_t *nsew, uint32_t *ncolors, uint32_t *v01, float *par, uint32_t *off,
                         uint32_t *cnt, uint32_t *rep);
/* out[10] = n, distance, bending, edges, distance colours, bending colours,
 * table size, multi-layer flag, virtual-particle count, adjacency length;
 * cell[1] = hash cell size */
tc_status tc_mesh_counts(tc_mesh *m, uint32_t out[10], float *cell);
tc_status tc_mesh_constraints(tc_mesh *m, uint32_t *dist_v01, float *dist_par, uint32_t *dist_off, uint32_t *dist_cnt,
                              uint32_t *bend_v0123, float *bend_par, uint32_t *bend_off, uint32_t *bend_cnt);
/* th_n = length of the two-hop CSR, star_n = number of star pairs */
tc_status tc_mesh_topology_sizes(tc_mesh *m, uint32_t *adj_n, uint32_t *th_n, uint32_t *star_n);
tc_status tc_mesh_topology(tc_mesh *m, uint32_t *adj_off, uint32_t *adj_idx, uint32_t *th_off, uint32_t *th_idx,
                           float *th_rest, float *local_len, uint32_t *star_off, uint32_t *star_idx, uint32_t *island,
                           uint32_t *layer, uint32_t *edges, uint32_t *edge_bits);

/* set_profiling_enabled / take_profile (simulation/mod.rs:1038-1053): while
 * enabled, frames run without the CUDA graph and every pass is bracketed by
 * CUDA events.  take_profile returns, per pass, its name (names joined by
 * newlines), total milliseconds and number of timed launch groups, then
 * clears the record. */
tc_status tc_set_profiling_enabled(tc_sim *s, int enable);
tc_status tc_take_profile(tc_sim *s, char *names, size_t names_len, float *ms, uint32_t *launches,
                          uint32_t max_entries, uint32_t *n_entries);
/* Persistent solver (default on when the device supports cooperative
 * launch): the constraint phase of a substep (of a whole frame when
 * self-collision is off) is one cooperative launch whose colours are
 * separated by bounded grid barriers; off = one launch per colour.  Both give
 * the same bits.  A barrier that waits past its poll limit makes tc_step
 * return TC_ERR_TIMEOUT.  New; the reference dispatches one pass per colour
 * (dispatch.rs:1449-1455). */
tc_status tc_set_persistent_solver(tc_sim *s, int enable);
/* Launch shape: persistent = 0 one launch per colour; 1 the persistent
 * solver with blocks_per_sm (1..limit); 2 the cluster solver for batched
 * instances without self-collision (each thread-block cluster of 8 CTAs runs
 * a bin of whole instances through the frame, colour steps separated by the
 * cluster barrier); 3 the staged cluster solver (the same bins with the
 * bin's vertex records held in the cluster's shared memory for the whole
 * frame, split into one slice per CTA and reached across CTAs through
 * distributed shared memory; needs every instance within 8 x the per-CTA
 * capacity).  TC_ERR_INVALID when a mode is not applicable.  Used by the
 * autotuner.  Results do not change. */
tc_status tc_set_launch_config(tc_sim *s, int persistent, uint32_t blocks_per_sm);
tc_status tc_get_launch_limits(tc_sim *s, uint32_t *max_blocks_per_sm, uint32_t *num_sms);
/* Diagnostics for the failure path: runs one barrier that can never be
 * released, with the given poll limit (1..4194304), and returns
 * TC_ERR_TIMEOUT when every wait ended by the limit.  Touches no state. */
tc_status tc_check_barrier_timeout(tc_sim *s, uint32_t spin_limit);
/* Diagnostics (new): out = edge pairs the latest self-collision pass handed to
 * the deferred edge-edge CCD kernel, and the queue capacity (pairs beyond it
 * run inline in the warp pass). */
tc_status tc_get_ccd_queue(tc_sim *s, uint32_t out[2]);
/* Kernel launches in the recorded frame (kernel nodes of its CUDA graph). */
tc_status tc_frame_kernel_count(tc_sim *s, uint32_t *count);
/* Device time of the latest frame in milliseconds (CUDA events). */
tc_status tc_last_frame_ms(tc_sim *s, float *ms);

/* Learned warm start; no counterpart in the reference.  A graph MLP (features
 * -> 64, two message-passing rounds [self, neighbour mean] 128 -> 64, SiLU,
 * head 64 -> 3; bf16 weights on the tensor cores, fp32 accumulation) predicts
 * each vertex's correction p_final - p_predicted of the coming substep, in
 * units of the vertex's local edge length.  While enabled, a substep moves p
 * by that prediction, runs (iterations - k_replaced) plain XPBD iterations,
 * computes the RMS constraint residual |C + alpha~ lambda| over all distance
 * and bending constraints and, when it is above res_thresh (the plain
 * solver's residual; +inf never falls back),
 * runs the k_replaced remaining iterations.  Needs cooperative launch. */
uint32_t tc_ws_param_count(void);
tc_status tc_ws_enable(tc_sim *s, int enable, uint32_t k_replaced, float res_thresh);
/* Tensor-core path of the network's message-passing layers (inference, and
 * training forward and backward): 0 (default) = tcgen05.mma with the
 * accumulators in tensor memory, 1 = warp-level mma.sync.  Both round at the
 * same points; the fp32 sums may differ in order. */
tc_status tc_ws_set_kernel(tc_sim *s, uint32_t kind);
/* Record training snapshots during the following plain frames: every
 * `every`-th substep until `capacity` snapshots are held; a new recording
 * replaces the old snapshots, capacity 0 stops and keeps them.  Frames run
 * without the CUDA graph while recording; results are unchanged. */
tc_status tc_ws_record(tc_sim *s, uint32_t capacity, uint32_t every);
tc_status tc_ws_recorded(tc_sim *s, uint32_t *count);
/* Adam over the recorded snapshots (epochs x snapshots steps, seeded
 * shuffle); mean MSE loss (of the normalised target) of the first and last
 * epoch.  The first training of a network that was not loaded with
 * tc_ws_set_params first fits its normalizer on the recorded snapshots. */
tc_status tc_ws_train(tc_sim *s, uint32_t epochs, float lr, uint64_t seed, float *loss_first, float *loss_last);
/* fp32 parameter blob (tc_ws_param_count() floats): W0[16][64] b0[64]
 * W1[128][64] b1[64] W2[128][64] b2[64] W3[64][3] b3[3], weights [in][out],
 * then the normalizer FS[16] YS[1]: features enter as bf16(feature * FS),
 * vertices move by Y * YS * L (YS <= 0 reads as 1).  Setting a blob keeps
 * its normalizer for later training. */
tc_status tc_ws_get_params(tc_sim *s, float *out, size_t len);
tc_status tc_ws_set_params(tc_sim *s, const float *params, size_t len);
/* out = warm-started substeps, substeps that fell back, max residual of the
 * latest substep's check, threshold */
tc_status tc_ws_stats(tc_sim *s, double out[4]);
/* Relative threshold (ratio > 0; 0 returns to res_thresh): a warm-started
 * substep falls back when its residual is above ratio x the RMS residual
 * |C| of its predicted positions (before the network moves them, lambda =
 * 0; at least 1e-6 of the mean edge length), so the threshold follows the
 * scene.  The ratio is the plain solver's
 * final / predicted residual (tc_get_predicted_residual), e.g. a percentile
 * over plain substeps.  tc_ws_stats then reports the latest threshold. */
tc_status tc_ws_set_relative_threshold(tc_sim *s, float ratio);
tc_status tc_ws_reset_stats(tc_sim *s);
/* Loss, parameter gradients and outputs of the warm-start network on one
 * graph, through the same kernels as training (for gradient checks).
 * feat n x 16 (rounded to bf16), adjacency CSR, target n x 3, mask n,
 * loss = sum_i mask_i |y_i - target_i|^2 / (3 n).  y_infer (optional, n x 3)
 * receives the outputs of the inference kernels (head fused into the last
 * layer) that the warm-started substep runs. */
tc_status tc_mlp_grad(uint32_t n, const float *feat, const uint32_t *adj_off, const uint32_t *adj_idx,
                      const float *target, const float *mask, const float *params, float *loss, float *grads,
                      float *y, float *y_infer, int device);

/* Spatial-hash build that allocates nothing; no counterpart in the reference.
 * For callers that cannot allocate device memory: applications whose device
 * buffers all come from their own allocator, threads that must not call
 * cudaMalloc / cudaFree (they synchronise the device), memory-capped hosts.
 * Builds cell_starts (table_size + 1 entries, exclusive prefix sums of the
 * bucket counts, last = n) and sorted (n vertex indices grouped by bucket,
 * ascending index within each bucket) from `positions` (device, n x 4
 * floats: x, y, z, unused; 16-byte aligned), on `stream` (cudaStream_t,
 * NULL = legacy default stream).  Given the simulator's predicted positions
 * (tc_get_state's p), cell size and table size, the output equals
 * tc_get_hash_state(which = 0).  All buffers are the caller's device memory;
 * scratch is a static array in the library of fixed size, so n <= 262144
 * and 1024 <= table_size <= 65536, and cell_size must be positive, else
 * TC_ERR_INVALID.  n = 0 gives all-zero cell_starts.  The first call on a
 * device looks up that array's device address, so make it before any stream
 * capture; after a reset of the device's primary context the library needs
 * a fresh process.  All calls on a device share the array: calls that
 * overlap on the GPU (different streams, or threads) race. */
tc_status tc_hash_build_static(const float *positions, uint32_t n, float cell_size, uint32_t table_size,
                               uint32_t *cell_starts, uint32_t *sorted, void *stream);

#ifdef __cplusplus
}
#endif
#endif
