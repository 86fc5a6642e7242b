/*
 * tcloth_oracle.h -- CPU oracle for the XPBD cloth substep.
 *
 * TEST INFRASTRUCTURE ONLY.  This library restates, as plain sequential C,
 * the algorithm of Taremin/TareminCloth's cloth_core substep so that the
 * CUDA product can be checked against it.  Nothing in the product links,
 * loads or calls it; only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg do.
 *
 * Parity pin: the reference's golden vectors
 * tests/fixtures/golden_master/step_case{1,2,3}_f1.npz (< 10 um after one
 * 20x2 frame) and case{1..4}.npz (per-frame tolerances), copied under
 * tests/golden/ by tests/golden/make_fixtures.py.
 *
 * Every function cites the reference file:line it follows (paths relative
 * to the reference project root).
 */
#ifndef TCLOTH_ORACLE_H
#define TCLOTH_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct OSim OSim;

/* Mesh + simulator construction.  Mirrors ClothMesh::from_raw_with_opts
 * (crates/cloth_core/src/mesh.rs:407-1377) without coarse constraints, followed by GpuClothSimulator::with_options
 * (crates/cloth_core/src/simulation/mod.rs:363-697) and
 * build_simulation_resources (simulation/pipelines.rs:114-912). */
OSim *ocl_create(const float *pos, int n, const uint32_t *edges, int ne,
                 const uint32_t *faces, int nf, const float *inv_masses,
                 const uint32_t *layer_ids, const float *thicknesses,
                 uint32_t layer_id, float thickness, float tension_k,
                 float compression_k, float shear_k, float bending_k);
/* ocl_create with sewing springs (nsew pairs; mesh.rs:706-947: sewing
 * constraints, seam-gated bending, sewing-contracted topology) */
OSim *ocl_create_sewn(const float *pos, int n, const uint32_t *edges, int ne,
                      const uint32_t *faces, int nf, const float *inv_masses,
                      const uint32_t *layer_ids, const float *thicknesses,
                      uint32_t layer_id, float thickness, float tension_k,
                      float compression_k, float shear_k, float bending_k,
                      const uint32_t *sew, int nsew, float shrink_speed);
void ocl_destroy(OSim *s);
/* simulator-level sewing settings (simulation/mod.rs:1211-1255) */
void ocl_set_sewing(OSim *s, float stiffness, int lock, float lock_dist, float shrink_speed);
/* sewing constraints in colour order: returns the count; any output may be NULL */
int ocl_get_sewing(const OSim *s, int *ncolors, uint32_t *v01, float *cur, uint32_t *off, uint32_t *cnt,
                   uint32_t *rep);

/* setters (simulation/mod.rs, cloth_py/src/lib.rs) */
void ocl_set_gravity(OSim *s, float gx, float gy, float gz);
void ocl_set_damping(OSim *s, float d);
void ocl_set_damping_all(OSim *s, float t, float c, float sh, float b);
void ocl_set_solver_iterations(OSim *s, int it);
void ocl_set_enable_self_collision(OSim *s, int on);
void ocl_set_self_collision_options(OSim *s, float relief, float max_disp_ratio,
                                    int exclude_neighbors, int untangle, int max_iter);
void ocl_set_compliance_all(OSim *s, float tension, float compression, float shear,
                            float bending);
void ocl_add_sphere(OSim *s, const float *c, float r, float fric, float rest);
void ocl_add_capsule(OSim *s, const float *a, const float *b, float r, float fric, float rest);
void ocl_add_plane(OSim *s, const float *pt, const float *nrm, float fric, float rest);
/* tris: T x 9 floats; attrs (nullable): T x 4 (friction, thickness, restitution, flags) */
void ocl_set_mesh_triangles(OSim *s, const float *tris, int T, float fric, float thick,
                            float rest, int single_sided, const float *attrs);
void ocl_clear_colliders(OSim *s);
/* edge colliders (edge_collision.wgsl; mod.rs:1007-1025), off by default */
void ocl_set_edge_collision(OSim *s, int enable, float margin_scale, float margin_offset);
int ocl_num_collider_edges(const OSim *s);
void ocl_set_pin(OSim *s, uint32_t v, const float *target, float w);
void ocl_clear_pins(OSim *s);
void ocl_set_coupled_collider(OSim *s, int on);
void ocl_set_collider_options(OSim *s, int cluster, int recovery, float sweep);
/* narrow-phase pair record of the direct self-collision pass: V-T pairs that
 * pass the cheap tests (self_collision.wgsl:477-520), E-E pairs counted within
 * max_search (self_collision_ee_direct.wgsl:330-360) */
void ocl_set_pair_recording(OSim *s, int on);
void ocl_get_pair_lists(OSim *s, uint32_t *vt, size_t vt_cap, uint32_t *ee, size_t ee_cap, uint32_t counts[2]);

/* time stepping: GpuClothSimulator::step (simulation/dispatch.rs:610-671) */
void ocl_step(OSim *s, float dt, int substeps);

/* state access */
int ocl_num_vertices(const OSim *s);
void ocl_get_positions(const OSim *s, float *out);            /* N*3 */
void ocl_get_state(const OSim *s, float *x, float *p, float *v); /* N*3 each */
void ocl_set_state(OSim *s, const float *x, const float *v);

/* introspection for parity tests */
void ocl_counts(const OSim *s, int *out8);
/* out8: [nd, nb, n_dist_colors, n_bend_colors, n_edges, table_size, num_virtual, multi_layer] */
void ocl_get_distance(const OSim *s, uint32_t *v01, float *rest, float *tc, float *cc,
                      uint32_t *type);
void ocl_get_bending(const OSim *s, uint32_t *v0123, float *rest, float *comp, float *pad0);
/* pad1 of each bending constraint (the seam gate distance of seam entries) */
void ocl_get_bending_gate(const OSim *s, float *pad1);
void ocl_get_dist_colors(const OSim *s, uint32_t *off, uint32_t *cnt);
void ocl_get_bend_colors(const OSim *s, uint32_t *off, uint32_t *cnt);
void ocl_get_edges(const OSim *s, uint32_t *e2, uint32_t *bits);
int ocl_topology_sizes(const OSim *s, int *adj_n, int *twohop_n, int *star_n);
void ocl_get_topology(const OSim *s, uint32_t *adj_off, uint32_t *adj_idx, uint32_t *th_off,
                      uint32_t *th_idx, float *th_rest, float *local_len, uint32_t *star_off,
                      uint32_t *star_idx, uint32_t *island, uint32_t *layer);
float ocl_cell_size(const OSim *s);
/* Builds the vertex (which=0) or edge (which=1) hash from the current
 * predicted positions; outputs cell_starts (table+1) and sorted (n). */
void ocl_build_hash(OSim *s, int which, uint32_t *cell_starts, uint32_t *sorted);
void ocl_get_mesh_triangles(const OSim *s, float *tris16);  /* T x 16 floats (sorted) */
/* self-collision / E-E substep intervals (dispatch.rs:105-114); defaults 1 / 1 */
void ocl_set_self_collision_intervals(OSim *s, int sc_interval, int ee_interval);
/* contact-pair cache (self-collision algorithm 1) */
void ocl_set_pair_cache(OSim *s, int enable, int final_fallback);
void ocl_set_pair_cache_options(OSim *s, uint32_t max_vt, uint32_t max_ee, uint32_t margin_mode, float safety,
                                float hscale, float maxh);
void ocl_get_active_pairs(const OSim *s, uint32_t *counts, uint32_t *vt, size_t vt_cap, uint32_t *ee, size_t ee_cap);

/* Bone SDF (skinning.wgsl, prep_bone_triangles.wgsl, bake_sdf.wgsl,
 * collision.wgsl:116-265).  Matrices: 16 floats, column-major
 * (row j, column k at [k*4 + j]); bind_inv row-major as mod.rs:2339-2345. */
void ocl_half_roundtrip(const float *in, int n, uint16_t *bits, float *out);
void ocl_bone_skin_mats(int nb, const float *world32, const float *bind_inv16, float *out16);
void ocl_bone_skin(int nv, const float *rest4, const uint32_t *bidx4, const float *bw4, const float *skin_mats,
                   float *out4);
void ocl_bone_prep(int nt, const float *skinned4, const float *inv_mats16, const uint32_t *src4,
                   const float *srcw4, float *out16);
void ocl_bone_bake(int nparams, const uint32_t *params16, const float *tris16, uint32_t *atlas);
/* single-mesh SDF bake of a closed mesh (sdf_baker.rs:939-1060,
 * bake_mesh_sdf.wgsl): dims[3], info[20]; texels (w x h x d) when non-NULL */
void ocl_bake_mesh_sdf(const float *verts, int nv, const int32_t *tris, int nt, float voxel, float margin,
                       float friction, float thickness, float restitution, uint32_t *dims, float *info,
                       uint32_t *texels);
void ocl_bake_mesh_sdf_coarse(const float *verts, int nv, const int32_t *tris, int nt, float voxel, float margin,
                              float thickness, uint32_t *dims, float *coarse_voxel, uint32_t *dist, uint32_t *near8);
int ocl_bake_mesh_sdf_hier(const float *verts, int nv, const int32_t *tris, int nt, float voxel, float margin,
                           float friction, float thickness, float restitution, uint32_t *dims, float *info,
                           uint32_t *texels);
void ocl_set_bone_sdf(OSim *s, uint32_t w, uint32_t h, uint32_t d, const uint32_t *atlas, int nbones,
                      const float *infos20, const float *xforms32);

#ifdef __cplusplus
}
#endif
#endif
