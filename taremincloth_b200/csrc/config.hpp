// The simulator's settings as the reference's SimConfig record
// (crates/cloth_core/src/config.rs:40-140, filled by
// crates/cloth_core/src/simulation/config_impl.rs:16-78), its JSON text and
// the FNV-1a hash of that text (config.rs:205-214).
#pragma once
#include <cstdint>
#include <string>

namespace tcloth {

struct SimSettings {
  float gravity[3] = {0.f, 0.f, -9.81f};
  float damping = 1.f, tension_damping = 0.f, compression_damping = 0.f, shear_damping = 0.f, bending_damping = 0.f;
  float tension_stiffness = 0.f, compression_stiffness = 0.f, shear_stiffness = 0.f, bending_stiffness = 0.f;
  uint32_t solver_iterations = 2, solver_mode = 0, workgroup_size = 32;
  bool enable_self_collision = true;
  float relief_factor = 0.2f, max_displacement_ratio = 0.2f;
  bool exclude_neighbors = true, enable_normal_untangling = true;
  uint32_t self_collision_max_iterations = 256, coupled_mode = 0;
  bool coupled_collider = false;
  uint32_t post_relaxation_iters = 1, substep_interval = 1, ee_substep_interval = 1, self_collision_algorithm = 0;
  bool enable_pair_cache = false;
  uint32_t pair_margin_mode = 1;
  float pair_safety_margin = 0.005f, pair_horizon_scale = 1.3f, pair_max_horizon = 0.02f;
  uint32_t pair_max_pairs = 65536;
  bool enable_pair_final_fallback = true, enable_edge_collision = false;
  float edge_margin_scale = 1.f, edge_margin_offset = 0.f;
  float sewing_stiffness = 10000.f, sewing_shrink_speed = 1.f;
  bool enable_sewing_lock = true;
  float sewing_lock_distance = 0.02f, areal_density = 0.15f;
  bool sewing_priority_enabled = false;
  float sewing_priority_threshold = 0.9f, sewing_priority_merge_dist = 0.005f;
  uint32_t sewing_priority_ramp_frames = 3, sewing_priority_max_frames = 600;
  bool enable_adaptive_substep = false;
  uint32_t min_substeps = 4, max_substeps = 64;
  bool auto_coupled_on_low_substeps = true, auto_compensate_iterations = true, enable_strain_adaptive = true;
  float strain_tolerance = 0.008f;
};

// compliance_to_stiffness (config_impl.rs:4-12) with scale 1
float compliance_to_stiffness(float compliance);
// compact JSON, fields in the record's declaration order
std::string settings_json(const SimSettings& s);
// 64-bit FNV-1a over the bytes of the JSON text
uint64_t settings_hash(const std::string& json);
// the f32 text of the JSON: shortest round-trip digits, positional when the
// decimal exponent allows, else d.ddde<exp>; non-finite values print null
std::string json_f32(float v);

}  // namespace tcloth
