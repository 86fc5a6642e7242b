// Adaptive substep and iteration control: host-side decisions made before a
// frame from the previous frames' feedback (maximum vertex displacement and
// the P95 tensile strain of a strided constraint sample).
//
// Restates compute_effective_substeps / compute_effective_iterations
// (crates/cloth_core/src/simulation/dispatch.rs:477-607) and the feedback
// reduction of update_feedback_from_floats (dispatch.rs:356-429), with the
// reference's defaults (simulation/mod.rs:668-680) and option setters
// (mod.rs:723-790).  All arithmetic is f32 in the reference's order.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

namespace tcloth {

struct AdaptiveCtl {
  bool enabled = false;
  uint32_t min_substeps = 4, max_substeps = 64, base_substeps = 20;
  uint32_t effective_substeps = 0;  // 0 = no history
  uint32_t effective_iterations = 0;
  float mesh_char_len = 0.01f, mesh_avg_edge_len = 0.02f, cloth_thickness = 0.005f;
  uint32_t mesh_diameter_hops = 10;
  bool auto_compensate = true;
  bool strain_adaptive = true;
  float strain_tolerance = 0.008f;
  float last_strain = 0.f;
  float last_max_disp = 0.f, pending_external = 0.f, last_effective_disp = 0.f;

  // set_adaptive_substep_options (mod.rs:723-745): re-applying while enabled
  // keeps the hysteresis history (clamped to the new range); disabling or the
  // first enable clears it and any pending external displacement
  void set_options(bool on, uint32_t mn, uint32_t mx) {
    const uint32_t lo = std::max(mn, 1u), hi = std::max(mx, lo);
    const bool was = enabled;
    enabled = on;
    min_substeps = lo;
    max_substeps = hi;
    if (!on || !was) {
      effective_substeps = 0;
      pending_external = 0.f;
    } else if (effective_substeps > 0) {
      effective_substeps = std::min(std::max(effective_substeps, lo), hi);
    }
  }
  void set_strain_options(bool on, float tol) {
    strain_adaptive = on;
    strain_tolerance = std::min(std::max(tol, 0.0001f), 0.1f);
  }
  void note_external(float d) {
    if (d > pending_external) pending_external = d;
  }

  // compute_effective_substeps (dispatch.rs:477-565)
  uint32_t substeps(float dt, uint32_t requested, const float g[3], uint32_t num_vertices) {
    if (!enabled) {
      effective_substeps = requested > 0 ? requested : base_substeps;
      return effective_substeps;
    }
    const uint32_t mn = std::max(min_substeps, 1u), mx = std::max(max_substeps, mn);
    if (dt <= 0.f || num_vertices == 0) {
      effective_substeps = mn;
      return mn;
    }
    const float ext = pending_external;
    const float max_disp = std::fmax(last_max_disp, ext);
    pending_external = 0.f;
    last_effective_disp = max_disp;
    const float cfl = std::fmax(std::fmin(0.5f * mesh_char_len, cloth_thickness * 1.0f), 0.0025f);
    const uint32_t cfl_steps = (cfl > 1e-6f && max_disp > 1e-6f) ? uint32_t(std::ceil(max_disp / cfl)) : mn;
    const float ga = std::sqrt((g[0] * g[0] + g[1] * g[1]) + g[2] * g[2]);
    const float ff = 0.5f * ga * dt * dt;
    const uint32_t grav_steps = (cfl > 1e-6f && ff > 1e-6f) ? uint32_t(std::ceil(std::sqrt(ff / cfl))) : 1u;
    uint32_t strain_steps = mn;
    if (strain_adaptive && strain_tolerance > 1e-5f) {
      const float ratio = last_strain / strain_tolerance;
      if (ratio > 1.25f) strain_steps = uint32_t(std::ceil(float(mn) * std::fmin(ratio, 2.0f)));
    }
    const uint32_t target = std::min(std::max(std::max(std::max(cfl_steps, grav_steps), strain_steps), mn), mx);
    uint32_t cur;
    if (effective_substeps == 0) {
      cur = target;
    } else {
      const uint32_t prev = std::min(std::max(effective_substeps, mn), mx);
      const int32_t diff = int32_t(target) - int32_t(prev);
      if (std::abs(diff) <= 1) {
        cur = prev;
      } else if (diff > 0) {
        const bool emergency = ext > 1e-4f || max_disp > cfl * 4.0f ||
                               (strain_adaptive && last_strain > strain_tolerance * 3.0f);
        cur = emergency ? target : std::min(target, prev + 2);
      } else {
        cur = std::max(target, prev >= 2 ? prev - 2 : 0u);
      }
    }
    cur = std::min(std::max(cur, mn), mx);
    effective_substeps = cur;
    return cur;
  }

  // compute_effective_iterations (dispatch.rs:568-607)
  uint32_t iterations(uint32_t solver_iterations, uint32_t substeps) {
    if (!enabled || !auto_compensate) {
      effective_iterations = solver_iterations;
      return solver_iterations;
    }
    const uint32_t budget = std::max(base_substeps, 1u) * std::max(solver_iterations, 1u);
    const uint32_t floor_hops = std::min(std::max(mesh_diameter_hops, 15u), 30u);
    const uint32_t base_target = std::min(budget, std::max(floor_hops, 20u));
    uint32_t target = base_target;
    if (strain_adaptive && strain_tolerance > 1e-5f) {
      const float ratio = last_strain / strain_tolerance;
      if (ratio > 1.0f) target = uint32_t(std::ceil(float(base_target) * std::fmin(ratio, 2.0f)));
    }
    const uint32_t comp = (target + substeps - 1) / std::max(substeps, 1u);
    const uint32_t mx = std::max(solver_iterations * 4, 8u);
    effective_iterations = std::min(std::max(comp, std::max(solver_iterations, 1u)), mx);
    return effective_iterations;
  }

  // P95 of the positive strains of a sample (update_feedback_from_floats):
  // element floor(len * 0.95) of the sorted positive values, or 0
  static float p95(std::vector<float> pos) {
    if (pos.empty()) return 0.f;
    size_t k = size_t(float(pos.size()) * 0.95f);
    k = std::min(k, pos.size() - 1);
    std::nth_element(pos.begin(), pos.begin() + k, pos.end());
    return pos[k];
  }
};

}  // namespace tcloth
