// SimConfig JSON and hash; field list in config.hpp.
#include "config.hpp"

#include <charconv>
#include <cmath>
#include <cstdlib>

namespace tcloth {

float compliance_to_stiffness(float c) {
  if (c <= 1e-9f) return 5000.f;
  if (c >= 1e9f) return 0.f;
  return 1.f / c;
}

std::string json_f32(float v) {
  if (!std::isfinite(v)) return "null";
  char buf[64];
  const auto r = std::to_chars(buf, buf + sizeof buf, v, std::chars_format::scientific);
  std::string s(buf, r.ptr);
  std::string out;
  if (s[0] == '-') {
    out = "-";
    s.erase(0, 1);
  }
  const size_t epos = s.find('e');
  const int e = std::atoi(s.c_str() + epos + 1);
  std::string dig;
  for (size_t i = 0; i < epos; ++i)
    if (s[i] != '.') dig.push_back(s[i]);
  // value = 0.<dig> x 10^kk, i.e. <dig> x 10^k
  const int len = int(dig.size()), kk = e + 1, k = kk - len;
  if (k >= 0 && kk <= 13) {
    out += dig + std::string(size_t(k), '0') + ".0";
  } else if (kk > 0 && kk <= 13) {
    out += dig.substr(0, size_t(kk)) + "." + dig.substr(size_t(kk));
  } else if (kk > -6 && kk <= 0) {
    out += "0." + std::string(size_t(-kk), '0') + dig;
  } else if (len == 1) {
    out += dig + "e" + std::to_string(kk - 1);
  } else {
    out += dig.substr(0, 1) + "." + dig.substr(1) + "e" + std::to_string(kk - 1);
  }
  return out;
}

namespace {
struct Obj {
  std::string t = "{";
  void key(const char* k) {
    if (t.size() > 1) t += ",";
    t += "\"";
    t += k;
    t += "\":";
  }
  void f(const char* k, float v) { key(k); t += json_f32(v); }
  void u(const char* k, uint32_t v) { key(k); t += std::to_string(v); }
  void b(const char* k, bool v) { key(k); t += v ? "true" : "false"; }
};
}  // namespace

std::string settings_json(const SimSettings& s) {
  Obj o;
  o.u("version", 1);
  o.key("gravity");
  o.t += "[" + json_f32(s.gravity[0]) + "," + json_f32(s.gravity[1]) + "," + json_f32(s.gravity[2]) + "]";
  o.f("damping", s.damping);
  o.f("tension_damping", s.tension_damping);
  o.f("compression_damping", s.compression_damping);
  o.f("shear_damping", s.shear_damping);
  o.f("bending_damping", s.bending_damping);
  o.f("tension_stiffness", s.tension_stiffness);
  o.f("compression_stiffness", s.compression_stiffness);
  o.f("shear_stiffness", s.shear_stiffness);
  o.f("bending_stiffness", s.bending_stiffness);
  o.u("solver_iterations", s.solver_iterations);
  o.u("solver_mode", s.solver_mode);
  o.u("workgroup_size", s.workgroup_size);
  o.b("enable_self_collision", s.enable_self_collision);
  o.f("relief_factor", s.relief_factor);
  o.f("max_displacement_ratio", s.max_displacement_ratio);
  o.b("exclude_neighbors", s.exclude_neighbors);
  o.b("enable_normal_untangling", s.enable_normal_untangling);
  o.u("self_collision_max_iterations", s.self_collision_max_iterations);
  o.u("coupled_mode", s.coupled_mode);
  o.b("coupled_collider", s.coupled_collider);
  o.u("post_relaxation_iters", s.post_relaxation_iters);
  o.u("substep_interval", s.substep_interval);
  o.u("ee_substep_interval", s.ee_substep_interval);
  o.u("self_collision_algorithm", s.self_collision_algorithm);
  o.b("enable_pair_cache", s.enable_pair_cache);
  o.u("pair_margin_mode", s.pair_margin_mode);
  o.f("pair_safety_margin", s.pair_safety_margin);
  o.f("pair_horizon_scale", s.pair_horizon_scale);
  o.f("pair_max_horizon", s.pair_max_horizon);
  o.u("pair_max_pairs", s.pair_max_pairs);
  o.b("enable_pair_final_fallback", s.enable_pair_final_fallback);
  o.b("enable_edge_collision", s.enable_edge_collision);
  o.f("edge_margin_scale", s.edge_margin_scale);
  o.f("edge_margin_offset", s.edge_margin_offset);
  o.f("sewing_stiffness", s.sewing_stiffness);
  o.f("sewing_shrink_speed", s.sewing_shrink_speed);
  o.b("enable_sewing_lock", s.enable_sewing_lock);
  o.f("sewing_lock_distance", s.sewing_lock_distance);
  o.b("sewing_priority_enabled", s.sewing_priority_enabled);
  o.f("sewing_priority_threshold", s.sewing_priority_threshold);
  o.f("sewing_priority_merge_dist", s.sewing_priority_merge_dist);
  o.u("sewing_priority_ramp_frames", s.sewing_priority_ramp_frames);
  o.u("sewing_priority_max_frames", s.sewing_priority_max_frames);
  o.f("areal_density", s.areal_density);
  o.b("enable_adaptive_substep", s.enable_adaptive_substep);
  o.u("min_substeps", s.min_substeps);
  o.u("max_substeps", s.max_substeps);
  o.b("auto_coupled_on_low_substeps", s.auto_coupled_on_low_substeps);
  o.b("auto_compensate_iterations", s.auto_compensate_iterations);
  o.b("enable_strain_adaptive", s.enable_strain_adaptive);
  o.f("strain_tolerance", s.strain_tolerance);
  o.t += "}";
  return o.t;
}

uint64_t settings_hash(const std::string& json) {
  uint64_t h = 0xcbf29ce484222325ull;
  for (unsigned char c : json) {
    h ^= c;
    h *= 0x100000001b3ull;
  }
  return h;
}

}  // namespace tcloth
