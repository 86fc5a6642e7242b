// Device vector math for the XPBD substep kernels.
//
// Every helper evaluates in the operand order of the reference WGSL
// (dot = (x*x + y*y) + z*z, mix = a*(1-t) + b*t, vector / scalar divides each
// component).  The library is compiled with --fmad=false and IEEE division /
// square root, so each float operation rounds once, exactly as written.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace tcloth {

struct V3 {
  float x, y, z;
};

__device__ __forceinline__ V3 mk(float x, float y, float z) { return V3{x, y, z}; }
__device__ __forceinline__ V3 mk(const float4& a) { return V3{a.x, a.y, a.z}; }
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3 operator-(V3 a) { return V3{-a.x, -a.y, -a.z}; }
__device__ __forceinline__ V3 operator*(V3 a, float s) { return V3{a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ V3 operator/(V3 a, float s) { return V3{a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 cross(V3 a, V3 b) {
  return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ float length(V3 a) { return sqrtf(dot(a, a)); }
__device__ __forceinline__ float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }
__device__ __forceinline__ V3 vmin(V3 a, V3 b) { return V3{fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)}; }
__device__ __forceinline__ V3 vmax(V3 a, V3 b) { return V3{fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)}; }
__device__ __forceinline__ float mixf(float a, float b, float t) { return a * (1.0f - t) + b * t; }
__device__ __forceinline__ V3 vmix(V3 a, V3 b, float t) {
  float u = 1.0f - t;
  return V3{a.x * u + b.x * t, a.y * u + b.y * t, a.z * u + b.z * t};
}
// f32 -> i32 of a floored value: saturating, NaN -> 0 (cvt.rzi semantics)
__device__ __forceinline__ int32_t f2i(float f) {
  if (f != f) return 0;
  if (f >= 2147483647.0f) return INT32_MAX;
  if (f <= -2147483648.0f) return INT32_MIN;
  return (int32_t)f;
}

constexpr float kEps = 1e-7f;

// hash_coords (shaders/spatial_grid_sort.wgsl:25-31)
__device__ __forceinline__ uint32_t hash3(int32_t cx, int32_t cy, int32_t cz, uint32_t table) {
  uint32_t h = ((uint32_t)cx * 73856093u) ^ ((uint32_t)cy * 19349663u) ^ ((uint32_t)cz * 83492791u);
  return h % table;
}
struct I3 {
  int32_t x, y, z;
};
__device__ __forceinline__ I3 cell_of(V3 p, float cell) {
  return I3{f2i(floorf(p.x / cell)), f2i(floorf(p.y / cell)), f2i(floorf(p.z / cell))};
}

// closest point on triangle with barycentrics (shaders/self_collision.wgsl:122-166;
// shaders/collision.wgsl:273-319 is the same with an "is face" flag)
__device__ __forceinline__ V3 closest_tri(V3 p, V3 a, V3 b, V3 c, bool& is_face, V3& bary) {
  V3 ab = b - a, ac = c - a, ap = p - a;
  float d1 = dot(ab, ap), d2 = dot(ac, ap);
  is_face = false;
  if (d1 <= 0.0f && d2 <= 0.0f) { bary = mk(1, 0, 0); return a; }
  V3 bp = p - b;
  float d3 = dot(ab, bp), d4 = dot(ac, bp);
  if (d3 >= 0.0f && d4 <= d3) { bary = mk(0, 1, 0); return b; }
  float vc = d1 * d4 - d3 * d2;
  if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) {
    float v = d1 / (d1 - d3);
    bary = mk(1.0f - v, v, 0.0f);
    return a + ab * v;
  }
  V3 cp = p - c;
  float d5 = dot(ab, cp), d6 = dot(ac, cp);
  if (d6 >= 0.0f && d5 <= d6) { bary = mk(0, 0, 1); return c; }
  float vb = d5 * d2 - d1 * d6;
  if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) {
    float w = d2 / (d2 - d6);
    bary = mk(1.0f - w, 0.0f, w);
    return a + ac * w;
  }
  float va = d3 * d6 - d5 * d4;
  if (va <= 0.0f && (d4 - d3) >= 0.0f && (d5 - d6) >= 0.0f) {
    float w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
    bary = mk(0.0f, 1.0f - w, w);
    return b + (c - b) * w;
  }
  float denom = 1.0f / (va + vb + vc);
  float v = vb * denom, w = vc * denom;
  is_face = true;
  bary = mk(1.0f - v - w, v, w);
  return (a + ab * v) + ac * w;
}

// segment-triangle CCD, Moller-Trumbore (shaders/collision.wgsl:322-361)
__device__ __forceinline__ bool seg_tri(V3 po, V3 pn, V3 a, V3 b, V3 c, float& t_out, float& u_out,
                                        float& v_out) {
  V3 d = pn - po;
  float ld = dot(d, d);
  if (ld < 1e-12f) return false;
  V3 e1 = b - a, e2 = c - a;
  V3 pv = cross(d, e2);
  float det = dot(e1, pv);
  float tn = dot(e1, e1) * dot(e2, e2);
  if (det * det <= tn * ld * 1e-10f || tn <= 1e-20f) return false;
  float inv = 1.0f / det;
  V3 tv = po - a;
  float u = dot(tv, pv) * inv;
  if (u < -0.05f || u > 1.05f) return false;
  V3 qv = cross(tv, e1);
  float v = dot(d, qv) * inv;
  if (v < -0.05f || (u + v) > 1.05f) return false;
  float t = dot(e2, qv) * inv;
  if (t >= 0.0f && t <= 1.0f) { t_out = t; u_out = u; v_out = v; return true; }
  return false;
}

// segment_sphere_dist_sq (shaders/collision.wgsl:364-375)
__device__ __forceinline__ float seg_point_d2(V3 a, V3 b, V3 c) {
  V3 ab = b - a;
  float s2 = dot(ab, ab);
  if (s2 <= 1e-12f) { V3 d = a - c; return dot(d, d); }
  float t = clampf(dot(c - a, ab) / s2, 0.0f, 1.0f);
  V3 cl = a + ab * t;
  V3 d = cl - c;
  return dot(d, d);
}

// closest_points_segments (shaders/self_collision_ee_direct.wgsl:152-190)
__device__ __forceinline__ void seg_seg(V3 p1, V3 q1, V3 p2, V3 q2, float& so, float& to) {
  V3 d1 = q1 - p1, d2 = q2 - p2, r = p1 - p2;
  float a = dot(d1, d1), e = dot(d2, d2), f = dot(d2, r);
  if (a <= 1e-12f && e <= 1e-12f) { so = 0.f; to = 0.f; return; }
  if (a <= 1e-12f) { so = 0.f; to = clampf(f / e, 0.0f, 1.0f); return; }
  float c = dot(d1, r);
  if (e <= 1e-12f) { so = clampf(-c / a, 0.0f, 1.0f); to = 0.f; return; }
  float b = dot(d1, d2);
  float den = a * e - b * b;
  float s = 0.0f;
  if (den > a * e * 1e-7f) s = clampf((b * f - c * e) / den, 0.0f, 1.0f);
  float t = (b * s + f) / e;
  if (t < 0.0f) { t = 0.0f; s = clampf(-c / a, 0.0f, 1.0f); }
  else if (t > 1.0f) { t = 1.0f; s = clampf((b - c) / a, 0.0f, 1.0f); }
  so = s;
  to = t;
}

}  // namespace tcloth
