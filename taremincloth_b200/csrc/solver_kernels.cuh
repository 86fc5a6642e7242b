// XPBD solver kernels: predict, pins, graph-coloured distance / bending
// projection, primitive + triangle-mesh collider response, velocity update.
//
// Device layout (structure of arrays, 16-byte records):
//   x4[i] = (x, inv_mass)        committed position ("position" in the reference)
//   p4[i] = (p, thickness)       predicted / corrected position ("prev_pos")
//   v4[i] = (v, layer bits)
// One thread per vertex / constraint; each kernel restates one WGSL entry
// point of crates/cloth_core/src/shaders/.
#pragma once
#include <cooperative_groups.h>

#include "bone_sdf.cuh"
#include "vmath.cuh"

namespace tcloth {

// Programmatic dependent launch: wait until the preceding kernel of the stream
// has finished and its writes are visible (a no-op for a launch without the
// attribute), then allow the next kernel to begin launching.  The per-colour
// kernels call it first, so only launch latency overlaps, never data.
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" :::);
}


// Loads of data that other blocks of a persistent launch write between two
// grid barriers go through L2 (ld.global.cg) so no SM reads a stale L1 line.
template <bool kCg>
__device__ __forceinline__ float4 ld4(const float4* p) {
  if constexpr (kCg) return __ldcg(p); else return *p;
}
template <bool kCg>
__device__ __forceinline__ float ld1(const float* p) {
  if constexpr (kCg) return __ldcg(p); else return *p;
}

// Where a per-element function reads and writes the vertex records.  GMem:
// the global arrays (kCg: loads through L2, for launches in which other
// blocks write the same records between barriers).  The staged cluster
// solver passes a policy over its shared-memory slices instead; the
// arithmetic is the same either way.
template <bool kCgLoads>
struct GMem {
  static constexpr bool kCg = kCgLoads;
  float4* x4;
  float4* p4;
  float4* v4;
  __device__ __forceinline__ float4 ldx(uint32_t i) const { return ld4<kCg>(x4 + i); }
  __device__ __forceinline__ float4 ldp(uint32_t i) const { return ld4<kCg>(p4 + i); }
  __device__ __forceinline__ float4 ldv(uint32_t i) const { return ld4<kCg>(v4 + i); }
  __device__ __forceinline__ void stx(uint32_t i, float4 v) const { x4[i] = v; }
  __device__ __forceinline__ void stp(uint32_t i, float4 v) const { p4[i] = v; }
  __device__ __forceinline__ void stv(uint32_t i, float4 v) const { v4[i] = v; }
};

struct SubstepParams {
  float dt;       // substep dt (already max(dt, 1e-8) where the shaders do so)
  float gx, gy, gz;
  float damping;  // air damping
  float td, cd, sd, bd;  // Rayleigh damping: tension, compression, shear, bending
};

// shaders/predict.wgsl:33-55
template <class M>
__device__ __forceinline__ void predict_vertex_m(uint32_t i, const M& m, const SubstepParams& sp) {
  float4 x = m.ldx(i), p = m.ldp(i), v = m.ldv(i);
  const float dt = fmaxf(sp.dt, 1e-8f);
  if (x.w <= 0.0f) {
    v.x = 0.f; v.y = 0.f; v.z = 0.f;
    p.x = x.x; p.y = x.y; p.z = x.z;
  } else {
    const float s = fmaxf(0.0f, 1.0f - sp.damping * dt);
    V3 vv = mk(v) * s + mk(sp.gx, sp.gy, sp.gz) * dt;
    V3 pp = mk(x) + vv * dt;
    v.x = vv.x; v.y = vv.y; v.z = vv.z;
    p.x = pp.x; p.y = pp.y; p.z = pp.z;
  }
  m.stp(i, p);
  m.stv(i, v);
}
template <bool kCg>
__device__ __forceinline__ void predict_vertex(uint32_t i, const float4* __restrict__ x4, float4* __restrict__ p4,
                                               float4* __restrict__ v4, const SubstepParams& sp) {
  predict_vertex_m(i, GMem<kCg>{const_cast<float4*>(x4), p4, v4}, sp);
}
__global__ void k_predict(uint32_t n, const float4* __restrict__ x4, float4* __restrict__ p4,
                          float4* __restrict__ v4, SubstepParams sp) {
  pdl_enter();
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  predict_vertex<false>(i, x4, p4, v4, sp);
}

// shaders/pin.wgsl:56-92; pins are on distinct vertices, so order is free
template <class M>
__device__ __forceinline__ void pin_one_m(uint32_t k, const uint32_t* __restrict__ pin_v,
                                          const float4* __restrict__ pin_t, const M& m, float dt_sub) {
  const uint32_t vi = pin_v[k];
  const float4 t = pin_t[k];  // target xyz, weight
  const float w = clampf(t.w, 0.0f, 1.0f);
  if (w <= 0.0f) return;
  const float im = m.ldx(vi).w;
  float4 p = m.ldp(vi);
  if (im <= 0.0f) {
    p.x = t.x; p.y = t.y; p.z = t.z;
    m.stp(vi, p);
    return;
  }
  V3 d = mk(p) - mk(t);
  float dist = length(d);
  if (!(dist > kEps)) return;
  V3 nn = d / dist;
  float dt = fmaxf(dt_sub, 1e-8f);
  float comp = 1e-3f * (1.0f - w) / fmaxf(w, 1e-6f);
  float alpha = comp / (dt * dt);
  float corr = -dist / (im + alpha);
  V3 np = mk(p) + nn * (im * corr);
  p.x = np.x; p.y = np.y; p.z = np.z;
  m.stp(vi, p);
}
template <bool kCg>
__device__ __forceinline__ void pin_one(uint32_t k, const uint32_t* __restrict__ pin_v,
                                        const float4* __restrict__ pin_t, const float4* __restrict__ x4,
                                        float4* __restrict__ p4, float dt_sub) {
  pin_one_m(k, pin_v, pin_t, GMem<kCg>{const_cast<float4*>(x4), p4, nullptr}, dt_sub);
}
__global__ void k_pin(uint32_t npins, const uint32_t* __restrict__ pin_v, const float4* __restrict__ pin_t,
                      const float4* __restrict__ x4, float4* __restrict__ p4, float dt_sub) {
  pdl_enter();
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= npins) return;
  pin_one<false>(k, pin_v, pin_t, x4, p4, dt_sub);
}

// One distance constraint (shaders/distance.wgsl:60-124).  dist_par =
// (rest, tension compliance, compression compliance, shear flag).
// distance_core takes the constraint's record (ids e, params c) and lambda l
// already loaded and writes the new lambda to *lam_out.
template <class M>
__device__ __forceinline__ void distance_core(uint2 e, float4 c, float l, float* __restrict__ lam_out, const M& m,
                                              const SubstepParams& sp, bool damped) {
  // every load of the constraint issued together: within a colour no other
  // thread writes these addresses, so this changes latency, not results
  const float4 xa = m.ldx(e.x), xb = m.ldx(e.y);
  const float4 q0 = m.ldp(e.x), q1 = m.ldp(e.y);
  const float w0 = xa.w, w1 = xb.w;
  const float ws = w0 + w1;
  if (ws <= kEps) return;
  const V3 p0 = mk(q0), p1 = mk(q1);
  const V3 delta = p0 - p1;
  const float dist = length(delta);
  if (dist <= kEps) return;
  const float cv = dist - c.x;
  const float comp = cv >= 0.0f ? c.y : c.z;
  if (comp >= 1e9f) return;
  const V3 dir = delta / dist;
  const float dt = fmaxf(sp.dt, 1e-8f);
  const float alpha = comp / (dt * dt);
  if (damped) {
    const float damp = c.w != 0.0f ? sp.sd : (cv >= 0.0f ? sp.td : sp.cd);
    const float tau = damp * 1e-5f;
    const float gamma = fminf(tau / dt, 1e4f);
    const V3 rel = (p0 - mk(xa)) - (p1 - mk(xb));
    const float vp = dot(dir, rel);
    const float dl = (-cv - alpha * l - gamma * vp) / ((1.0f + gamma) * ws + alpha);
    *lam_out = l + dl;
    const V3 n0 = p0 + dir * (w0 * dl), n1 = p1 + dir * (-w1 * dl);
    m.stp(e.x, make_float4(n0.x, n0.y, n0.z, q0.w));
    m.stp(e.y, make_float4(n1.x, n1.y, n1.z, q1.w));
    return;
  }
  // gamma == 0: (-cv - alpha*l - 0*vp) / (1*ws + alpha)
  const float dl = (-cv - alpha * l) / (1.0f * ws + alpha);
  *lam_out = l + dl;
  const V3 n0 = p0 + dir * (w0 * dl), n1 = p1 + dir * (-w1 * dl);
  m.stp(e.x, make_float4(n0.x, n0.y, n0.z, q0.w));
  m.stp(e.y, make_float4(n1.x, n1.y, n1.z, q1.w));
}
template <class M>
__device__ __forceinline__ void project_distance_m(uint32_t ci, const uint2* __restrict__ ids,
                                                   const float4* __restrict__ par, const M& m,
                                                   float* __restrict__ lam, const SubstepParams& sp, bool damped) {
  distance_core(ids[ci], par[ci], ld1<M::kCg>(lam + ci), lam + ci, m, sp, damped);
}
template <bool kCg>
__device__ __forceinline__ void project_distance(uint32_t ci, const uint2* __restrict__ ids,
                                                 const float4* __restrict__ par, float4* __restrict__ x4,
                                                 float4* __restrict__ p4, float* __restrict__ lam,
                                                 const SubstepParams& sp, bool damped) {
  project_distance_m(ci, ids, par, GMem<kCg>{x4, p4, nullptr}, lam, sp, damped);
}

// The constraint records are written only by host uploads, never by a
// kernel, so they are loaded before griddepcontrol.wait, while the previous
// kernel of the stream may still run; lambda and the vertices, which the
// previous kernel may write, are loaded after it.
__global__ void k_distance(uint32_t off, uint32_t cnt, const uint2* __restrict__ ids, const float4* __restrict__ par,
                           float4* __restrict__ x4, float4* __restrict__ p4, float* __restrict__ lam,
                           SubstepParams sp, bool damped) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  uint2 e = make_uint2(0u, 0u);
  float4 c = make_float4(0.f, 0.f, 0.f, 0.f);
  if (k < cnt) {
    e = ids[off + k];
    c = par[off + k];
  }
  pdl_enter();
  if (k >= cnt) return;
  distance_core(e, c, lam[off + k], lam + off + k, GMem<false>{x4, p4, nullptr}, sp, damped);
}

// One bending constraint (shaders/bending.wgsl:59-126).  bend_par =
// (rest, compliance, kind, seam gap).
// bending_core: the record (ids e, params c) and lambda l already loaded
template <class M>
__device__ __forceinline__ void bending_core(uint4 e, float4 c, float l, float* __restrict__ lam_out, const M& m,
                                             const SubstepParams& sp, bool damped) {
  if (c.y >= 1e9f) return;
  // loads of the written pair issued together (see project_distance)
  const float4 xc = m.ldx(e.z), xd = m.ldx(e.w);
  const float4 q2 = m.ldp(e.z), q3 = m.ldp(e.w);
  const float w2 = xc.w, w3 = xd.w;
  const float ws = w2 + w3;
  if (ws <= kEps) return;
  const V3 p2 = mk(q2), p3 = mk(q3);
  const V3 delta = p2 - p3;
  const float dist = length(delta);
  if (dist <= kEps) return;
  if (c.z > 0.5f && c.z < 1.5f) {
    if (dist >= c.x) return;
    float gap = length(mk(m.ldp(e.x)) - mk(m.ldp(e.y)));
    if (gap > c.w) return;
  }
  const V3 dir = delta / dist;
  const float dt = fmaxf(sp.dt, 1e-8f);
  const float alpha = c.y / (dt * dt);
  const float cv = dist - c.x;
  float dl;
  if (damped) {
    const float tau = sp.bd * 1e-5f;
    const float gamma = fminf(tau / dt, 1e4f);
    const V3 rel = (p2 - mk(xc)) - (p3 - mk(xd));
    const float vp = dot(dir, rel);
    dl = (-cv - alpha * l - gamma * vp) / ((1.0f + gamma) * ws + alpha);
  } else {
    dl = (-cv - alpha * l) / (1.0f * ws + alpha);
  }
  *lam_out = l + dl;
  const V3 n2 = p2 + dir * (w2 * dl), n3 = p3 + dir * (-w3 * dl);
  m.stp(e.z, make_float4(n2.x, n2.y, n2.z, q2.w));
  m.stp(e.w, make_float4(n3.x, n3.y, n3.z, q3.w));
}
template <class M>
__device__ __forceinline__ void project_bending_m(uint32_t ci, const uint4* __restrict__ ids,
                                                  const float4* __restrict__ par, const M& m,
                                                  float* __restrict__ lam, const SubstepParams& sp, bool damped) {
  const float4 c = par[ci];
  if (c.y >= 1e9f) return;
  bending_core(ids[ci], c, ld1<M::kCg>(lam + ci), lam + ci, m, sp, damped);
}
template <bool kCg>
__device__ __forceinline__ void project_bending(uint32_t ci, const uint4* __restrict__ ids,
                                                const float4* __restrict__ par, float4* __restrict__ x4,
                                                float4* __restrict__ p4, float* __restrict__ lam,
                                                const SubstepParams& sp, bool damped) {
  project_bending_m(ci, ids, par, GMem<kCg>{x4, p4, nullptr}, lam, sp, damped);
}

// (records loaded before griddepcontrol.wait, as in k_distance)
__global__ void k_bending(uint32_t off, uint32_t cnt, const uint4* __restrict__ ids, const float4* __restrict__ par,
                          float4* __restrict__ x4, float4* __restrict__ p4, float* __restrict__ lam,
                          SubstepParams sp, bool damped) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  uint4 e = make_uint4(0u, 0u, 0u, 0u);
  float4 c = make_float4(0.f, 0.f, 0.f, 0.f);
  if (k < cnt) {
    e = ids[off + k];
    c = par[off + k];
  }
  pdl_enter();
  if (k >= cnt || c.y >= 1e9f) return;
  bending_core(e, c, lam[off + k], lam + off + k, GMem<false>{x4, p4, nullptr}, sp, damped);
}

// Sewing settings of a frame (dispatch.rs:29-35): compliance 0 when the
// simulator's sewing stiffness is >= 5000, else 1 / max(stiffness, 1);
// lock > 0.5 latches a closing seam; lock_dist its distance floor.
struct SewParams {
  float compliance, lock, lock_dist;
};
// Shrink of the sewing rest lengths, once per substep before predict
// (shaders/sewing_shrink.wgsl:38-49).  rest = (current, target).
__global__ void k_sew_shrink(uint32_t cnt, float2* __restrict__ rest, float speed, float dt_sub) {
  pdl_enter();
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= cnt) return;
  float2 r = rest[k];
  const float dt = fmaxf(dt_sub, 1e-8f);
  r.x = fmaxf(r.y, r.x - speed * dt);
  rest[k] = r;
}
// One sewing constraint (shaders/sewing.wgsl:57-110): XPBD towards the
// current rest length; within max(thickness sum, lock distance) with the
// lock on, a hard constraint towards the target length, which also becomes
// the current one.
template <bool kCg>
__device__ __forceinline__ void project_sewing(uint32_t ci, const uint2* __restrict__ ids, float2* __restrict__ rest,
                                               const float4* __restrict__ x4, float4* __restrict__ p4,
                                               float* __restrict__ lam, float dt_sub, const SewParams& sw) {
  const uint2 e = ids[ci];
  const float4 xa = ld4<kCg>(x4 + e.x), xb = ld4<kCg>(x4 + e.y);
  const float4 qa = ld4<kCg>(p4 + e.x), qb = ld4<kCg>(p4 + e.y);
  const float w0 = xa.w, w1 = xb.w;
  const float ws = w0 + w1;
  if (ws <= kEps) return;
  const V3 p0 = mk(qa), p1 = mk(qb);
  const V3 delta = p0 - p1;
  const float dist = length(delta);
  if (dist <= kEps) return;
  const float dt = fmaxf(dt_sub, 1e-8f);
  const V3 dir = delta / dist;
  const float2 r = kCg ? __ldcg(rest + ci) : rest[ci];
  float target = r.x, comp = sw.compliance;
  const float lock_thresh = fmaxf(qa.w + qb.w, sw.lock_dist);
  if (sw.lock > 0.5f && dist <= lock_thresh) {
    comp = 0.0f;
    target = r.y;
    rest[ci] = make_float2(r.y, r.y);
  }
  const float alpha = comp / (dt * dt);
  const float cv = dist - target;
  const float l = ld1<kCg>(lam + ci);
  const float dl = (-cv - alpha * l) / (ws + alpha);
  lam[ci] = l + dl;
  const V3 n0 = p0 + dir * (w0 * dl), n1 = p1 + dir * (-w1 * dl);
  p4[e.x] = make_float4(n0.x, n0.y, n0.z, qa.w);
  p4[e.y] = make_float4(n1.x, n1.y, n1.z, qb.w);
}
// gate: null, or the warm start's fallback flag (skipped unless set)
__global__ void k_sewing(uint32_t off, uint32_t cnt, const uint2* __restrict__ ids, float2* __restrict__ rest,
                         const float4* __restrict__ x4, float4* __restrict__ p4, float* __restrict__ lam,
                         float dt_sub, SewParams sw, const unsigned int* gate) {
  pdl_enter();
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= cnt || (gate && !*gate)) return;
  project_sewing<false>(off + k, ids, rest, x4, p4, lam, dt_sub, sw);
}

// shaders/update_vel.wgsl:33-53
template <class M>
__device__ __forceinline__ void update_vertex_m(uint32_t i, const M& m, float dt_sub) {
  float4 x = m.ldx(i);
  const float4 p = m.ldp(i);
  float4 v = m.ldv(i);
  const float dt = fmaxf(dt_sub, 1e-8f);
  if (x.w > 0.0f) {
    V3 vv = (mk(p) - mk(x)) / dt;
    v.x = vv.x; v.y = vv.y; v.z = vv.z;
  } else {
    v.x = 0.f; v.y = 0.f; v.z = 0.f;
  }
  x.x = p.x; x.y = p.y; x.z = p.z;
  m.stx(i, x);
  m.stv(i, v);
}
template <bool kCg>
__device__ __forceinline__ void update_vertex(uint32_t i, float4* __restrict__ x4, const float4* __restrict__ p4,
                                              float4* __restrict__ v4, float dt_sub) {
  update_vertex_m(i, GMem<kCg>{x4, const_cast<float4*>(p4), v4}, dt_sub);
}
__global__ void k_update_vel(uint32_t n, float4* __restrict__ x4, const float4* __restrict__ p4,
                             float4* __restrict__ v4, float dt_sub) {
  pdl_enter();
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  update_vertex<false>(i, x4, p4, v4, dt_sub);
}

// ---------------------------------------------------------------------
// colliders
// ---------------------------------------------------------------------
struct Prim {      // sphere (0), capsule (1), plane (2)
  float4 h;        // friction, restitution, radius, type
  float4 a, b;     // point a / b (plane: point, normal)
};
struct MeshTri {   // 64 B, Morton-sorted (simulation/mod.rs:2613-2641)
  float4 p0f;      // p0, friction
  float4 p1t;      // p1, thickness
  float4 p2r;      // p2, restitution
  float4 fl;       // flags bits, 0, 0, 0
};

// apply_contact_response (shaders/collision.wgsl:83-108)
__device__ __forceinline__ void contact(V3 target, V3 n, float fric, float rest, float dt, V3 p_init, V3& xn,
                                        V3& p) {
  V3 total = target - xn;
  V3 tang = total - n * dot(total, n);
  p = target - tang * clampf(fric, 0.0f, 1.0f);
  float edt = fmaxf(dt, 1e-6f);
  float vin = dot((p_init - xn) / edt, n);
  float des = 0.0f;
  if (vin < 0.0f) des = -clampf(rest, 0.0f, 1.0f) * vin;
  float dxn = dot(target - xn, n) - des * edt;
  xn = xn + n * dxn;
}

struct MeshState {
  bool front = false, has_rec = false;
  float best_depth = 999999.0f, bf = 0.f, br = 0.f;
  V3 bpos, bn;
};

// one triangle of the mesh collider loop (shaders/collision.wgsl:461-541)
__device__ __forceinline__ void mesh_triangle(const MeshTri& tri, float thickness, V3 xpos, V3& p, V3& xn, float dt,
                                              V3 pinit, bool recovery_on, MeshState& st) {
  const V3 t0 = mk(tri.p0f), t1 = mk(tri.p1t), t2 = mk(tri.p2r);
  const float fric = tri.p0f.w, tthick = tri.p1t.w, rest = tri.p2r.w;
  const uint32_t flags = __float_as_uint(tri.fl.x);
  const float td = thickness + tthick;
  const V3 cr = cross(t1 - t0, t2 - t0);
  const float cl = length(cr);
  if (cl < kEps) return;
  const V3 fn = cr / cl;
  const bool single = (flags & 1u) != 0u;
  float th, tu, tv;
  if (seg_tri(xpos, p, t0, t1, t2, th, tu, tv)) {
    V3 hit = xpos + (p - xpos) * th;
    V3 nn = fn;
    if (dot(p - xpos, fn) > 0.0f && !single) nn = -fn;
    contact(hit + nn * td, nn, fric, rest, dt, pinit, xn, p);
    st.front = true;
  }
  bool isf;
  V3 bary;
  const V3 q = closest_tri(p, t0, t1, t2, isf, bary);
  const V3 delta = p - q;
  const float dist = length(delta);
  const float sd = dot(delta, fn);
  if (single) {
    if (sd >= 0.0f) {
      if (dist < td) {
        V3 nn = fn;
        if (dist > kEps) nn = delta / dist;
        contact(p + nn * (td - dist), nn, fric, rest, dt, pinit, xn, p);
        st.front = true;
      }
    } else {
      const bool rdis = (flags & 2u) != 0u;
      if (recovery_on && !rdis) {
        const float maxd = td * 3.0f;
        if (isf && dist < maxd && dist <= fabsf(sd) * 1.1f + kEps) {
          if (dist < st.best_depth) {
            st.best_depth = dist;
            st.bn = fn;
            st.bpos = p + fn * (td - sd);
            st.bf = fric;
            st.br = rest;
            st.has_rec = true;
          }
        }
      }
    }
  } else {
    if (dist < td && sd >= -td) {
      V3 nn = fn;
      if (dist > kEps) nn = delta / dist;
      contact(p + nn * (td - dist), nn, fric, rest, dt, pinit, xn, p);
      st.front = true;
    }
  }
}

struct ColliderArgs {
  const Prim* prims;
  uint32_t nprims;
  // batched instances: primitive range (offset, count) of each vertex's
  // instance; null when every vertex sees every primitive
  const uint32_t* vinst;
  const uint2* inst_prims;
  const MeshTri* tris;
  const float4* bounds;   // per triangle: centroid, r
  const float4* cl16;     // per 16 triangles: conservative sphere for 1.5 r
  const float4* cl256;    // per 256 triangles
  const float4* cl4096;   // per 4,096 triangles
  uint32_t ntris;
  bool recovery;
  BoneSdfArgs bone;       // bone SDF colliders (nbones == 0: off)
};

// Conservative skip test for a group of triangles: true only when every
// member triangle would fail its own test seg_point_d2 > (1.5 r + th)^2.
__device__ __forceinline__ bool group_far(V3 a, V3 b, float4 g, float th) {
  float R = g.w + th;
  float d2 = seg_point_d2(a, b, mk(g));
  return d2 > R * R * 1.0004f + 1e-12f;
}

// shaders/collision.wgsl:378-652 (cluster culling off, the reference
// default).  The triangle loop visits triangles in ascending (Morton) order
// exactly like the reference; three levels of conservative bounding spheres
// (4,096, 256 and 16 triangles, each enclosing its members' own test
// spheres) skip runs of triangles none of which could pass the per-triangle
// test, so the sequence of applied contacts is unchanged.
template <bool kBone, class M>
__device__ __forceinline__ void collide_vertex_m(uint32_t i, const M& m, const ColliderArgs& ca, float dt) {
  float4 x = m.ldx(i);
  if (x.w <= 0.0f) return;
  float4 pr = m.ldp(i);
  V3 p = mk(pr), pinit = p, xn = mk(x);
  const V3 xpos = mk(x);
  const float th = pr.w;
  uint32_t kb = 0, ke = ca.nprims;
  if (ca.vinst) {
    const uint2 r = ca.inst_prims[ca.vinst[i]];
    kb = r.x;
    ke = r.x + r.y;
  }
  for (uint32_t k = kb; k < ke; ++k) {
    const Prim c = ca.prims[k];
    const uint32_t type = __float_as_uint(c.h.w);
    const float fric = c.h.x, rest = c.h.y, r = c.h.z;
    if (type == 0u) {
      float tr = r + th;
      V3 d = p - mk(c.a);
      float dist = length(d);
      if (dist < tr) {
        V3 nn = mk(0.f, 0.f, 1.f);
        if (dist > kEps) nn = d / dist;
        contact(mk(c.a) + nn * tr, nn, fric, rest, dt, pinit, xn, p);
      }
    } else if (type == 1u) {
      float tr = r + th;
      V3 A = mk(c.a), ab = mk(c.b) - A;
      float l2 = dot(ab, ab);
      float t = 0.0f;
      if (l2 > kEps) t = clampf(dot(p - A, ab) / l2, 0.0f, 1.0f);
      V3 cl = A + ab * t;
      V3 d = p - cl;
      float dist = length(d);
      if (dist < tr) {
        V3 nn = mk(0.f, 0.f, 1.f);
        if (dist > kEps) nn = d / dist;
        contact(cl + nn * tr, nn, fric, rest, dt, pinit, xn, p);
      }
    } else if (type == 2u) {
      V3 B = mk(c.b);
      V3 pn = B / length(B);
      float dist = dot(p - mk(c.a), pn);
      if (dist < th) contact(p + pn * (th - dist), pn, fric, rest, dt, pinit, xn, p);
    }
  }
  if (ca.ntris > 0) {
    MeshState st;
    st.bpos = p;
    st.bn = mk(0.f, 0.f, 0.f);
    const uint32_t ng256 = (ca.ntris + 255u) / 256u, ng4096 = (ca.ntris + 4095u) / 4096u;
    for (uint32_t g4 = 0; g4 < ng4096; ++g4) {
      if (group_far(xpos, p, ca.cl4096[g4], th)) continue;
      const uint32_t g_end = min((g4 + 1u) * 16u, ng256);
      for (uint32_t g = g4 * 16u; g < g_end; ++g) {
        if (group_far(xpos, p, ca.cl256[g], th)) continue;
        const uint32_t c_end = min((g + 1u) * 16u, (ca.ntris + 15u) / 16u);
        for (uint32_t cgi = g * 16u; cgi < c_end; ++cgi) {
          if (group_far(xpos, p, ca.cl16[cgi], th)) continue;
          const uint32_t t_end = min((cgi + 1u) * 16u, ca.ntris);
          for (uint32_t t = cgi * 16u; t < t_end; ++t) {
            const float4 b = ca.bounds[t];
            const float r = b.w * 1.5f + th;
            if (seg_point_d2(xpos, p, mk(b)) > r * r) continue;
            mesh_triangle(ca.tris[t], th, xpos, p, xn, dt, pinit, ca.recovery, st);
          }
        }
      }
    }
    if (!st.front && st.has_rec) contact(st.bpos, st.bn, st.bf, st.br, dt, pinit, xn, p);
  }
  // phase 3: bone SDF, judged at the current p (collision.wgsl:648)
  if (kBone && ca.bone.nbones > 0u) {
    V3 tgt, bn;
    float bf, br;
    if (bone_sdf_contact(ca.bone, p, th, ca.ntris > 0u, tgt, bn, bf, br)) {
      const V3 pb = p;
      contact(tgt, bn, bf, br, dt, pb, xn, p);
    }
  }
  m.stp(i, make_float4(p.x, p.y, p.z, pr.w));
  m.stx(i, make_float4(xn.x, xn.y, xn.z, x.w));
}
template <bool kCg, bool kBone = false>
__device__ __forceinline__ void collide_vertex(uint32_t i, float4* __restrict__ x4, float4* __restrict__ p4,
                                               const ColliderArgs& ca, float dt) {
  collide_vertex_m<kBone>(i, GMem<kCg>{x4, p4, nullptr}, ca, dt);
}
// kBone: with the bone SDF phase (a separate instantiation, so that kernels
// without bone colliders keep their register budget)
template <bool kBone>
// order: null, or a permutation of the vertices that keeps a warp's vertices
// close in space (they then visit nearly the same collider triangles); each
// vertex's contacts depend on that vertex alone, so any order gives the
// same results.
__global__ void k_collision(uint32_t n, float4* __restrict__ x4, float4* __restrict__ p4, ColliderArgs ca,
                            float dt, const uint32_t* __restrict__ order) {
  pdl_enter();
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (order) i = order[i];
  collide_vertex<false, kBone>(i, x4, p4, ca, dt);
}

// ---------------------------------------------------------------------
// persistent solver kernel
// ---------------------------------------------------------------------
// Grid barrier for a cooperative launch (all blocks resident).  Waits are
// bounded: after spin_limit polls a block records an error and every block
// leaves the kernel at its next barrier, so a stuck barrier ends with a status
// instead of a hang.  `expected` is the number of arrivals that releases the
// barrier (gridDim.x in normal operation).
struct GridBar {
  unsigned int count;
  unsigned int gen;
  int err;
  unsigned int pad;
};
__device__ __forceinline__ bool grid_sync(GridBar* b, unsigned int expected, unsigned int spin_limit) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned int* vgen = &b->gen;
    volatile int* verr = &b->err;
    const unsigned int g = *vgen;
    __threadfence();
    if (*verr == 0) {
      if (atomicAdd(&b->count, 1u) == expected - 1u) {
        atomicExch(&b->count, 0u);
        __threadfence();
        atomicAdd(&b->gen, 1u);
      } else {
        unsigned int spins = 0;
        while (*vgen == g && *verr == 0) {
          if (++spins > spin_limit) {
            atomicExch(&b->err, 1);
            break;
          }
          __nanosleep(100);
        }
      }
    }
    __threadfence();
  }
  __syncthreads();
  return *((volatile int*)&b->err) == 0;
}

struct SolverArgs {
  uint32_t n, nsub, iters, npins, ndc, nbc;
  bool hascol, coupled, ddamp, bdamp, with_update;
  SubstepParams sp;
  float4 *x4, *p4, *v4;
  const uint2* dist_ids;
  const float4* dist_par;
  float* dlam;
  uint32_t nd;
  const uint4* bend_ids;
  const float4* bend_par;
  float* blam;
  uint32_t nb;
  const uint32_t* dist_off;  // per colour
  const uint32_t* dist_cnt;
  const uint32_t* bend_off;
  const uint32_t* bend_cnt;
  const uint32_t* pin_v;
  const float4* pin_t;
  ColliderArgs ca;
  // sewing: shrink at the start of each substep, the nsc colours after the
  // distance colours of every iteration, and, with with_update, once more
  // after the final pins (the final sewing pass before the velocity update)
  uint32_t nsw, nsc;
  const uint2* sew_ids;
  float2* sew_rest;
  float* slam;
  const uint32_t* sew_off;
  const uint32_t* sew_cnt;
  float sew_speed;
  SewParams sw;
  GridBar* bar;
  unsigned int expected;  // arrivals per barrier
  unsigned int spin_limit;
  // learned warm start: predict ran outside (skip_predict), the iteration
  // correction p - p_pred goes to dprev, and after iters (the reduced count)
  // the RMS residual |C + alpha~ lambda| over all distance and bending
  // constraints decides whether iters_extra more iterations run
  // (res_thresh: the plain solver's residual).  The sum is reduced in a
  // fixed order (per block, then over res_part[] by every block), so every
  // block takes the same decision and runs are bit-reproducible.
  bool skip_predict;
  const float4* ppred;
  float4* dprev;
  uint32_t iters_extra;
  float res_thresh;
  float res_ratio;            // > 0: the threshold is max(res_ratio * *res_pred, res_floor) instead
  float res_floor;
  const float* res_pred;      // RMS residual of the predicted positions (lambda = 0)
  float* res_part;            // [gridDim.x] per-block sums of squares
  float* res_out;             // RMS of the latest check
  unsigned int* fallbacks;    // count of substeps that ran the extra iterations
};

__device__ __forceinline__ float residual_dist(uint32_t ci, const uint2* ids, const float4* par, const float4* p4,
                                               const float* lam, float dt) {
  const uint2 e = ids[ci];
  const float4 c = par[ci];
  const float cv = length(mk(__ldcg(p4 + e.x)) - mk(__ldcg(p4 + e.y))) - c.x;
  const float comp = cv >= 0.f ? c.y : c.z;
  return comp < 1e9f ? fabsf(cv + comp / (dt * dt) * (lam ? __ldcg(lam + ci) : 0.f)) : 0.f;
}
__device__ __forceinline__ float residual_bend(uint32_t ci, const uint4* ids, const float4* par, const float4* p4,
                                               const float* lam, float dt) {
  const uint4 e = ids[ci];
  const float4 c = par[ci];
  if (c.y >= 1e9f) return 0.f;
  const float cv = length(mk(__ldcg(p4 + e.z)) - mk(__ldcg(p4 + e.w))) - c.x;
  return fabsf(cv + c.y / (dt * dt) * (lam ? __ldcg(lam + ci) : 0.f));
}

// Sum of the squared residuals of this thread's grid-stride share of the
// distance and bending constraints, reduced over the block (red: 8 floats of
// shared memory); the block's sum is returned on thread 0.  The per-colour
// check and the persistent solver share this and ws_total_residual, so that
// with the same grid both take the same decision bit for bit.
__device__ __forceinline__ float ws_block_residual(uint32_t tid, uint32_t stride, uint32_t nd, uint32_t nb,
                                                   const uint2* dist_ids, const float4* dist_par,
                                                   const uint4* bend_ids, const float4* bend_par, const float4* p4,
                                                   const float* dlam, const float* blam, float dt, float* red) {
  float r2 = 0.f;
  for (uint32_t k = tid; k < nd; k += stride) {
    const float r = residual_dist(k, dist_ids, dist_par, p4, dlam, dt);
    r2 += r * r;
  }
  for (uint32_t k = tid; k < nb; k += stride) {
    const float r = residual_bend(k, bend_ids, bend_par, p4, blam, dt);
    r2 += r * r;
  }
  for (int o = 16; o > 0; o >>= 1) r2 += __shfl_down_sync(0xffffffffu, r2, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = r2;
  __syncthreads();
  float b = 0.f;
  if (threadIdx.x == 0)
    for (int w = 0; w < int(blockDim.x >> 5); ++w) b += red[w];
  return b;
}
// RMS over all constraints from the per-block sums (called by one full
// warp; the result is valid on lane 0)
__device__ __forceinline__ float ws_total_residual(const float* res_part, uint32_t nparts, uint32_t ncons) {
  float t = 0.f;
  for (uint32_t q = threadIdx.x; q < nparts; q += 32) t += __ldcg(res_part + q);
  for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
  return sqrtf(t / float(max(ncons, 1u)));
}

// Residual check of a warm-started substep in the per-colour path: block
// sums (launched with the persistent solver's grid), then one warp decides
// and sets *gate, which the fallback iterations' kernels read.
struct WsCheckArgs {
  uint32_t nd, nb;
  const uint2* dist_ids;
  const float4* dist_par;
  const uint4* bend_ids;
  const float4* bend_par;
  const float4* p4;
  const float* dlam;
  const float* blam;
  float dt, res_thresh;
  float res_ratio;         // > 0: the threshold is max(res_ratio * *res_pred, res_floor)
  float res_floor;
  float* res_pred;         // RMS residual of the predicted positions
  float* res_part;
  float* res_out;
  unsigned int* fallbacks;
  unsigned int* gate;
};
__global__ void __launch_bounds__(256) k_ws_res_part(WsCheckArgs a) {
  pdl_enter();
  __shared__ float red[8];
  const float b = ws_block_residual(blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x, a.nd, a.nb,
                                    a.dist_ids, a.dist_par, a.bend_ids, a.bend_par, a.p4, a.dlam, a.blam,
                                    fmaxf(a.dt, 1e-8f), red);
  if (threadIdx.x == 0) a.res_part[blockIdx.x] = b;
}
__global__ void k_ws_res_decide(WsCheckArgs a, uint32_t nparts) {
  pdl_enter();
  const float rms = ws_total_residual(a.res_part, nparts, a.nd + a.nb);
  if (threadIdx.x == 0) {
    const float thr = a.res_ratio > 0.f ? fmaxf(a.res_ratio * *a.res_pred, a.res_floor) : a.res_thresh;
    const unsigned int extra = rms > thr ? 1u : 0u;
    *a.res_out = rms;
    *a.gate = extra;
    if (extra) *a.fallbacks += 1u;
  }
}
// RMS residual of the predicted positions (block sums of k_ws_res_part
// launched with null lambdas): the reference level of a relative threshold
__global__ void k_ws_res_pred(WsCheckArgs a, uint32_t nparts) {
  pdl_enter();
  const float rms = ws_total_residual(a.res_part, nparts, a.nd + a.nb);
  if (threadIdx.x == 0) *a.res_pred = rms;
}
// Sum of squared residuals of the predicted positions (lambda = 0) into
// *sum, for residual tracking
__global__ void k_residual_pred(uint32_t nd, uint32_t nb, const uint2* dist_ids, const float4* dist_par,
                                const uint4* bend_ids, const float4* bend_par, const float4* p4, float dt,
                                float* sum) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  float r = 0.f;
  if (k < nd) r = residual_dist(k, dist_ids, dist_par, p4, nullptr, dt);
  else if (k < nd + nb) r = residual_bend(k - nd, bend_ids, bend_par, p4, nullptr, dt);
  float s2 = r * r;
  for (int o = 16; o > 0; o >>= 1) s2 += __shfl_down_sync(0xffffffffu, s2, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(sum, s2);
}
// The fallback iterations of the per-colour path: the element functions of
// k_pin / k_distance / k_bending / k_collision, skipped unless *gate is set.
__global__ void k_pin_gated(const unsigned int* gate, uint32_t npins, const uint32_t* __restrict__ pin_v,
                            const float4* __restrict__ pin_t, const float4* __restrict__ x4, float4* __restrict__ p4,
                            float dt_sub) {
  pdl_enter();
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= npins || !*gate) return;
  pin_one<false>(k, pin_v, pin_t, x4, p4, dt_sub);
}
__global__ void k_distance_gated(const unsigned int* gate, uint32_t off, uint32_t cnt, const uint2* __restrict__ ids,
                                 const float4* __restrict__ par, float4* __restrict__ x4, float4* __restrict__ p4,
                                 float* __restrict__ lam, SubstepParams sp, bool damped) {
  pdl_enter();
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= cnt || !*gate) return;
  project_distance<false>(off + k, ids, par, x4, p4, lam, sp, damped);
}
__global__ void k_bending_gated(const unsigned int* gate, uint32_t off, uint32_t cnt, const uint4* __restrict__ ids,
                                const float4* __restrict__ par, float4* __restrict__ x4, float4* __restrict__ p4,
                                float* __restrict__ lam, SubstepParams sp, bool damped) {
  pdl_enter();
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= cnt || !*gate) return;
  project_bending<false>(off + k, ids, par, x4, p4, lam, sp, damped);
}
template <bool kBone>
__global__ void k_collision_gated(const unsigned int* gate, uint32_t n, float4* __restrict__ x4,
                                  float4* __restrict__ p4, ColliderArgs ca, float dt,
                                  const uint32_t* __restrict__ order) {
  pdl_enter();
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !*gate) return;
  if (order) i = order[i];
  collide_vertex<false, kBone>(i, x4, p4, ca, dt);
}

// One cooperative launch runs `nsub` substeps of the constraint phase
// (dispatch.rs:104-250: lambda clear, predict, iterations of pins / distance
// colours / bending colours / coupled collision, decoupled collision, final
// pin) and, with_update set, the velocity update; colours are separated by
// grid barriers instead of kernel launches.  Same per-element functions, so
// the same bits as the launch-per-colour path.
template <bool kBone>
__global__ void __launch_bounds__(256) k_solver_persistent(SolverArgs a) {
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t stride = gridDim.x * blockDim.x;
  const float dts = a.sp.dt;
  for (uint32_t sub = 0; sub < a.nsub; ++sub) {
    for (uint32_t i = tid; i < a.nd; i += stride) a.dlam[i] = 0.f;
    for (uint32_t i = tid; i < a.nb; i += stride) a.blam[i] = 0.f;
    for (uint32_t i = tid; i < a.nsw; i += stride) {
      a.slam[i] = 0.f;
      float2 r = __ldcg(a.sew_rest + i);
      r.x = fmaxf(r.y, r.x - a.sew_speed * fmaxf(dts, 1e-8f));
      a.sew_rest[i] = r;
    }
    if (!a.skip_predict)
      for (uint32_t i = tid; i < a.n; i += stride) predict_vertex<true>(i, a.x4, a.p4, a.v4, a.sp);
    if (!grid_sync(a.bar, a.expected, a.spin_limit)) return;
    uint32_t n_it = a.iters;
    for (uint32_t it = 0; it < n_it; ++it) {
      if (a.npins) {
        for (uint32_t k = tid; k < a.npins; k += stride) pin_one<true>(k, a.pin_v, a.pin_t, a.x4, a.p4, dts);
        if (!grid_sync(a.bar, a.expected, a.spin_limit)) return;
      }
      for (uint32_t c = 0; c < a.ndc; ++c) {
        const uint32_t off = a.dist_off[c], cnt = a.dist_cnt[c];
        if (!cnt) continue;
        for (uint32_t k = tid; k < cnt; k += stride)
          project_distance<true>(off + k, a.dist_ids, a.dist_par, a.x4, a.p4, a.dlam, a.sp, a.ddamp);
        if (!grid_sync(a.bar, a.expected, a.spin_limit)) return;
      }
      for (uint32_t c = 0; c < a.nsc; ++c) {
        const uint32_t off = a.sew_off[c], cnt = a.sew_cnt[c];
        if (!cnt) continue;
        for (uint32_t k = tid; k < cnt; k += stride)
          project_sewing<true>(off + k, a.sew_ids, a.sew_rest, a.x4, a.p4, a.slam, dts, a.sw);
        if (!grid_sync(a.bar, a.expected, a.spin_limit)) return;
      }
      for (uint32_t c = 0; c < a.nbc; ++c) {
        const uint32_t off = a.bend_off[c], cnt = a.bend_cnt[c];
        if (!cnt) continue;
        for (uint32_t k = tid; k < cnt; k += stride)
          project_bending<true>(off + k, a.bend_ids, a.bend_par, a.x4, a.p4, a.blam, a.sp, a.bdamp);
        if (!grid_sync(a.bar, a.expected, a.spin_limit)) return;
      }
      if (a.hascol && a.coupled) {
        for (uint32_t i = tid; i < a.n; i += stride) collide_vertex<true, kBone>(i, a.x4, a.p4, a.ca, dts);
        if (!grid_sync(a.bar, a.expected, a.spin_limit)) return;
      }
      if (it + 1 == a.iters && a.iters_extra > 0) {
        __shared__ float red[8];
        __shared__ int extra;
        const float b = ws_block_residual(tid, stride, a.nd, a.nb, a.dist_ids, a.dist_par, a.bend_ids, a.bend_par,
                                          a.p4, a.dlam, a.blam, fmaxf(dts, 1e-8f), red);
        if (threadIdx.x == 0) __stcg(a.res_part + blockIdx.x, b);
        if (!grid_sync(a.bar, a.expected, a.spin_limit)) return;
        if (threadIdx.x < 32) {
          const float rms = ws_total_residual(a.res_part, gridDim.x, a.nd + a.nb);
          if (threadIdx.x == 0) {
            const float thr = a.res_ratio > 0.f ? fmaxf(a.res_ratio * __ldcg(a.res_pred), a.res_floor) : a.res_thresh;
            extra = rms > thr ? 1 : 0;
            if (blockIdx.x == 0) {
              *a.res_out = rms;
              if (extra) atomicAdd(a.fallbacks, 1u);
            }
          }
        }
        __syncthreads();
        if (extra) n_it = a.iters + a.iters_extra;
        // res_part is rewritten at the next check only after further barriers
      }
    }
    if (a.dprev)
      for (uint32_t i = tid; i < a.n; i += stride) {
        const float4 p = __ldcg(a.p4 + i), q = a.ppred[i];
        a.dprev[i] = make_float4(p.x - q.x, p.y - q.y, p.z - q.z, 0.f);
      }
    if (a.hascol && !a.coupled) {
      for (uint32_t i = tid; i < a.n; i += stride) collide_vertex<true, kBone>(i, a.x4, a.p4, a.ca, dts);
      if (!grid_sync(a.bar, a.expected, a.spin_limit)) return;
    }
    if (a.npins) {
      for (uint32_t k = tid; k < a.npins; k += stride) pin_one<true>(k, a.pin_v, a.pin_t, a.x4, a.p4, dts);
      if (!grid_sync(a.bar, a.expected, a.spin_limit)) return;
    }
    if (a.with_update)  // final sewing (dispatch.rs:323-337); with self-collision it runs after it, outside
      for (uint32_t c = 0; c < a.nsc; ++c) {
        const uint32_t off = a.sew_off[c], cnt = a.sew_cnt[c];
        if (!cnt) continue;
        for (uint32_t k = tid; k < cnt; k += stride)
          project_sewing<true>(off + k, a.sew_ids, a.sew_rest, a.x4, a.p4, a.slam, dts, a.sw);
        if (!grid_sync(a.bar, a.expected, a.spin_limit)) return;
      }
    if (a.with_update) {
      for (uint32_t i = tid; i < a.n; i += stride) update_vertex<true>(i, a.x4, a.p4, a.v4, dts);
      if (!grid_sync(a.bar, a.expected, a.spin_limit)) return;
    }
  }
}

// ---------------------------------------------------------------------
// cluster solver for batched instances
// ---------------------------------------------------------------------
// Instances share no vertex, so a thread-block cluster can own a bin of
// whole instances (a contiguous vertex range) and run the complete frame on
// it, separating colour steps with the cluster barrier instead of a grid
// barrier or a kernel launch.  Constraints are visited through a permutation
// sorted by (bin, colour): every constraint still runs the same device
// function in its colour step, and constraints of one colour share no vertex,
// so the results are the bits of the one-launch-per-colour path.  Loads of
// data that other CTAs write go around L1 (ld.global.cg).
struct ClusterTables {
  const uint2* vrange;     // [bins] vertex range [x, y)
  const uint2* pins;       // [bins] (first, count) into pin_v / pin_t
  const uint2* dist;       // [bins * ndc] (first, count) into dist_perm
  const uint2* bend;       // [bins * nbc] (first, count) into bend_perm
  const uint32_t* dist_perm;
  const uint32_t* bend_perm;
};
template <bool kBone>
__global__ void __launch_bounds__(256) k_solver_cluster(SolverArgs a, ClusterTables t) {
  cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
  const uint32_t bin = blockIdx.x / cl.dim_blocks().x;
  const uint32_t tid = cl.block_rank() * blockDim.x + threadIdx.x;
  const uint32_t stride = cl.num_blocks() * blockDim.x;
  const float dts = a.sp.dt;
  const uint2 vr = t.vrange[bin], pr = t.pins[bin];
  // the bin's constraints are contiguous in the permutations across colours
  const uint32_t d0 = a.ndc ? t.dist[bin * a.ndc].x : 0u;
  const uint32_t d1 = a.ndc ? t.dist[bin * a.ndc + a.ndc - 1].x + t.dist[bin * a.ndc + a.ndc - 1].y : 0u;
  const uint32_t b0 = a.nbc ? t.bend[bin * a.nbc].x : 0u;
  const uint32_t b1 = a.nbc ? t.bend[bin * a.nbc + a.nbc - 1].x + t.bend[bin * a.nbc + a.nbc - 1].y : 0u;
  for (uint32_t sub = 0; sub < a.nsub; ++sub) {
    for (uint32_t k = d0 + tid; k < d1; k += stride) a.dlam[t.dist_perm[k]] = 0.f;
    for (uint32_t k = b0 + tid; k < b1; k += stride) a.blam[t.bend_perm[k]] = 0.f;
    for (uint32_t i = vr.x + tid; i < vr.y; i += stride) predict_vertex<true>(i, a.x4, a.p4, a.v4, a.sp);
    cl.sync();
    for (uint32_t it = 0; it < a.iters; ++it) {
      if (pr.y) {
        for (uint32_t k = pr.x + tid; k < pr.x + pr.y; k += stride) pin_one<true>(k, a.pin_v, a.pin_t, a.x4, a.p4, dts);
        cl.sync();
      }
      for (uint32_t c = 0; c < a.ndc; ++c) {
        const uint2 r = t.dist[bin * a.ndc + c];
        if (!r.y) continue;
        for (uint32_t k = r.x + tid; k < r.x + r.y; k += stride)
          project_distance<true>(t.dist_perm[k], a.dist_ids, a.dist_par, a.x4, a.p4, a.dlam, a.sp, a.ddamp);
        cl.sync();
      }
      for (uint32_t c = 0; c < a.nbc; ++c) {
        const uint2 r = t.bend[bin * a.nbc + c];
        if (!r.y) continue;
        for (uint32_t k = r.x + tid; k < r.x + r.y; k += stride)
          project_bending<true>(t.bend_perm[k], a.bend_ids, a.bend_par, a.x4, a.p4, a.blam, a.sp, a.bdamp);
        cl.sync();
      }
      if (a.hascol && a.coupled) {
        for (uint32_t i = vr.x + tid; i < vr.y; i += stride) collide_vertex<true, kBone>(i, a.x4, a.p4, a.ca, dts);
        cl.sync();
      }
    }
    if (a.hascol && !a.coupled) {
      for (uint32_t i = vr.x + tid; i < vr.y; i += stride) collide_vertex<true, kBone>(i, a.x4, a.p4, a.ca, dts);
      cl.sync();
    }
    if (pr.y) {
      for (uint32_t k = pr.x + tid; k < pr.x + pr.y; k += stride) pin_one<true>(k, a.pin_v, a.pin_t, a.x4, a.p4, dts);
      cl.sync();
    }
    for (uint32_t i = vr.x + tid; i < vr.y; i += stride) update_vertex<true>(i, a.x4, a.p4, a.v4, dts);
    cl.sync();
  }
}


// ---------------------------------------------------------------------
// staged cluster solver for batched instances
// ---------------------------------------------------------------------
// The bins of the cluster solver with their vertex records on chip for the
// whole frame.  A bin's vertex range is split into K contiguous slices, one
// per CTA of the cluster; each CTA keeps its slice's x4, p4 and v4 records
// in shared memory.  A constraint reads and writes its two (bending: four)
// vertices in their owners' slices, its own CTA's directly and the others'
// through distributed shared memory, so the colour steps touch no global
// vertex data and are separated only by the cluster barrier.  Each (bin,
// colour) constraint range is split by the owner of the constraint's first
// vertex, so most accesses stay in the CTA.  Per-vertex passes (predict,
// pins, collision, velocity update) run on the owner's slice.  The
// per-element functions and the colour order are those of the other paths,
// so the results are the same bits.
struct SMem {
  static constexpr bool kCg = false;  // constraint lambdas: written and read by the same thread
  float4* sx;
  float4* sp;
  float4* sv;
  uint32_t base, chunk, rank;
  __device__ __forceinline__ float4* at(float4* a, uint32_t i) const {
    const uint32_t o = i - base;
    const uint32_t r = o / chunk;
    float4* q = a + (o - r * chunk);
    return r == rank ? q : cooperative_groups::this_cluster().map_shared_rank(q, r);
  }
  __device__ __forceinline__ float4 ldx(uint32_t i) const { return *at(sx, i); }
  __device__ __forceinline__ float4 ldp(uint32_t i) const { return *at(sp, i); }
  __device__ __forceinline__ float4 ldv(uint32_t i) const { return *at(sv, i); }
  __device__ __forceinline__ void stx(uint32_t i, float4 v) const { *at(sx, i) = v; }
  __device__ __forceinline__ void stp(uint32_t i, float4 v) const { *at(sp, i) = v; }
  __device__ __forceinline__ void stv(uint32_t i, float4 v) const { *at(sv, i) = v; }
};
// The constraint records are copied into staged arrays in (bin, colour,
// owner) order, so a colour step reads them coalesced without an index
// indirection; the staged lambdas are the solver's lambdas in that order
// (cleared every substep, read and written only by their own constraint).
// The same slices addressed by staged vertex ids (owner rank << 16 | slot in
// the owner's slice), which the staged constraint records carry: no division
// per access.
struct SMemE {
  static constexpr bool kCg = false;
  float4* sx;
  float4* sp;
  uint32_t rank;
  __device__ __forceinline__ float4* at(float4* a, uint32_t id) const {
    const uint32_t r = id >> 16;
    float4* q = a + (id & 0xFFFFu);
    return r == rank ? q : cooperative_groups::this_cluster().map_shared_rank(q, r);
  }
  __device__ __forceinline__ float4 ldx(uint32_t i) const { return *at(sx, i); }
  __device__ __forceinline__ float4 ldp(uint32_t i) const { return *at(sp, i); }
  __device__ __forceinline__ void stx(uint32_t i, float4 v) const { *at(sx, i) = v; }
  __device__ __forceinline__ void stp(uint32_t i, float4 v) const { *at(sp, i) = v; }
};
struct StageTables {
  const uint2* vrange;        // [bins] vertex range [x, y)
  const uint2* pins;          // [bins * K] (first, count) into pin_v / pin_t, by owning slice
  const uint32_t* dist;       // [bins * ndc * (K + 1)] offsets into the staged distance arrays
  const uint32_t* bend;       // [bins * nbc * (K + 1)]
  const uint2* dist_ids;      // staged records (vertex ids as staged ids, see SMemE) and lambdas
  const float4* dist_par;
  float* dist_lam;
  const uint4* bend_ids;
  const float4* bend_par;
  float* bend_lam;
  uint32_t cap;               // vertices per slice (the shared-memory capacity)
};
// gather of the staged records: out[k] = in[perm[k]]
template <class T>
__global__ void k_stage_gather(uint32_t cnt, const uint32_t* __restrict__ perm, const T* __restrict__ in,
                               T* __restrict__ out) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < cnt) out[k] = in[perm[k]];
}
// Records of a colour step held one step ahead: the first kStagePf
// constraints of this thread in the colour (k = lo + tid + q * blockDim).
constexpr int kStagePf = 2;
template <class Id>
struct StageBuf {
  Id e[kStagePf];
  float4 c[kStagePf];
  float l[kStagePf];
};
template <class Id>
__device__ __forceinline__ void stage_fetch(StageBuf<Id>& b, uint32_t lo, uint32_t hi, const Id* ids,
                                            const float4* par, const float* lam) {
#pragma unroll
  for (int q = 0; q < kStagePf; ++q) {
    const uint32_t k = lo + threadIdx.x + uint32_t(q) * blockDim.x;
    if (k < hi) {
      b.e[q] = ids[k];
      b.c[q] = par[k];
      b.l[q] = lam[k];
    }
  }
}
template <uint32_t K, bool kBone>
__global__ void __launch_bounds__(512, 1) k_solver_staged(SolverArgs a, StageTables t) {
  cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
  extern __shared__ float4 stage[];
  const uint32_t rank = cl.block_rank();
  const uint32_t bin = blockIdx.x / K;
  const uint2 vr = t.vrange[bin];
  const uint32_t nv = vr.y - vr.x;
  const uint32_t chunk = nv > 0 ? (nv + K - 1) / K : 1u;
  const SMem m{stage, stage + t.cap, stage + 2 * t.cap, vr.x, chunk, rank};
  const SMemE me{stage, stage + t.cap, rank};
  const uint32_t lo = vr.x + min(rank * chunk, nv), hi = vr.x + min((rank + 1u) * chunk, nv);
  for (uint32_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
    m.sx[i - lo] = a.x4[i];
    m.sp[i - lo] = a.p4[i];
    m.sv[i - lo] = a.v4[i];
  }
  const uint2 pr = t.pins[bin * K + rank];
  const uint32_t* dtab = t.dist + size_t(bin) * a.ndc * (K + 1u);
  const uint32_t* btab = t.bend + size_t(bin) * a.nbc * (K + 1u);
  const float dts = a.sp.dt;
  for (uint32_t sub = 0; sub < a.nsub; ++sub) {
    // each CTA clears the lambdas of its own constraints (which only it reads)
    for (uint32_t c = 0; c < a.ndc; ++c)
      for (uint32_t k = dtab[c * (K + 1u) + rank] + threadIdx.x; k < dtab[c * (K + 1u) + rank + 1u]; k += blockDim.x)
        t.dist_lam[k] = 0.f;
    for (uint32_t c = 0; c < a.nbc; ++c)
      for (uint32_t k = btab[c * (K + 1u) + rank] + threadIdx.x; k < btab[c * (K + 1u) + rank + 1u]; k += blockDim.x)
        t.bend_lam[k] = 0.f;
    for (uint32_t i = lo + threadIdx.x; i < hi; i += blockDim.x) predict_vertex_m(i, m, a.sp);
    cl.sync();
    for (uint32_t it = 0; it < a.iters; ++it) {
      if (a.npins) {
        for (uint32_t k = pr.x + threadIdx.x; k < pr.x + pr.y; k += blockDim.x) pin_one_m(k, a.pin_v, a.pin_t, m, dts);
        cl.sync();
      }
      // colour steps; each loads the next colour's first records before its
      // own work, so their latency overlaps the work and the barrier
      if (a.ndc) {
        StageBuf<uint2> cur, nxt;
        stage_fetch(cur, dtab[rank], dtab[rank + 1u], t.dist_ids, t.dist_par, t.dist_lam);
        for (uint32_t c = 0; c < a.ndc; ++c) {
          const uint32_t* r = dtab + c * (K + 1u);
          if (c + 1u < a.ndc)
            stage_fetch(nxt, r[K + 1u + rank], r[K + 2u + rank], t.dist_ids, t.dist_par, t.dist_lam);
          if (r[0] != r[K]) {  // the bin has constraints of this colour (same test in every CTA)
            const uint32_t lo = r[rank], hi = r[rank + 1u];
#pragma unroll
            for (int q = 0; q < kStagePf; ++q) {
              const uint32_t k = lo + threadIdx.x + uint32_t(q) * blockDim.x;
              if (k < hi) distance_core(cur.e[q], cur.c[q], cur.l[q], t.dist_lam + k, me, a.sp, a.ddamp);
            }
            for (uint32_t k = lo + threadIdx.x + kStagePf * blockDim.x; k < hi; k += blockDim.x)
              distance_core(t.dist_ids[k], t.dist_par[k], t.dist_lam[k], t.dist_lam + k, me, a.sp, a.ddamp);
            cl.sync();
          }
          cur = nxt;
        }
      }
      if (a.nbc) {
        StageBuf<uint4> cur, nxt;
        stage_fetch(cur, btab[rank], btab[rank + 1u], t.bend_ids, t.bend_par, t.bend_lam);
        for (uint32_t c = 0; c < a.nbc; ++c) {
          const uint32_t* r = btab + c * (K + 1u);
          if (c + 1u < a.nbc)
            stage_fetch(nxt, r[K + 1u + rank], r[K + 2u + rank], t.bend_ids, t.bend_par, t.bend_lam);
          if (r[0] != r[K]) {
            const uint32_t lo = r[rank], hi = r[rank + 1u];
#pragma unroll
            for (int q = 0; q < kStagePf; ++q) {
              const uint32_t k = lo + threadIdx.x + uint32_t(q) * blockDim.x;
              if (k < hi) bending_core(cur.e[q], cur.c[q], cur.l[q], t.bend_lam + k, me, a.sp, a.bdamp);
            }
            for (uint32_t k = lo + threadIdx.x + kStagePf * blockDim.x; k < hi; k += blockDim.x)
              bending_core(t.bend_ids[k], t.bend_par[k], t.bend_lam[k], t.bend_lam + k, me, a.sp, a.bdamp);
            cl.sync();
          }
          cur = nxt;
        }
      }
      if (a.hascol && a.coupled) {
        for (uint32_t i = lo + threadIdx.x; i < hi; i += blockDim.x) collide_vertex_m<kBone>(i, m, a.ca, dts);
        cl.sync();
      }
    }
    // the rest of the substep touches only the CTA's own slice
    if (a.hascol && !a.coupled)
      for (uint32_t i = lo + threadIdx.x; i < hi; i += blockDim.x) collide_vertex_m<kBone>(i, m, a.ca, dts);
    __syncthreads();
    for (uint32_t k = pr.x + threadIdx.x; k < pr.x + pr.y; k += blockDim.x) pin_one_m(k, a.pin_v, a.pin_t, m, dts);
    __syncthreads();
    for (uint32_t i = lo + threadIdx.x; i < hi; i += blockDim.x) update_vertex_m(i, m, dts);
    cl.sync();
  }
  for (uint32_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
    a.x4[i] = m.sx[i - lo];
    a.p4[i] = m.sp[i - lo];
    a.v4[i] = m.sv[i - lo];
  }
}

}  // namespace tcloth
