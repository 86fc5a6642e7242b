// Contact-pair cache for self-collision (the reference's "Active Pair
// Caching", self-collision algorithm 1), off by default as in the reference.
//
// At the first substep of a frame one thread per vertex scans the 27
// neighbour cells of the vertex hash and keeps, per vertex, the quota
// (1..8) nearest vertex-triangle and edge-edge candidates inside a widened
// margin (safety margin plus a velocity horizon).  The lists are written to
// fixed vertex-major slots (vertex * quota + k, unused slots hold the
// sentinel 0xFFFFFFFF), so the narrow-phase kernels of every later substep
// run one thread per slot with no hash scan and no compaction.
//
// Kernels:
//   k_pair_collect  shaders/self_collision_collect_pairs.wgsl:293-661
//   k_pair_vt       shaders/self_collision_solve_vt.wgsl:227-414
//   k_pair_ee       shaders/self_collision_solve_ee.wgsl:230-589
// Contacts go through the same integer accumulators as the direct path
// (add_disp / add_pin / add_ccd), so they are order-free.  A top-K list keeps
// the K smallest distinct keys under the total order (distance, key), so the
// stored pairs do not depend on the scan order either; only the evaluation
// and drop counters count in scan order (cell order, then the canonical
// in-bucket order of the hash).
#pragma once
#include "selfcol_kernels.cuh"

namespace tcloth {

constexpr uint32_t kPairQuotaMax = 8;  // PAIR_QUOTA_MAX, simulation/mod.rs
constexpr uint32_t kPairSentinel = 0xFFFFFFFFu;

struct PairArgs {
  float safety;       // safety_margin
  float dt_frame;     // frame dt for the velocity horizon
  float hscale;       // velocity_horizon_scale
  float max_h;        // max_horizon
  uint32_t margin_mode;  // 0 fixed, 1 velocity horizon
  uint32_t quota_vt, quota_ee;
  const uint32_t* island;
  float* hz;          // per-vertex horizon x mode (k_pair_horizon)
  uint4* vt;          // n * quota_vt slots (vert_i, c0, c1, c2)
  uint4* ee;          // n * quota_ee slots (v_i, v_ui, c_j, c_vj)
  uint32_t* counters; // vt_count, ee_count, vt_dropped, ee_dropped
};

// |floor(a) - floor(b)| > 1 on one axis, with the two's-complement wrap and
// the abs(INT_MIN) = INT_MIN rule of 32-bit integer vectors
__device__ __forceinline__ bool pc_far_axis(int32_t a, int32_t b) {
  const uint32_t d = (uint32_t)a - (uint32_t)b;
  const uint32_t ad = ((int32_t)d < 0) ? 0u - d : d;
  return (int32_t)ad > 1;
}

__device__ __forceinline__ float pc_horizon(const PairArgs& a, float4 v) {
  return fminf(length(mk(v)) * a.dt_frame * a.hscale, a.max_h);
}

// Per-vertex velocity horizon times the margin mode, the term every bound of
// the broad phase adds per vertex (collect_pairs.wgsl:328-330, :354-360,
// :277-278): min(|v| dt_frame scale, max_horizon) * mode.
__global__ void k_pair_horizon(uint32_t n, const float4* __restrict__ v4, PairArgs a) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  a.hz[i] = pc_horizon(a, v4[i]) * (float)a.margin_mode;
}

// can_ee_anchor_reach (self_collision_collect_pairs.wgsl:262-283); the cells
// are the hash pass's floor(p / cell) of the same positions
__device__ __forceinline__ bool pc_anchor_reach(const SCArgs& s, const PairArgs& a, uint32_t u, uint32_t w) {
  if (s.x4[u].w <= 0.0f) return false;
  const int4 cu = s.vcell[u], cw = s.vcell[w];
  if (pc_far_axis(cu.x, cw.x) || pc_far_axis(cu.y, cw.y) || pc_far_axis(cu.z, cw.z)) return false;
  const float4 pu = s.p4[u], pw = s.p4[w];
  const V3 d = mk(pu) - mk(pw);
  const float d2 = dot(d, d);
  const float b = pu.w + pw.w + (s.local_len[u] + s.local_len[w]) * 1.3f + a.safety + a.hz[u] + a.hz[w];
  if (d2 > b * b) return false;
  if (a.island[u] == a.island[w] && s.exclude_neighbors) {
    if (near_folded(s, u, w, sqrtf(fmaxf(d2, 0.0f)))) return false;
  }
  return true;
}
// is_smaller_anchor_reachable (:286-292): anchor (u, w) before (cu, cw) in
// lexicographic order, and reachable
__device__ __forceinline__ bool pc_lex_lt(uint32_t u, uint32_t w, uint32_t cu, uint32_t cw) {
  return !(u > cu || (u == cu && w >= cw));
}
__device__ __forceinline__ bool pc_smaller_anchor(const SCArgs& s, const PairArgs& a, uint32_t u, uint32_t w,
                                                  uint32_t cu, uint32_t cw) {
  return pc_lex_lt(u, w, cu, cw) && pc_anchor_reach(s, a, u, w);
}

__device__ __forceinline__ bool key_lt(uint3 a, uint3 b) {
  return a.x < b.x || (a.x == b.x && (a.y < b.y || (a.y == b.y && a.z < b.z)));
}

// Per-vertex top-K (distance ascending, then key), with duplicate keys
// rejected (collect_pairs.wgsl:428-475, :558-604).  Fixed-bound loops keep
// the lists in registers.
struct TopK {
  uint32_t n, eval, drop;
  float d[kPairQuotaMax];
  uint3 k[kPairQuotaMax];
};
__device__ __forceinline__ void topk_init(TopK& t) {
  t.n = t.eval = t.drop = 0u;
#pragma unroll
  for (int q = 0; q < (int)kPairQuotaMax; ++q) { t.d[q] = 0.0f; t.k[q] = make_uint3(0u, 0u, 0u); }
}
__device__ __forceinline__ bool topk_has(const TopK& t, uint3 key) {
  bool f = false;
#pragma unroll
  for (uint32_t q = 0; q < kPairQuotaMax; ++q)
    if (q < t.n && t.k[q].x == key.x && t.k[q].y == key.y && t.k[q].z == key.z) f = true;
  return f;
}
__device__ __forceinline__ void topk_insert(TopK& t, uint32_t quota, float d, uint3 key) {
  bool dup = false;
#pragma unroll
  for (uint32_t q = 0; q < kPairQuotaMax; ++q)
    if (q < t.n && t.k[q].x == key.x && t.k[q].y == key.y && t.k[q].z == key.z) dup = true;
  if (dup) return;
  ++t.eval;
  uint32_t pos = t.n;
  bool found = false;
#pragma unroll
  for (uint32_t q = 0; q < kPairQuotaMax; ++q) {
    if (!found && q < t.n) {
      const bool tie = (d == t.d[q]) && key_lt(key, t.k[q]);
      if (d < t.d[q] || tie) { pos = q; found = true; }
    }
  }
  if (pos < quota) {
    const uint32_t up = min(t.n, quota - 1u);
#pragma unroll
    for (uint32_t q = kPairQuotaMax - 1u; q >= 1u; --q)
      if (q <= up && q > pos) { t.d[q] = t.d[q - 1u]; t.k[q] = t.k[q - 1u]; }
#pragma unroll
    for (uint32_t q = 0; q < kPairQuotaMax; ++q)
      if (q == pos) { t.d[q] = d; t.k[q] = key; }
    if (t.n < quota) ++t.n;
  } else {
    ++t.drop;
  }
}

// ---------------- broad phase: self_collision_collect_pairs.wgsl:293-661
// Two launches over the same scan, one per list (kList 0: vertex-triangle,
// 1: edge-edge): each list and its counters see the reference's insertion
// sequence, and each launch holds one top-K in registers.
// Same visiting order and predicates as the reference; pure predicates are
// evaluated in a cheaper order, which changes no outcome:
// * candidates come from the hash pass's sorted records (p, thickness,
//   cell, index, local length, inverse mass);
// * a key already in the list is skipped before its distance is computed
//   (the insert would reject it as a duplicate);
// * the seven "smaller anchor" terms of an edge pair are split by what they
//   depend on: (j, index) once per j, (ui, j) and (j, ui) once per ui,
//   (index, vj) and (vj, index) once per j as a mask over vj, and only
//   (ui, vj) and (vj, ui) per pair; any true term skips the pair.
template <int kList>  // 0: vertex-triangle list, 1: edge-edge list
__global__ void __launch_bounds__(128) k_pair_collect(SCArgs s, PairArgs a) {
  // thread k takes the k-th vertex in hash order: the lanes of a warp share
  // cells and so walk the same candidates (each vertex's result does not
  // depend on which thread computes it)
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= s.n) return;
  const uint32_t index = s.srt[tid];
  const float4 xi4 = s.x4[index], pi4 = s.p4[index];
  const bool pin_i = xi4.w <= 0.0f;
  const V3 pi = mk(pi4);
  const float lli = s.local_len[index];
  const float thi = pi4.w;
  const int4 base = s.vcell[index];
  const uint32_t qvt = min(max(a.quota_vt, 1u), kPairQuotaMax);
  const uint32_t qee = min(max(a.quota_ee, 1u), kPairQuotaMax);
  const float margin = a.safety;
  const float hie = a.hz[index];
  const uint32_t isl_i = a.island[index];
  TopK vt, ee;
  topk_init(vt);
  topk_init(ee);
  // a pinned vertex collects no edge pairs (:525)
  const int gx0 = (kList == 1 && pin_i) ? 2 : -1;
  for (int gx = gx0; gx <= 1; ++gx)
    for (int gy = -1; gy <= 1; ++gy)
      for (int gz = -1; gz <= 1; ++gz) {
        const int32_t cx = base.x + gx, cy = base.y + gy, cz = base.z + gz;
        const uint32_t h = hash3(cx, cy, cz, s.table);
        const uint32_t b0 = s.cs[h], b1 = s.cs[h + 1];
        for (uint32_t k = b0; k < b1; ++k) {
          const int4 jc = s.vs_c[k];
          const uint32_t j = (uint32_t)jc.w;
          if (j >= s.n || j == index) continue;
          if (jc.x != cx || jc.y != cy || jc.z != cz) continue;
          const float4 q = s.vs_q[k];  // local length, layer, inverse mass, |p - x|
          const bool pin_j = q.z <= 0.0f;
          if (pin_i && pin_j) continue;
          const float4 pj4 = s.vs_p[k];
          const V3 pj = mk(pj4);
          const float hj = a.hz[j];
          const V3 dvv = pi - pj;
          const float d2vv = dot(dvv, dvv);
          const float eth = thi + pj4.w;
          const float llj = q.x;
          const float broad = eth + (lli + llj) * 1.3f + margin + hie + hj;
          if (!(d2vv <= broad * broad)) continue;
          const bool same_island = isl_i == a.island[j];
          if (same_island && s.exclude_neighbors && near_folded(s, index, j, sqrtf(fmaxf(d2vv, 0.0f)))) continue;
          const float check = eth + margin + hie + hj;
          // 1. vertex-triangle candidates over j's star (:380-476)
          if constexpr (kList == 0) {
          const float vtb = eth + llj * 1.3f + margin + hie + hj;
          const bool near2 = s.exclude_neighbors && within2(s, index, j);
          if (d2vv <= vtb * vtb && !near2) {
            const uint32_t ss0 = s.star_off[j], ss1 = s.star_off[j + 1];
            if (ss0 < ss1) {
              const uint32_t ns = min(ss1 - ss0, 8u);
              for (uint32_t t = 0; t < ns; ++t) {
                const uint2 pr = s.star_idx[ss0 + t];
                const uint32_t v0 = pr.x, v1 = pr.y;
                if (index == v0 || index == v1 || v0 >= s.n || v1 >= s.n) continue;
                // cyclic normalisation: smallest index first, winding kept
                uint32_t c0 = j, c1 = v0, c2 = v1;
                if (v0 < j && v0 < v1) { c0 = v0; c1 = v1; c2 = j; }
                else if (v1 < j && v1 < v0) { c0 = v1; c1 = j; c2 = v0; }
                const uint3 key = make_uint3(c0, c1, c2);
                if (topk_has(vt, key)) continue;
                bool isf;
                V3 bary;
                const V3 cp = closest_tri(pi, mk(s.p4[c0]), mk(s.p4[c1]), mk(s.p4[c2]), isf, bary);
                const V3 dvt = pi - cp;
                const float d2vt = dot(dvt, dvt);
                if (d2vt < check * check) {
                  if (s.exclude_neighbors && (within2(s, index, v0) || within2(s, index, v1))) continue;
                  topk_insert(vt, qvt, d2vt, key);
                }
              }
            }
          }
          continue;
          }
          // 2. edge-edge candidates over both one-rings (:478-612); only a
          // free vertex collects them
          if (pin_i) continue;
          const float eeb = eth + (lli + llj) * 1.3f + margin + hie + hj;
          if (!(d2vv <= eeb * eeb)) continue;
          const uint32_t ai0 = s.adj_off[index], ai1 = s.adj_off[index + 1];
          const uint32_t aj0 = s.adj_off[j], aj1 = s.adj_off[j + 1];
          if (!(ai0 < ai1 && aj0 < aj1)) continue;
          if (pc_smaller_anchor(s, a, j, index, index, j)) continue;
          const uint32_t nei = min(ai1 - ai0, 8u), nej = min(aj1 - aj0, 8u);
          uint32_t skipv = 0u;
          for (uint32_t e2 = 0; e2 < nej; ++e2) {
            const uint32_t vj = s.adj_idx[aj0 + e2];
            if (vj >= s.n) continue;
            if (pc_smaller_anchor(s, a, index, vj, index, j) || pc_smaller_anchor(s, a, vj, index, index, j))
              skipv |= 1u << e2;
          }
          for (uint32_t e1 = 0; e1 < nei; ++e1) {
            const uint32_t ui = s.adj_idx[ai0 + e1];
            if (ui >= s.n) continue;
            const V3 pui = mk(s.p4[ui]);
            const float llui = s.local_len[ui];
            const V3 li = pui - pi;
            const float lsi = dot(li, li);
            const float mli = (lli + llui) * 1.5f;
            if (lsi > mli * mli || lsi <= 1e-12f) continue;
            if (pc_smaller_anchor(s, a, ui, j, index, j) || pc_smaller_anchor(s, a, j, ui, index, j)) continue;
            for (uint32_t e2 = 0; e2 < nej; ++e2) {
              const uint32_t vj = s.adj_idx[aj0 + e2];
              if (vj >= s.n) continue;
              if (!(ui != j && ui != vj && index != vj)) continue;
              if ((skipv >> e2) & 1u) continue;
              const uint32_t cj = min(j, vj), cvj = max(j, vj);
              const uint3 key = make_uint3(ui, cj, cvj);
              if (topk_has(ee, key)) continue;
              const V3 pvj = mk(s.p4[vj]);
              const float llvj = s.local_len[vj];
              const V3 lj = pvj - pj;
              const float lsj = dot(lj, lj);
              const float mlj = (llj + llvj) * 1.5f;
              if (lsj > mlj * mlj || lsj <= 1e-12f) continue;
              if (pc_smaller_anchor(s, a, ui, vj, index, j) || pc_smaller_anchor(s, a, vj, ui, index, j)) continue;
              const V3 pcj = j < vj ? pj : pvj;
              const V3 pcvj = j < vj ? pvj : pj;
              float sp, tp;
              seg_seg(pi, pui, pcj, pcvj, sp, tp);
              const V3 pt1 = pi + (pui - pi) * sp;
              const V3 pt2 = pcj + (pcvj - pcj) * tp;
              const V3 dee = pt1 - pt2;
              const float d2ee = dot(dee, dee);
              if (d2ee < check * check && d2ee > kEps * kEps) {
                if (s.exclude_neighbors) {
                  if (near_folded(s, index, vj, length(pi - pvj)) || near_folded(s, ui, j, length(pui - pj)) ||
                      near_folded(s, ui, vj, length(pui - pvj)))
                    continue;
                }
                topk_insert(ee, qee, d2ee, key);
              }
            }
          }
        }
      }
  // vertex-major slots, sentinel-filled (:614-640)
  if constexpr (kList == 0) {
    const size_t bv = (size_t)index * qvt;
#pragma unroll
    for (uint32_t q = 0; q < kPairQuotaMax; ++q)
      if (q < qvt)
        a.vt[bv + q] = q < vt.n ? make_uint4(index, vt.k[q].x, vt.k[q].y, vt.k[q].z)
                                : make_uint4(kPairSentinel, 0u, 0u, 0u);
    if (vt.eval) atomicAdd(&a.counters[0], vt.eval);
    if (vt.drop) atomicAdd(&a.counters[2], vt.drop);
  } else {
    const size_t be = (size_t)index * qee;
#pragma unroll
    for (uint32_t q = 0; q < kPairQuotaMax; ++q)
      if (q < qee)
        a.ee[be + q] = q < ee.n ? make_uint4(index, ee.k[q].x, ee.k[q].y, ee.k[q].z)
                                : make_uint4(kPairSentinel, 0u, 0u, 0u);
    if (ee.eval) atomicAdd(&a.counters[1], ee.eval);
    if (ee.drop) atomicAdd(&a.counters[3], ee.drop);
  }
}

// record_untangle_cand (self_collision_solve_vt.wgsl:99-108): the nearest
// inner-layer vertex wins through an unsigned max of (rank << 22 | j + 1)
__device__ __forceinline__ void pc_untangle_cand(int32_t* acc, uint32_t n, uint32_t vi, uint32_t j, float dist,
                                                 float cap) {
  if (vi >= n || j >= 0x3FFFFEu || dist >= cap) return;
  const float ratio = clampf(dist / fmaxf(cap, kEps), 0.0f, 1.0f);
  const uint32_t rank = 1023u - (uint32_t)(ratio * 1023.0f);
  const uint32_t packed = (rank << 22) | ((j + 1u) & 0x3FFFFFu);
  atomicMax((uint32_t*)&acc[(size_t)vi * A_N + A_UT], packed);
}

// ---------------- narrow phase V-T: self_collision_solve_vt.wgsl:227-414
__global__ void __launch_bounds__(128) k_pair_vt(SCArgs s, PairArgs a, uint32_t slots) {
  const uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t n = s.n;
  if (n == 0u || slot >= slots) return;
  const uint4 pr = a.vt[slot];
  if (pr.x == kPairSentinel) return;
  const uint32_t index = pr.x, j = pr.y, v0 = pr.z, v1 = pr.w;
  if (index >= n || j >= n || v0 >= n || v1 >= n) return;
  if (index == j || index == v0 || index == v1 || v0 == v1 || j == v0 || j == v1) return;
  int32_t* acc = s.acc;
  const float4 xi4 = s.x4[index], pi4 = s.p4[index];
  const bool pin_i = xi4.w <= 0.0f;
  const V3 pi = mk(pi4), xo = mk(xi4);
  const float4 xj4 = s.x4[j], pj4 = s.p4[j];
  const float4 x04 = s.x4[v0], p04 = s.p4[v0];
  const float4 x14 = s.x4[v1], p14 = s.p4[v1];
  const V3 pj = mk(pj4), pv0 = mk(p04), pv1 = mk(p14);
  const V3 pjo = mk(xj4), pv0o = mk(x04), pv1o = mk(x14);
  const float wi = xi4.w, wj = xj4.w, wv0 = x04.w, wv1 = x14.w;
  const float eth = pi4.w + pj4.w;
  const V3 tmove = (((pj - pjo) + (pv0 - pv0o)) + (pv1 - pv1o)) / 3.0f;
  const bool tpin = (wj <= 0.0f) || (wv0 <= 0.0f) || (wv1 <= 0.0f);
  const bool upair = s.untangle && !pin_i && (layer_of(s.v4, index) > layer_of(s.v4, j));
  const V3 niraw = upair ? mk(s.nrm[index]) : mk(0.0f, 0.0f, 0.0f);
  const float nil = length(niraw);
  const V3 niu = nil > 0.5f ? niraw / fmaxf(nil, kEps) : mk(0.0f, 0.0f, 0.0f);
  const V3 rel = xo + tmove;
  float ht = 0.0f, hu = 0.0f, hv = 0.0f;
  if (seg_tri(rel, pi, pj, pv0, pv1, ht, hu, hv)) {
    // 1. trajectory CCD (:287-351)
    const V3 mv = pi - rel;
    const V3 hp = rel + mv * ht;
    const V3 tc = cross(pv0 - pj, pv1 - pj);
    const float tl = length(tc);
    const V3 tn = tl > 1e-12f ? tc / tl : mk(0.0f, 1.0f, 0.0f);
    const float hor = dot(rel - pj, tn);
    bool utc = false;
    if (upair && tl > 1e-12f) {
      const bool allow = tpin || (nil <= 0.5f) || (dot(niu, tn) > 0.0f);
      const bool ret = (hor < 0.0f) && (dot(mv, tn) > 0.0f);
      utc = allow && ret;
    }
    if (!utc) {
      const float ss = fabsf(hor) > 1e-6f ? hor : dot(-mv, tn);
      const V3 ns = ss >= 0.0f ? tn : -tn;
      const float ho = fmaxf(dot(rel - hp, ns), 0.0f);
      const float hs = fmaxf(ho, eth * 0.25f);
      const V3 psafe = hp + ns * hs;
      const V3 tccd = psafe - pi;
      const float pcs = fmaxf(0.0f, eth - hs);
      if (tpin) {
        if (!pin_i) add_ccd(acc, index, tccd + ns * pcs, false);
      } else if (pin_i) {
        const V3 bc = mk(clampf(1.0f - hu - hv, 0.0f, 1.0f), clampf(hu, 0.0f, 1.0f), clampf(hv, 0.0f, 1.0f));
        const float wt = bc.x * bc.x * wj + bc.y * bc.y * wv0 + bc.z * bc.z * wv1;
        if (wt > kEps) {
          const V3 full = tccd + ns * pcs;
          if (wj > 0.0f) add_ccd(acc, j, (-full) * (bc.x * wj / wt), false);
          if (wv0 > 0.0f) add_ccd(acc, v0, (-full) * (bc.y * wv0 / wt), false);
          if (wv1 > 0.0f) add_ccd(acc, v1, (-full) * (bc.z * wv1 / wt), false);
        }
      } else {
        const V3 bc = mk(clampf(1.0f - hu - hv, 0.0f, 1.0f), clampf(hu, 0.0f, 1.0f), clampf(hv, 0.0f, 1.0f));
        const float wt = bc.x * bc.x * wj + bc.y * bc.y * wv0 + bc.z * bc.z * wv1;
        const float wtot = wi + wt;
        if (wtot > kEps) {
          add_ccd(acc, index, tccd * (wi / wtot), false);
          if (wj > 0.0f) add_ccd(acc, j, (-tccd) * (bc.x * wj / wtot), false);
          if (wv0 > 0.0f) add_ccd(acc, v0, (-tccd) * (bc.y * wv0 / wtot), false);
          if (wv1 > 0.0f) add_ccd(acc, v1, (-tccd) * (bc.z * wv1 / wtot), false);
          if (pcs > kEps) {
            const V3 tp = ns * (pcs * 0.6f);
            add_disp(acc, index, tp * (wi / wtot));
            if (wj > 0.0f) add_disp(acc, j, (-tp) * (bc.x * wj / wtot));
            if (wv0 > 0.0f) add_disp(acc, v0, (-tp) * (bc.y * wv0 / wtot));
            if (wv1 > 0.0f) add_disp(acc, v1, (-tp) * (bc.z * wv1 / wtot));
          }
        }
      }
    } else {
      pc_untangle_cand(acc, n, index, j, length(pi - hp), eth * 2.5f);
    }
    return;
  }
  // 2. closest-point repulsion with barycentric reaction (:352-413)
  bool isf;
  V3 bary;
  const V3 cp = closest_tri(pi, pj, pv0, pv1, isf, bary);
  const V3 dvt = pi - cp;
  const float dist = length(dvt);
  const V3 tc = cross(pv0 - pj, pv1 - pj);
  const float tl = length(tc);
  const V3 tn = tl > kEps ? tc / fmaxf(tl, kEps) : mk(0.0f, 0.0f, 0.0f);
  const float hvt = tl > kEps ? dot(dvt, tn) : 0.0f;
  const bool allow = tpin || (nil <= 0.5f) || (dot(niu, tn) > 0.0f);
  const bool utv = upair && (tl > kEps) && allow && (hvt < 0.0f);
  if (utv) pc_untangle_cand(acc, n, index, j, dist, eth * 2.5f);
  if (!pin_i && !utv && dist < eth && dist > kEps) {
    const V3 nvt = dvt / dist;
    const float pen = eth - dist;
    if (tpin) {
      add_pin(acc, index, nvt * pen + tmove * 0.5f);
    } else {
      const float wt = bary.x * bary.x * wj + bary.y * bary.y * wv0 + bary.z * bary.z * wv1;
      const float wtot = wi + wt;
      if (wtot > kEps) {
        const V3 tp = nvt * (pen * 0.6f);
        add_disp(acc, index, tp * (wi / wtot));
        if (wj > 0.0f) add_disp(acc, j, (-tp) * (bary.x * wj / wtot));
        if (wv0 > 0.0f) add_disp(acc, v0, (-tp) * (bary.y * wv0 / wtot));
        if (wv1 > 0.0f) add_disp(acc, v1, (-tp) * (bary.z * wv1 / wtot));
      }
    }
  }
}

// ---------------- narrow phase E-E: self_collision_solve_ee.wgsl:230-589
__global__ void __launch_bounds__(128) k_pair_ee(SCArgs s, PairArgs a, uint32_t slots) {
  const uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t n = s.n;
  if (n == 0u || slot >= slots) return;
  const uint4 pr = a.ee[slot];
  if (pr.x == kPairSentinel) return;
  const uint32_t u0 = pr.x, u1 = pr.y, j = pr.z, vj = pr.w;
  if (u0 >= n || u1 >= n || j >= n || vj >= n) return;
  if (u0 == u1 || j == vj || u0 == j || u0 == vj || u1 == j || u1 == vj) return;
  int32_t* acc = s.acc;
  const float4 xa0 = s.x4[u0], xa1 = s.x4[u1], xb0 = s.x4[j], xb1 = s.x4[vj];
  const float4 pa0 = s.p4[u0], pa1 = s.p4[u1], pb0 = s.p4[j], pb1 = s.p4[vj];
  const float w_u0 = xa0.w, w_u1 = xa1.w, w_j = xb0.w, w_vj = xb1.w;
  const bool apin = (w_u0 <= 0.0f) || (w_u1 <= 0.0f);
  const bool bpin = (w_j <= 0.0f) || (w_vj <= 0.0f);
  if (apin && bpin) return;
  const V3 p_u0 = mk(pa0), p_u1 = mk(pa1), p_j = mk(pb0), p_vj = mk(pb1);
  const V3 p_u0o = mk(xa0), p_u1o = mk(xa1), p_jo = mk(xb0), p_vjo = mk(xb1);
  const float thu0 = pa0.w, thu1 = pa1.w, thj = pb0.w, thvj = pb1.w;
  // selective CCD gate and end-of-step closest points (:290-322)
  float s1, t1;
  seg_seg(p_u0, p_u1, p_j, p_vj, s1, t1);
  const V3 d1c = vmix(p_u0, p_u1, s1) - vmix(p_j, p_vj, t1);
  const float d2c = dot(d1c, d1c);
  const float eth = mixf(thu0, thu1, s1) + mixf(thj, thvj, t1);
  const float meth = fmaxf(thu0, thu1) + fmaxf(thj, thvj);
  const V3 dv0 = p_u0 - p_u0o, dv1 = p_u1 - p_u1o, dvj = p_j - p_jo, dvvj = p_vj - p_vjo;
  const V3 va = (dv0 + dv1) * 0.5f, vb = (dvj + dvvj) * 0.5f;
  const float rd = length(va - vb) + 0.5f * (length(dv1 - dv0) + length(dvvj - dvj));
  const float reach = meth + rd;
  if (d2c > reach * reach) return;
  const V3 d0g = vmix(p_u0o, p_u1o, s1) - vmix(p_jo, p_vjo, t1);
  const bool run_ccd = (rd > eth * 0.5f) || (dot(d0g, d1c) <= 0.0f);
  const uint32_t la = layer_of(s.v4, u0), lb = layer_of(s.v4, j);
  if (run_ccd) {
    float msd = 1e20f, btau = 0.0f, hs = 0.125f, ms = 0.f, mt = 0.f;
    float pv = seg_vol(p_u0o, p_u0, p_u1o, p_u1, p_jo, p_j, p_vjo, p_vj, 0.0f);
    float zc = -1.0f;
    for (uint32_t k = 0; k <= 8u; ++k) {
      const float tk = (float)k * 0.125f;
      float es, et;
      const float ed = seg_eval(p_u0o, p_u0, p_u1o, p_u1, p_jo, p_j, p_vjo, p_vj, tk, es, et);
      if (ed < msd) { msd = ed; btau = tk; ms = es; mt = et; }
      if (k > 0u) {
        const float vol = seg_vol(p_u0o, p_u0, p_u1o, p_u1, p_jo, p_j, p_vjo, p_vj, tk);
        if (pv * vol <= 0.0f && zc < 0.0f) zc = tk - 0.0625f;
        pv = vol;
      }
    }
    if (zc >= 0.0f) {
      float es, et;
      const float ed = seg_eval(p_u0o, p_u0, p_u1o, p_u1, p_jo, p_j, p_vjo, p_vj, zc, es, et);
      if (ed < msd) { msd = ed; btau = zc; hs = 0.0625f; ms = es; mt = et; }
    }
    float tlo = fmaxf(0.0f, btau - hs), thi = fminf(1.0f, btau + hs);
    float dstar = msd, ss = ms, ts = mt;
    for (int it = 0; it < 6; ++it) {
      const float m1 = tlo + (thi - tlo) * (1.0f / 3.0f);
      const float mm2 = thi - (thi - tlo) * (1.0f / 3.0f);
      float e1s, e1t, e2s, e2t;
      const float e1 = seg_eval(p_u0o, p_u0, p_u1o, p_u1, p_jo, p_j, p_vjo, p_vj, m1, e1s, e1t);
      const float e2 = seg_eval(p_u0o, p_u0, p_u1o, p_u1, p_jo, p_j, p_vjo, p_vj, mm2, e2s, e2t);
      if (e1 < dstar) { dstar = e1; ss = e1s; ts = e1t; }
      if (e2 < dstar) { dstar = e2; ss = e2s; ts = e2t; }
      if (e1 < e2) thi = mm2; else tlo = m1;
    }
    const float ets = mixf(thu0, thu1, ss) + mixf(thj, thvj, ts);
    if (dstar >= ets * ets) return;
    bool utc = false;
    if (s.untangle && la != lb) {
      const bool afx = (w_u0 == 0.0f) && (w_u1 == 0.0f);
      const bool bfx = (w_j == 0.0f) && (w_vj == 0.0f);
      const V3 d0u = ((p_u0o + p_u1o) - (p_jo + p_vjo)) * 0.5f;
      const V3 d1u = ((p_u0 + p_u1) - (p_j + p_vj)) * 0.5f;
      const V3 mu = d1u - d0u;
      if (la > lb && !afx) {
        const V3 ni = mk(s.nrm[j]), no = mk(s.nrm[u0]);
        const bool allow = bfx || (dot(no, no) <= 0.25f);
        utc = allow && (dot(ni, ni) > 0.25f) && (dot(d0u, ni) < 0.0f) && (dot(mu, ni) > 0.0f);
      } else if (lb > la && !bfx) {
        const V3 ni = mk(s.nrm[u0]), no = mk(s.nrm[j]);
        const bool allow = afx || (dot(no, no) <= 0.25f);
        utc = allow && (dot(ni, ni) > 0.25f) && (dot(-d0u, ni) < 0.0f) && (dot(-mu, ni) > 0.0f);
      }
    }
    if (utc) return;
    float s0, t0p;
    seg_seg(p_u0o, p_u1o, p_jo, p_vjo, s0, t0p);
    const V3 d0 = vmix(p_u0o, p_u1o, s0) - vmix(p_jo, p_vjo, t0p);
    const float dist0 = length(d0);
    if (dist0 > kEps) {
      const V3 n0 = d0 / dist0;
      const V3 de = vmix(p_u0, p_u1, ss) - vmix(p_j, p_vj, ts);
      const float he = dot(de, n0);
      const bool crossed = (he <= 0.0f) || (dot(d1c, n0) <= 0.0f);
      if (he < ets && crossed) {
        const float pc = ets - he;
        const bool aall = (w_u0 == 0.0f) && (w_u1 == 0.0f);
        const bool ball = (w_j == 0.0f) && (w_vj == 0.0f);
        const bool cpe = !(aall || ball);
        if (bpin) {
          const V3 em = ((p_j - p_jo) + (p_vj - p_vjo)) * 0.5f;
          const float aa = 1.0f - ss, bb = ss;
          const float den = aa * aa * w_u0 + bb * bb * w_u1;
          if (den > kEps) {
            const V3 pb = n0 * pc + em * 0.5f;
            if (w_u0 > 0.0f) add_ccd(acc, u0, pb * fminf((aa * w_u0) / den, 2.0f), cpe);
            if (w_u1 > 0.0f) add_ccd(acc, u1, pb * fminf((bb * w_u1) / den, 2.0f), cpe);
          }
        } else if (apin) {
          const V3 em = ((p_u0 - p_u0o) + (p_u1 - p_u1o)) * 0.5f;
          const float aa = 1.0f - ts, bb = ts;
          const float den = aa * aa * w_j + bb * bb * w_vj;
          if (den > kEps) {
            const V3 pb = (-n0) * pc + em * 0.5f;
            if (w_j > 0.0f) add_ccd(acc, j, pb * fminf((aa * w_j) / den, 2.0f), cpe);
            if (w_vj > 0.0f) add_ccd(acc, vj, pb * fminf((bb * w_vj) / den, 2.0f), cpe);
          }
        } else {
          const float we1 = (1.0f - ss) * (1.0f - ss) * w_u0 + ss * ss * w_u1;
          const float we2 = (1.0f - ts) * (1.0f - ts) * w_j + ts * ts * w_vj;
          const float wtot = we1 + we2;
          if (wtot > kEps) {
            const V3 tcc = n0 * pc;
            if (w_u0 > 0.0f) add_ccd(acc, u0, tcc * ((1.0f - ss) * w_u0 / wtot), true);
            if (w_u1 > 0.0f) add_ccd(acc, u1, tcc * (ss * w_u1 / wtot), true);
            if (w_j > 0.0f) add_ccd(acc, j, (-tcc) * ((1.0f - ts) * w_j / wtot), true);
            if (w_vj > 0.0f) add_ccd(acc, vj, (-tcc) * (ts * w_vj / wtot), true);
          }
        }
        return;
      }
    }
  }
  // discrete segment repulsion (:495-588)
  if (d2c >= eth * eth || d2c <= kEps * kEps) return;
  const float del = sqrtf(d2c);
  bool ute = false;
  if (s.untangle) {
    const bool afx = (w_u0 <= 0.0f) && (w_u1 <= 0.0f);
    const bool bfx = (w_j <= 0.0f) && (w_vj <= 0.0f);
    ute = outer_behind(s, la, lb, u0, u1, j, vj, afx, bfx, d1c);
  }
  if (ute) return;
  const V3 ne = d1c / del;
  const float pen = eth - del;
  if (bpin) {
    const V3 em = ((p_j - p_jo) + (p_vj - p_vjo)) * 0.5f;
    const float aa = 1.0f - s1, bb = s1;
    const float den = aa * aa * w_u0 + bb * bb * w_u1;
    if (den > kEps) {
      const V3 pb = ne * pen + em * 0.5f;
      if (w_u0 > 0.0f) add_pin(acc, u0, pb * fminf((aa * w_u0) / den, 2.0f));
      if (w_u1 > 0.0f) add_pin(acc, u1, pb * fminf((bb * w_u1) / den, 2.0f));
    }
  } else if (apin) {
    const V3 em = ((p_u0 - p_u0o) + (p_u1 - p_u1o)) * 0.5f;
    const float aa = 1.0f - t1, bb = t1;
    const float den = aa * aa * w_j + bb * bb * w_vj;
    if (den > kEps) {
      const V3 pb = (-ne) * pen + em * 0.5f;
      if (w_j > 0.0f) add_pin(acc, j, pb * fminf((aa * w_j) / den, 2.0f));
      if (w_vj > 0.0f) add_pin(acc, vj, pb * fminf((bb * w_vj) / den, 2.0f));
    }
  } else {
    const float we1 = (1.0f - s1) * (1.0f - s1) * w_u0 + s1 * s1 * w_u1;
    const float we2 = (1.0f - t1) * (1.0f - t1) * w_j + t1 * t1 * w_vj;
    const float wtot = we1 + we2;
    if (wtot > kEps) {
      const V3 td = ne * (pen * 0.6f);
      if (w_u0 > 0.0f) add_disp(acc, u0, td * ((1.0f - s1) * w_u0 / wtot));
      if (w_u1 > 0.0f) add_disp(acc, u1, td * (s1 * w_u1 / wtot));
      if (w_j > 0.0f) add_disp(acc, j, (-td) * ((1.0f - t1) * w_j / wtot));
      if (w_vj > 0.0f) add_disp(acc, vj, (-td) * (t1 * w_vj / wtot));
    }
  }
}

}  // namespace tcloth
