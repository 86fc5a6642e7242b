// Self-collision kernels: area-weighted normals, the spatial-hash counting
// sort (vertex and edge-midpoint keys), vertex-vertex / vertex-triangle
// contacts, multi-layer untangling, edge-edge contacts and the apply pass.
//
// Contacts accumulate into a per-vertex 16 x int32 record with integer
// atomics (fixed point x1e6), so results do not depend on thread order.
// The one order-dependent piece of the reference, the in-bucket order of the
// counting sort (atomic scatter, shaders/spatial_grid_sort.wgsl:182-194), is
// made canonical here: each bucket is sorted by ascending element index.
#pragma once
#include "vmath.cuh"

namespace tcloth {

enum : int {
  A_DX, A_DY, A_DZ, A_CNT, A_PDX, A_PDY, A_PDZ, A_PCNT,
  A_CPX, A_CPY, A_CPZ, A_CNX, A_CNY, A_CNZ, A_UT, A_EEC, A_N
};

struct SCArgs {
  uint32_t n, ne, table;
  float cell;
  float relief;
  int enable_relief;
  float max_disp_ratio;
  int exclude_neighbors;
  int untangle;  // effective: option && multiple layers
  uint32_t max_search;
  const float4* x4;
  const float4* p4;
  const float4* v4;  // layer bits in .w
  const float* local_len;
  const uint32_t* adj_off;
  const uint32_t* adj_idx;
  const uint32_t* th_off;
  const uint32_t* th_idx;
  const float* th_rest;
  const uint32_t* star_off;
  const uint2* star_idx;
  const uint2* edges;
  const uint32_t* edge_bits;
  const uint32_t* cs;    // vertex cell starts (table + 1)
  const uint32_t* srt;   // vertex sorted indices
  const uint32_t* ecs;   // edge cell starts
  const uint32_t* esrt;  // edge sorted indices
  const float4* nrm;
  int32_t* acc;
  // per-substep caches written by the hash pass (same float operations as
  // the reference performs per candidate, done once per element)
  // per vertex j: bounding box of p over j and its star triangles' vertices,
  // and the range of their motion p - x: (lo, mlo.x), (hi, mlo.y), (mhi, mlo.z)
  const float4* sbox;
  const int4* vcell;    // floor(p / cell) per vertex
  const float* mlen;    // |p - x| per vertex
  const int4* ecell;    // floor(midpoint / cell) per edge
  const float4* eamin;  // min of both endpoints' p and x per edge
  const float4* eamax;
  // candidate records in hash-sorted order (slot k of the sorted arrays)
  const float4* vs_p;   // p, thickness of vertex srt[k]
  const int4* vs_c;     // cell, index of vertex srt[k]
  const float4* vs_q;   // local edge length, layer bits, inverse mass, |p - x| of vertex srt[k]
  const int4* es_c;     // cell, index of edge esrt[k]
  const uint2* es_v;    // endpoints of edge esrt[k]
  const float4* es_lo;  // swept AABB of edge esrt[k]; .w: bits of its first endpoint
  const float4* es_hi;  // .w: bits of its second endpoint
  // pairs that need the continuous (CCD) search are deferred to k_ee_ccd
  uint2* ccd_q;
  uint32_t* ccd_n;
  uint32_t ccd_cap;
  // (edge, edge) pairs counted by k_ee, worked one lane each by k_ee_pairs.
  // The list is split into kEeSeg segments of ee_cap / kEeSeg entries with a
  // counter each (ee_n[kEeSeg]); block b of k_ee appends to segment
  // b % kEeSeg, so that no one counter takes every warp's atomic.  A counter
  // may run past its segment's capacity (k_ee_pairs reads min(count, cap));
  // the pairs past it are worked inside k_ee.  ee_cap = 0 keeps all of the
  // contact work inside k_ee.
  uint2* ee_q;
  uint32_t* ee_n;
  uint32_t ee_cap;
  // optional record of the narrow-phase input (null when off): the
  // (vertex, triangle) pairs that pass the cheap tests of sc_solve and the
  // (edge, edge) pairs counted within max_search; rec_n[0] / rec_n[1] count
  // them, entries past the capacities are dropped
  uint4* rec_vt;
  uint2* rec_ee;
  uint32_t* rec_n;
  uint32_t rec_vt_cap, rec_ee_cap;
};

__device__ __forceinline__ void record_vt(const SCArgs& s, uint32_t i, uint32_t a, uint32_t b, uint32_t c) {
  const uint32_t k = atomicAdd(&s.rec_n[0], 1u);
  if (k < s.rec_vt_cap) s.rec_vt[k] = make_uint4(i, a, b, c);
}
__device__ __forceinline__ void record_ee(const SCArgs& s, uint32_t ea, uint32_t eb) {
  const uint32_t k = atomicAdd(&s.rec_n[1], 1u);
  if (k < s.rec_ee_cap) s.rec_ee[k] = make_uint2(ea, eb);
}

// A vertex's sorted two-hop list (and rest lengths), in shared memory when it
// fits, else in global memory; binary search as in
// shaders/self_collision.wgsl:243-293.
struct TwoHop {
  const uint32_t* idx;
  const float* rest;
  uint32_t n;
};
__device__ __forceinline__ bool th_find(const TwoHop& t, uint32_t b, uint32_t& pos) {
  uint32_t lo = 0, hi = t.n;
  while (lo < hi) {
    const uint32_t mid = lo + (hi - lo) / 2u;
    const uint32_t v = t.idx[mid];
    if (v == b) { pos = mid; return true; }
    if (v < b) lo = mid + 1u; else hi = mid;
  }
  return false;
}
__device__ __forceinline__ bool within2_t(const TwoHop& t, uint32_t a, uint32_t b) {
  uint32_t q;
  if (a == b) return true;
  return th_find(t, b, q);
}
__device__ __forceinline__ bool near_folded_t(const TwoHop& t, uint32_t a, uint32_t b, float d) {
  uint32_t q;
  if (a == b) return true;
  if (!th_find(t, b, q)) return false;
  return !(d < t.rest[q] * 0.5f);
}
__device__ __forceinline__ bool near_folded_sq_t(const TwoHop& t, uint32_t a, uint32_t b, float d2) {
  uint32_t q;
  if (a == b) return true;
  if (!th_find(t, b, q)) return false;
  const float l0 = t.rest[q];
  return !(d2 < (l0 * l0) * 0.25f);
}
constexpr uint32_t kTwoHopCache = 64;
constexpr uint32_t kRounds = 4;  // candidates per warp chunk = 32 * kRounds
constexpr uint32_t kEeSeg = 256;       // segments of the E-E pair list
constexpr uint32_t kEePairBlocks = 4;  // k_ee_pairs blocks per segment
// Stage vertex v's two-hop list in shared memory (whole warp participates).
__device__ __forceinline__ TwoHop stage_two_hop(const uint32_t* th_off, const uint32_t* th_idx, const float* th_rest,
                                               uint32_t v, uint32_t* sh_idx, float* sh_rest, int lane) {
  const uint32_t b = th_off[v], e = th_off[v + 1];
  TwoHop t;
  t.n = e - b;
  if (t.n <= kTwoHopCache) {
    for (uint32_t k = lane; k < t.n; k += 32u) {
      sh_idx[k] = th_idx[b + k];
      sh_rest[k] = th_rest[b + k];
    }
    __syncwarp();
    t.idx = sh_idx;
    t.rest = sh_rest;
  } else {
    t.idx = th_idx + b;
    t.rest = th_rest + b;
  }
  return t;
}

__device__ __forceinline__ uint32_t layer_of(const float4* v4, uint32_t i) { return __float_as_uint(v4[i].w); }

// Star boxes for the vertex-triangle pass (see SCArgs::sbox): one thread per
// vertex over its star pairs.
__global__ void k_star_box(uint32_t n, const uint32_t* __restrict__ star_off, const uint2* __restrict__ star_idx,
                           const float4* __restrict__ x4, const float4* __restrict__ p4, float4* __restrict__ sbox) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const V3 pj = mk(p4[j]);
  V3 lo = pj, hi = pj, mlo = pj - mk(x4[j]), mhi = mlo;
  for (uint32_t k = star_off[j]; k < star_off[j + 1]; ++k) {
    const uint2 pr = star_idx[k];
    const V3 a = mk(p4[pr.x]), b = mk(p4[pr.y]);
    const V3 ma = a - mk(x4[pr.x]), mb = b - mk(x4[pr.y]);
    lo = vmin(lo, vmin(a, b));
    hi = vmax(hi, vmax(a, b));
    mlo = vmin(mlo, vmin(ma, mb));
    mhi = vmax(mhi, vmax(ma, mb));
  }
  sbox[3 * size_t(j)] = make_float4(lo.x, lo.y, lo.z, mlo.x);
  sbox[3 * size_t(j) + 1] = make_float4(hi.x, hi.y, hi.z, mlo.y);
  sbox[3 * size_t(j) + 2] = make_float4(mhi.x, mhi.y, mhi.z, mlo.z);
}

// ---------------- normals: shaders/compute_normals.wgsl:25-58
__global__ void k_normals(uint32_t n, const float4* __restrict__ x4, const uint32_t* __restrict__ star_off,
                          const uint2* __restrict__ star_idx, float4* __restrict__ nrm) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const V3 pi = mk(x4[i]);
  V3 s = mk(0.f, 0.f, 0.f);
  for (uint32_t k = star_off[i]; k < star_off[i + 1]; ++k) {
    const uint2 pr = star_idx[k];
    s = s + cross(mk(x4[pr.x]) - pi, mk(x4[pr.y]) - pi);
  }
  const float l = length(s);
  V3 r = l > kEps ? s / l : mk(0.f, 0.f, 0.f);
  nrm[i] = make_float4(r.x, r.y, r.z, 0.f);
}

// ---------------- spatial hash (spatial_hash.rs:158-247, spatial_grid_sort*.wgsl)
// which == 0: key of vertex i is its predicted position; which == 1: key of
// edge i is the midpoint of its two predicted endpoints.
__global__ void k_hash_count(uint32_t cnt, int which, const float4* __restrict__ x4, const float4* __restrict__ p4,
                             const uint2* __restrict__ edges, float cell, uint32_t table, uint32_t* __restrict__ keys,
                             uint32_t* __restrict__ counts, int4* __restrict__ cells, float* __restrict__ mlen,
                             float4* __restrict__ amin, float4* __restrict__ amax) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= cnt) return;
  V3 q;
  if (which == 0) {
    q = mk(p4[i]);
    mlen[i] = length(q - mk(x4[i]));
  } else {
    const uint2 e = edges[i];
    const V3 p0 = mk(p4[e.x]), p1 = mk(p4[e.y]);
    q = (p0 + p1) * 0.5f;
    const V3 lo = vmin(vmin(p0, p1), vmin(mk(x4[e.x]), mk(x4[e.y])));
    const V3 hi = vmax(vmax(p0, p1), vmax(mk(x4[e.x]), mk(x4[e.y])));
    amin[i] = make_float4(lo.x, lo.y, lo.z, 0.f);
    amax[i] = make_float4(hi.x, hi.y, hi.z, 0.f);
  }
  const I3 c = cell_of(q, cell);
  cells[i] = make_int4(c.x, c.y, c.z, 0);
  const uint32_t h = hash3(c.x, c.y, c.z, table);
  keys[i] = h;
  // warp-aggregated increment: lanes with the same bucket share one atomic
  const uint32_t active = __activemask();
  const uint32_t peers = __match_any_sync(active, h);
  const int leader = __ffs(peers) - 1;
  const int lane = threadIdx.x & 31;
  if (lane == leader) atomicAdd(&counts[h], __popc(peers));
}

// Exclusive scan of counts[table] into starts[table + 1] in two launches:
// k_scan_blocks scans 1024-entry tiles (coalesced loads, warp-shuffle scans)
// and writes tile totals; k_scan_finish adds the scanned tile totals.
__device__ __forceinline__ uint32_t block_incl_scan_1024(uint32_t v, uint32_t* warp_tot, uint32_t& total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  if (lane == 31) warp_tot[wid] = v;
  __syncthreads();
  if (wid == 0) {
    uint32_t w = warp_tot[lane];
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += t;
    }
    warp_tot[lane] = w;
  }
  __syncthreads();
  total = warp_tot[31];
  return v + (wid > 0 ? warp_tot[wid - 1] : 0u);
}
__global__ void __launch_bounds__(1024) k_scan_blocks(uint32_t table, const uint32_t* __restrict__ counts,
                                                      uint32_t* __restrict__ starts, uint32_t* __restrict__ tile_sum) {
  __shared__ uint32_t warp_tot[32];
  const uint32_t i = blockIdx.x * 1024u + threadIdx.x;
  const uint32_t c = i < table ? counts[i] : 0u;
  uint32_t total;
  const uint32_t incl = block_incl_scan_1024(c, warp_tot, total);
  if (i < table) starts[i] = incl - c;
  if (threadIdx.x == 0) tile_sum[blockIdx.x] = total;
}
__global__ void __launch_bounds__(1024) k_scan_finish(uint32_t table, uint32_t ntiles, const uint32_t* __restrict__ tile_sum,
                                                      uint32_t* __restrict__ starts) {
  __shared__ uint32_t tile_off[64];
  if (threadIdx.x < 64) {
    // ntiles <= 64 (table <= 65536): scan of tile sums by the first warp pair
    uint32_t v = threadIdx.x < ntiles ? tile_sum[threadIdx.x] : 0u;
    tile_off[threadIdx.x] = v;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t acc = 0;
    for (uint32_t t = 0; t < ntiles; ++t) { const uint32_t v = tile_off[t]; tile_off[t] = acc; acc += v; }
    starts[table] = acc;
  }
  __syncthreads();
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < table; i += gridDim.x * blockDim.x)
    starts[i] += tile_off[i >> 10];
}

__global__ void k_hash_scatter(uint32_t cnt, const uint32_t* __restrict__ keys, const uint32_t* __restrict__ starts,
                               uint32_t* __restrict__ cursor, uint32_t* __restrict__ sorted) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= cnt) return;
  const uint32_t h = keys[i];
  sorted[starts[h] + atomicAdd(&cursor[h], 1u)] = i;
}

// Candidate records in sorted order, so a warp scanning one bucket reads
// consecutive slots instead of chasing sorted index -> element -> data.
__global__ void k_gather_vertices(uint32_t n, const uint32_t* __restrict__ srt, const float4* __restrict__ x4,
                                  const float4* __restrict__ p4, const float4* __restrict__ v4,
                                  const float* __restrict__ local_len, const float* __restrict__ mlen,
                                  const int4* __restrict__ vcell, float4* __restrict__ vs_p, int4* __restrict__ vs_c,
                                  float4* __restrict__ vs_q) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const uint32_t j = srt[k];
  vs_p[k] = p4[j];
  const int4 c = vcell[j];
  vs_c[k] = make_int4(c.x, c.y, c.z, (int)j);
  vs_q[k] = make_float4(local_len[j], v4[j].w, x4[j].w, mlen[j]);
}
__global__ void k_gather_edges(uint32_t ne, const uint32_t* __restrict__ esrt, const uint2* __restrict__ edges,
                               const int4* __restrict__ ecell, const float4* __restrict__ amin,
                               const float4* __restrict__ amax, int4* __restrict__ es_c, uint2* __restrict__ es_v,
                               float4* __restrict__ es_lo, float4* __restrict__ es_hi) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ne) return;
  const uint32_t e = esrt[k];
  const int4 c = ecell[e];
  es_c[k] = make_int4(c.x, c.y, c.z, (int)e);
  const uint2 v = edges[e];
  es_v[k] = v;
  // the box records also carry the endpoints (bits in .w), so the E-E
  // filter needs no separate endpoint load
  float4 lo = amin[e], hi = amax[e];
  lo.w = __uint_as_float(v.x);
  hi.w = __uint_as_float(v.y);
  es_lo[k] = lo;
  es_hi[k] = hi;
}

// Canonical in-bucket order: ascending index.  Buckets hold a few to a few
// dozen entries; each thread sorts one bucket in a local array (registers /
// L1) and writes it back; larger buckets fall back to in-place insertion.
__global__ void k_hash_sort_buckets(uint32_t table, const uint32_t* __restrict__ starts, uint32_t* __restrict__ sorted) {
  const uint32_t h = blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= table) return;
  const uint32_t b = starts[h], e = starts[h + 1];
  const uint32_t n = e - b;
  if (n < 2) return;
  constexpr uint32_t kLocal = 64;
  if (n <= kLocal) {
    uint32_t a[kLocal];
    for (uint32_t k = 0; k < n; ++k) a[k] = sorted[b + k];
    for (uint32_t k = 1; k < n; ++k) {
      const uint32_t v = a[k];
      uint32_t j = k;
      while (j > 0 && a[j - 1] > v) { a[j] = a[j - 1]; --j; }
      a[j] = v;
    }
    for (uint32_t k = 0; k < n; ++k) sorted[b + k] = a[k];
    return;
  }
  for (uint32_t k = b + 1; k < e; ++k) {
    const uint32_t v = sorted[k];
    uint32_t j = k;
    while (j > b && sorted[j - 1] > v) { sorted[j] = sorted[j - 1]; --j; }
    sorted[j] = v;
  }
}

// The same canonical order (each bucket ascending), one warp per bucket: up
// to 64 entries are sorted in registers by a bitonic network (two per lane,
// padding 0xFFFFFFFF, which no index reaches); up to kSortRankCap entries by
// rank in shared memory; longer buckets fall back to the serial insertion
// sort on lane 0.  Blocks of 8 warps.
constexpr uint32_t kSortRankCap = 1024;
__global__ void __launch_bounds__(256) k_hash_sort_buckets_warp(uint32_t table, const uint32_t* __restrict__ starts,
                                                                uint32_t* __restrict__ sorted) {
  __shared__ uint32_t sh_sort[8][kSortRankCap];
  const uint32_t h = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const uint32_t lane = threadIdx.x & 31u;
  if (h >= table) return;  // whole warp
  const uint32_t b = starts[h], e = starts[h + 1];
  const uint32_t n = e - b;
  if (n < 2) return;
  if (n > 64 && n <= kSortRankCap) {
    // rank sort in shared memory: the entries are distinct indices, so the
    // rank of v (the number of smaller entries) is its sorted position
    uint32_t* buf = sh_sort[threadIdx.x >> 5];
    for (uint32_t i = lane; i < n; i += 32u) buf[i] = sorted[b + i];
    __syncwarp();
    for (uint32_t i = lane; i < n; i += 32u) {
      const uint32_t v = buf[i];
      uint32_t r = 0;
      for (uint32_t k = 0; k < n; ++k) r += buf[k] < v ? 1u : 0u;
      sorted[b + r] = v;
    }
    return;
  }
  if (n > 64) {  // larger than kSortRankCap: insertion sort by one lane
    if (lane == 0)
      for (uint32_t k = b + 1; k < e; ++k) {
        const uint32_t v = sorted[k];
        uint32_t j = k;
        while (j > b && sorted[j - 1] > v) { sorted[j] = sorted[j - 1]; --j; }
        sorted[j] = v;
      }
    return;
  }
  uint32_t a0 = lane < n ? sorted[b + lane] : 0xFFFFFFFFu;
  uint32_t a1 = lane + 32u < n ? sorted[b + lane + 32u] : 0xFFFFFFFFu;
  const uint32_t kmax = n > 32 ? 64u : 32u;
  for (uint32_t k = 2; k <= kmax; k <<= 1) {
    for (uint32_t j = k >> 1; j > 0; j >>= 1) {
      if (j == 32u) {  // partners lane and lane + 32 live in one lane
        const uint32_t lo = min(a0, a1), hi = max(a0, a1);
        const bool up = (lane & k) == 0u;
        a0 = up ? lo : hi;
        a1 = up ? hi : lo;
      } else {
        const uint32_t o0 = __shfl_xor_sync(0xffffffffu, a0, j);
        const uint32_t o1 = __shfl_xor_sync(0xffffffffu, a1, j);
        const bool lower = (lane & j) == 0u;
        const bool up0 = (lane & k) == 0u, up1 = ((lane + 32u) & k) == 0u;
        a0 = (lower == up0) ? min(a0, o0) : max(a0, o0);
        a1 = (lower == up1) ? min(a1, o1) : max(a1, o1);
      }
    }
  }
  if (lane < n) sorted[b + lane] = a0;
  if (lane + 32u < n) sorted[b + lane + 32u] = a1;
}

// ---------------- accumulation helpers (shaders/self_collision.wgsl:77-118)
__device__ __forceinline__ int32_t to_fixed(float x) { return f2i(clampf(x * 1000000.0f, -50000000.0f, 50000000.0f)); }
__device__ __forceinline__ void add_disp(int32_t* acc, uint32_t v, V3 d) {
  int32_t* a = acc + (size_t)v * A_N;
  atomicAdd(&a[A_DX], to_fixed(d.x));
  atomicAdd(&a[A_DY], to_fixed(d.y));
  atomicAdd(&a[A_DZ], to_fixed(d.z));
  atomicAdd((uint32_t*)&a[A_CNT], 1u);
}
__device__ __forceinline__ void add_pin(int32_t* acc, uint32_t v, V3 d) {
  int32_t* a = acc + (size_t)v * A_N;
  atomicAdd(&a[A_PDX], to_fixed(d.x));
  atomicAdd(&a[A_PDY], to_fixed(d.y));
  atomicAdd(&a[A_PDZ], to_fixed(d.z));
  atomicAdd((uint32_t*)&a[A_PCNT], 1u);
}
__device__ __forceinline__ void add_ccd(int32_t* acc, uint32_t v, V3 d, bool count_ee) {
  int32_t* a = acc + (size_t)v * A_N;
  const int32_t ix = to_fixed(d.x), iy = to_fixed(d.y), iz = to_fixed(d.z);
  if (ix > 0) atomicMax(&a[A_CPX], ix); else if (ix < 0) atomicMin(&a[A_CNX], ix);
  if (iy > 0) atomicMax(&a[A_CPY], iy); else if (iy < 0) atomicMin(&a[A_CNY], iy);
  if (iz > 0) atomicMax(&a[A_CPZ], iz); else if (iz < 0) atomicMin(&a[A_CNZ], iz);
  if (count_ee) {
    const float lf = clampf(length(d) * 1000000.0f, 0.0f, 2000000000.0f);
    const uint32_t u = lf != lf ? 0u : (uint32_t)lf;
    if (u > 0u) atomicAdd((uint32_t*)&a[A_EEC], 1u);
  }
}

__device__ __forceinline__ bool th_search(const SCArgs& s, uint32_t a, uint32_t b, uint32_t& pos) {
  uint32_t lo = s.th_off[a], hi = s.th_off[a + 1];
  while (lo < hi) {
    const uint32_t mid = lo + (hi - lo) / 2u;
    const uint32_t v = s.th_idx[mid];
    if (v == b) { pos = mid; return true; }
    if (v < b) lo = mid + 1u; else hi = mid;
  }
  return false;
}
// is_within_two_hops (shaders/self_collision.wgsl:243-264)
__device__ __forceinline__ bool within2(const SCArgs& s, uint32_t a, uint32_t b) {
  uint32_t q;
  if (a == b) return true;
  return th_search(s, a, b, q);
}
// is_topologically_near_folded (:268-293)
__device__ __forceinline__ bool near_folded(const SCArgs& s, uint32_t a, uint32_t b, float d) {
  uint32_t q;
  if (a == b) return true;
  if (!th_search(s, a, b, q)) return false;
  return !(d < s.th_rest[q] * 0.5f);
}
// is_topologically_near_folded_sq (shaders/self_collision_ee_direct.wgsl:237-262)
__device__ __forceinline__ bool near_folded_sq(const SCArgs& s, uint32_t a, uint32_t b, float d2) {
  uint32_t q;
  if (a == b) return true;
  if (!th_search(s, a, b, q)) return false;
  const float l0 = s.th_rest[q];
  return !(d2 < (l0 * l0) * 0.25f);
}

// ---------------- sc_solve: shaders/self_collision.wgsl:317-681
// One warp per vertex i.  The 27 neighbour buckets are flattened in the
// reference's visiting order (cx outer, cz inner, bucket order inside a cell)
// and lane L takes flattened candidates L, L+32, ...  Contacts accumulate with
// integer atomics (order-free); the multi-layer untangle candidate, which the
// reference picks with a first-strict-minimum scan, is the warp argmin of
// (distance^2, flattened position).
struct VertCtx {
  uint32_t index;
  float wi;
  bool pin_i;
  V3 xi, pi;
  float mli, thi, lli;
  I3 cell;
  uint32_t li;
  bool untangle, track;
};

// Cheap tests of one candidate (shaders/self_collision.wgsl:356-391): bucket
// cell match, untangle-candidate tracking, and the geometric bound; true when
// the contact work must run.
__device__ __forceinline__ bool sc_filter(const SCArgs& s, const VertCtx& c, const TwoHop& th, uint32_t slot,
                                          int32_t cx, int32_t cy, int32_t cz, uint32_t t, float& best_in,
                                          uint32_t& best_j, uint32_t& best_t) {
  const uint32_t index = c.index;
  // one level of loads: the three hash-ordered records of this slot
  const int4 jc = s.vs_c[slot];
  const float4 pj4 = s.vs_p[slot];
  const float4 q = s.vs_q[slot];
  const uint32_t j = (uint32_t)jc.w;
  if (j >= s.n || j == index) return false;
  const V3 pi = c.pi;
  const float thi = c.thi, lli = c.lli;
  const uint32_t li = c.li;
  const bool track = c.track;
  const V3 pj = mk(pj4);
  if (!(jc.x == cx && jc.y == cy && jc.z == cz)) return false;
  const V3 dvv = pi - pj;
  const float d2 = dot(dvv, dvv);
  const float thj = pj4.w, llj = q.x;
  const float eth = fmaxf(thi + thj, fminf(lli, llj) * 0.06f);
  const float mgd = eth + (lli + llj) * 1.3f;
  const uint32_t lj = __float_as_uint(q.y);
  if (track && lj < li && d2 < best_in) {
    const float ur = eth * 2.5f + llj * 1.3f;
    if (d2 <= ur * ur && !within2_t(th, index, j)) { best_in = d2; best_j = j; best_t = t; }
  }
  return d2 <= mgd * mgd;
}

// Contact work for one candidate that passed sc_filter
// (shaders/self_collision.wgsl:392-670), part 1: the vertex-vertex contact
// and the vertex-triangle gate.  Returns true with the star range of j when
// j's incident triangles must be tested (part 2, vt_entry).
__device__ __forceinline__ bool sc_work_vv(const SCArgs& s, const VertCtx& c, const TwoHop& th, uint32_t slot,
                                           uint32_t& st_b, uint32_t& st_e, float4& rec0, float4& rec1) {
  const uint32_t index = c.index;
  const int4 jc = s.vs_c[slot];
  const uint32_t j = (uint32_t)jc.w;
  const float wi = c.wi;
  const bool pin_i = c.pin_i;
  const V3 pi = c.pi;
  const float mli = c.mli, thi = c.thi, lli = c.lli;
  const uint32_t li = c.li;
  const bool untangle = c.untangle;
  int32_t* acc = s.acc;
  const float4 pj4 = s.vs_p[slot];
  const float4 q = s.vs_q[slot];
  const V3 pj = mk(pj4);
  const V3 dvv = pi - pj;
  const float d2 = dot(dvv, dvv);
  const float thj = pj4.w, llj = q.x;
  const float eth = fmaxf(thi + thj, fminf(lli, llj) * 0.06f);
  const uint32_t lj = __float_as_uint(q.y);
  const float dvl = sqrtf(fmaxf(d2, 0.0f));
  // one search of i's two-hop list serves both tests on j: near_folded
  // (:268-293) and, below, within_two_hops (:243-264); j != index here
  uint32_t thq = 0;
  const bool j_in2 = th_find(th, j, thq);
  if (j_in2 && !(dvl < th.rest[thq] * 0.5f)) return false;
  const V3 pjo = mk(s.x4[j]);
  const float wj = q.z;
  const bool both = wj > 0.0f;
  const float eth2 = eth * eth;
  // 1. vertex-vertex
  if (!pin_i && (!both || index < j)) {
    if (d2 < eth2 && d2 > kEps * kEps) {
      bool utv = false;
      if (untangle && li != lj) {
        const V3 ni = mk(s.nrm[index]), nj = mk(s.nrm[j]);
        const float nil = length(ni), njl = length(nj);
        if (li > lj) {
          if (njl > 0.5f) {
            const V3 nju = nj / njl;
            const bool allow = (wj <= 0.0f) || (nil <= 0.5f) || (dot(ni / fmaxf(nil, kEps), nju) > 0.0f);
            utv = allow && (dot(dvv, nju) < 0.0f);
          }
        } else if (both && nil > 0.5f) {
          const V3 niu = ni / nil;
          const bool allow = (njl <= 0.5f) || (dot(nj / fmaxf(njl, kEps), niu) > 0.0f);
          utv = allow && (dot(-dvv, niu) < 0.0f);
        }
      }
      if (!utv) {
        const V3 nn = dvv / dvl;
        const float pen = eth - dvl;
        const float ws = wi + wj;
        if (ws > kEps) {
          if (wj <= 0.0f) {
            add_pin(acc, index, nn * pen + (pj - pjo) * 0.5f);
          } else {
            const V3 disp = nn * (pen * 0.5f);
            add_disp(acc, index, disp * (wi / ws));
            add_disp(acc, j, (-disp) * (wj / ws));
          }
        }
      }
    }
  }
  // 2. vertex-triangle
  const float mlj = q.w;
  const float vtb = eth + llj * 1.3f + mli + mlj;
  if (!(d2 <= vtb * vtb) || j_in2) return false;
  {
    // Every triangle of j's star is skipped by its own swept-box test
    // (smin > tmax or smax < tmin on an axis) when the widest possible swept
    // box of i, over the star's motion range plus a 10 um rounding margin,
    // misses the star's box: skipping the whole star is then exact.
    const float4 b0 = s.sbox[3 * size_t(j)], b1 = s.sbox[3 * size_t(j) + 1], b2 = s.sbox[3 * size_t(j) + 2];
    const V3 xi = c.xi;
    const float sl = 1e-5f;
    const float rl[3] = {xi.x + b0.w - sl, xi.y + b1.w - sl, xi.z + b2.w - sl};
    const float rh[3] = {xi.x + b2.x + sl, xi.y + b2.y + sl, xi.z + b2.z + sl};
    const float pa[3] = {pi.x, pi.y, pi.z};
    const float lo[3] = {b0.x, b0.y, b0.z}, hi[3] = {b1.x, b1.y, b1.z};
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
      const float smin_lb = fminf(rl[ax], pa[ax]) - eth - sl;
      const float smax_ub = fmaxf(rh[ax], pa[ax]) + eth + sl;
      if (smin_lb > hi[ax] || smax_ub < lo[ax]) return false;
    }
  }
  st_b = s.star_off[j];
  st_e = s.star_off[j + 1];
  // what the triangle filter needs of j: p, contact thickness, x, index
  rec0 = make_float4(pj.x, pj.y, pj.z, eth);
  rec1 = make_float4(pjo.x, pjo.y, pjo.z, __uint_as_float(j));
  return st_e > st_b;
}

// Part 2: one (candidate j, incident triangle) pair, star entry `st` of j
// (shaders/self_collision.wgsl:477-667).  kHeavy = false runs the cheap tests
// (ownership, swept bounds, two-hop exclusion) on j's values cached by
// sc_work_vv (rec0 = p_j, contact thickness; rec1 = x_j, j) and returns
// whether the pair needs the contact math; kHeavy = true reloads j and runs
// the whole pair.  Each pair is independent (its output goes through the
// order-free integer accumulators).
template <bool kHeavy>
__device__ __forceinline__ bool vt_entry(const SCArgs& s, const VertCtx& c, const TwoHop& th, uint32_t slot,
                                         uint32_t st, float4 rec0 = float4(), float4 rec1 = float4()) {
  const uint32_t index = c.index;
  const float wi = c.wi;
  const bool pin_i = c.pin_i;
  const V3 xi = c.xi, pi = c.pi;
  const float mli = c.mli, thi = c.thi, lli = c.lli;
  const I3 cell = c.cell;
  const uint32_t li = c.li;
  const bool untangle = c.untangle;
  int32_t* acc = s.acc;
  V3 pj, pjo;
  uint32_t j, lj = 0u;
  float eth, wj = 0.f;
  if (kHeavy) {
    j = (uint32_t)s.vs_c[slot].w;
    const float4 pj4 = s.vs_p[slot];
    const float4 q = s.vs_q[slot];
    pj = mk(pj4);
    eth = fmaxf(thi + pj4.w, fminf(lli, q.x) * 0.06f);
    lj = __float_as_uint(q.y);
    pjo = mk(s.x4[j]);
    wj = q.z;
  } else {
    pj = mk(rec0);
    eth = rec0.w;
    pjo = mk(rec1);
    j = __float_as_uint(rec1.w);
  }
  const float eth2 = eth * eth;

  const uint2 pr = s.star_idx[st];
  const uint32_t v0 = pr.x, v1 = pr.y;
  if (v0 == index || v1 == index) return false;
  const float4 q0 = s.p4[v0], q1 = s.p4[v1];
  const V3 pv0 = mk(q0), pv1 = mk(q1);
  // ownership (:486-500): the triangle is tested from its in-range vertex of
  // smallest index, so only a vertex below j can take it away; the in-range
  // test of v0 (v1) runs, and loads its data, only when v0 < j (v1 < j)
  if (j > v0) {
    const V3 d0 = pi - pv0;
    const float ll0 = s.local_len[v0];
    const float et0 = fmaxf(thi + q0.w, fminf(lli, ll0) * 0.06f);
    const float b0 = et0 + ll0 * 1.3f + mli + s.mlen[v0];
    const int4 c0 = s.vcell[v0];
    if (abs(c0.x - cell.x) <= 1 && abs(c0.y - cell.y) <= 1 && abs(c0.z - cell.z) <= 1 && (dot(d0, d0) <= b0 * b0))
      return false;
  }
  if (j > v1) {
    const V3 d1 = pi - pv1;
    const float ll1 = s.local_len[v1];
    const float et1 = fmaxf(thi + q1.w, fminf(lli, ll1) * 0.06f);
    const float b1 = et1 + ll1 * 1.3f + mli + s.mlen[v1];
    const int4 c1 = s.vcell[v1];
    if (abs(c1.x - cell.x) <= 1 && abs(c1.y - cell.y) <= 1 && abs(c1.z - cell.z) <= 1 && (dot(d1, d1) <= b1 * b1))
      return false;
  }
  const float4 o0 = s.x4[v0], o1 = s.x4[v1];
  const V3 pv0o = mk(o0), pv1o = mk(o1);
  const float wv0 = o0.w, wv1 = o1.w;
  const V3 tmove = (((pj - pjo) + (pv0 - pv0o)) + (pv1 - pv1o)) / 3.0f;
  const bool tpin = (wj <= 0.0f) || (wv0 <= 0.0f) || (wv1 <= 0.0f);
  const V3 rel = xi + tmove;
  const V3 E = mk(eth, eth, eth);
  const V3 smin = vmin(rel, pi) - E, smax = vmax(rel, pi) + E;
  const V3 tmin = vmin(vmin(pj, pv0), pv1), tmax = vmax(vmax(pj, pv0), pv1);
  if (smin.x > tmax.x || smin.y > tmax.y || smin.z > tmax.z || smax.x < tmin.x || smax.y < tmin.y ||
      smax.z < tmin.z)
    return false;
  if (within2_t(th, index, v0) || within2_t(th, index, v1)) return false;
  if (!kHeavy) return true;
  const V3 mv = pi - rel;
  const float msq = dot(mv, mv);
  float ht = 1.0f, hu = 0.0f, hv = 0.0f;
  bool hit = false;
  if (msq > 1e-12f) hit = seg_tri(rel, pi, pj, pv0, pv1, ht, hu, hv);
  if (hit) {
    const V3 hp = rel + mv * ht;
    const V3 tc = cross(pv0 - pj, pv1 - pj);
    const float tl = length(tc);
    const V3 tn = tl > 1e-12f ? tc / tl : mk(0.0f, 1.0f, 0.0f);
    const float hor = dot(rel - pj, tn);
    bool utc = false;
    if (untangle && !pin_i && (li > lj) && tl > 1e-12f) {
      const V3 ni = mk(s.nrm[index]);
      const float nil = length(ni);
      const bool allow = tpin || (nil <= 0.5f) || (dot(ni / fmaxf(nil, kEps), tn) > 0.0f);
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
    }
  } else {
    bool isf;
    V3 bary;
    const V3 cp = closest_tri(pi, pj, pv0, pv1, isf, bary);
    const V3 dvt = pi - cp;
    const float d2vt = dot(dvt, dvt);
    if (!pin_i && d2vt < eth2 && d2vt > kEps * kEps) {
      const float dvtl = sqrtf(d2vt);
      bool utv = false;
      if (untangle && li > lj) {
        const V3 tc = cross(pv0 - pj, pv1 - pj);
        const float tl = length(tc);
        if (tl > kEps) {
          const V3 tn = tc / tl;
          if (dot(dvt, tn) < 0.0f) {
            const V3 ni = mk(s.nrm[index]);
            const float nil = length(ni);
            utv = tpin || (nil <= 0.5f) || (dot(ni / fmaxf(nil, kEps), tn) > 0.0f);
          }
        }
      }
      if (!utv) {
        const V3 nvt = dvt / dvtl;
        const float pvt = eth - dvtl;
        if (tpin) {
          add_pin(acc, index, nvt * pvt + tmove * 0.5f);
        } else {
          const float wt = bary.x * bary.x * wj + bary.y * bary.y * wv0 + bary.z * bary.z * wv1;
          const float wtot = wi + wt;
          if (wtot > kEps) {
            const V3 tp = nvt * (pvt * 0.6f);
            add_disp(acc, index, tp * (wi / wtot));
            if (wj > 0.0f) add_disp(acc, j, (-tp) * (bary.x * wj / wtot));
            if (wv0 > 0.0f) add_disp(acc, v0, (-tp) * (bary.y * wv0 / wtot));
            if (wv1 > 0.0f) add_disp(acc, v1, (-tp) * (bary.z * wv1 / wtot));
          }
        }
      }
    }
  }
  return true;
}

__global__ void __launch_bounds__(256, 4) k_sc_solve(SCArgs s) {
  __shared__ uint32_t sh_start[8][28], sh_end[8][28], sh_beg[8][28];
  __shared__ uint32_t sh_th[8][kTwoHopCache];
  __shared__ float sh_thr[8][kTwoHopCache];
  __shared__ uint32_t sh_q[8][32 * kRounds];
  __shared__ uint32_t pr_slot[8][32], pr_sb[8][32], pr_ex[8][32];  // survivors' star ranges
  __shared__ uint32_t tq_slot[8][64], tq_st[8][64];                 // (candidate, triangle) pairs
  __shared__ float4 pr_rec0[8][32], pr_rec1[8][32];                 // survivors' cached values
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t index = blockIdx.x * 8u + warp;
  if (index >= s.n) return;  // whole warp
  VertCtx c;
  c.index = index;
  const float4 xi4 = s.x4[index], pi4 = s.p4[index];
  c.wi = xi4.w;
  c.pin_i = c.wi <= 0.0f;
  c.xi = mk(xi4);
  c.pi = mk(pi4);
  c.mli = s.mlen[index];
  if (c.pin_i && c.mli < kEps) return;  // whole warp
  const TwoHop th = stage_two_hop(s.th_off, s.th_idx, s.th_rest, index, sh_th[warp], sh_thr[warp], lane);
  c.thi = pi4.w;
  c.lli = s.local_len[index];
  {
    const int4 vc = s.vcell[index];
    c.cell = I3{vc.x, vc.y, vc.z};
  }
  c.li = layer_of(s.v4, index);
  c.untangle = s.untangle != 0;
  c.track = c.untangle && !c.pin_i && c.li > 0u;
  // bucket ranges of the 27 neighbour cells, lane k = (dx+1)*9 + (dy+1)*3 + (dz+1)
  uint32_t cnt = 0, beg = 0;
  if (lane < 27) {
    const uint32_t h = hash3(c.cell.x - 1 + lane / 9, c.cell.y - 1 + (lane / 3) % 3, c.cell.z - 1 + lane % 3, s.table);
    beg = s.cs[h];
    cnt = s.cs[h + 1] - beg;
  }
  uint32_t incl = cnt;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  if (lane < 27) {
    sh_start[warp][lane] = incl - cnt;
    sh_end[warp][lane] = incl;
    sh_beg[warp][lane] = beg;
  }
  __syncwarp();
  const uint32_t total = __shfl_sync(0xffffffffu, incl, 26);
  float best_in = 1e20f;
  uint32_t best_j = 0xFFFFFFFFu, best_t = 0xFFFFFFFFu;
  int k = 0;
  uint32_t* queue = sh_q[warp];
  const uint32_t lt_mask = (1u << lane) - 1u;
  uint32_t tqn = 0;
  for (uint32_t chunk = 0; chunk < total; chunk += 32u * kRounds) {
    // phase 1: cheap filters on 32 x kRounds candidates, survivors compacted
    uint32_t qn = 0;
    for (uint32_t r = 0; r < kRounds; ++r) {
      const uint32_t t = chunk + r * 32u + lane;
      bool pass = false;
      uint32_t slot = 0;
      if (t < total) {
        while (t >= sh_end[warp][k]) ++k;
        slot = sh_beg[warp][k] + (t - sh_start[warp][k]);
        pass = sc_filter(s, c, th, slot, c.cell.x - 1 + k / 9, c.cell.y - 1 + (k / 3) % 3, c.cell.z - 1 + k % 3, t,
                         best_in, best_j, best_t);
      }
      const uint32_t b = __ballot_sync(0xffffffffu, pass);
      if (pass) queue[qn + __popc(b & lt_mask)] = slot;
      qn += __popc(b);
    }
    __syncwarp();
    // phase 2: vertex-vertex work on the survivors, 32 at a time; each
    // survivor's incident triangles become (survivor, star entry) pairs
    for (uint32_t base = 0; base < qn; base += 32u) {
      const uint32_t q = base + lane;
      uint32_t sb = 0, se = 0;
      float4 r0 = make_float4(0.f, 0.f, 0.f, 0.f), r1 = r0;
      const uint32_t slot = q < qn ? queue[q] : 0u;
      const bool vt = q < qn && sc_work_vv(s, c, th, slot, sb, se, r0, r1);
      const uint32_t cnt = vt ? se - sb : 0u;
      uint32_t incl = cnt;
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
      }
      const uint32_t npairs = __shfl_sync(0xffffffffu, incl, 31);
      pr_slot[warp][lane] = slot;
      pr_sb[warp][lane] = sb;
      pr_ex[warp][lane] = incl - cnt;
      pr_rec0[warp][lane] = r0;
      pr_rec1[warp][lane] = r1;
      __syncwarp();
      // phase 3: cheap tests of each pair; passing pairs are compacted into
      // tq and the contact math runs on full batches of 32
      for (uint32_t eb = 0; eb < npairs; eb += 32u) {
        const uint32_t e = eb + uint32_t(lane);
        bool pass = false;
        uint32_t ps = 0, pst = 0;
        if (e < npairs) {
          uint32_t lo = 0, hi = 31;  // owner: the last lane whose range starts at or before e
          while (lo < hi) {
            const uint32_t mid = (lo + hi + 1u) >> 1;
            if (pr_ex[warp][mid] <= e) lo = mid; else hi = mid - 1u;
          }
          ps = pr_slot[warp][lo];
          pst = pr_sb[warp][lo] + (e - pr_ex[warp][lo]);
          pass = vt_entry<false>(s, c, th, ps, pst, pr_rec0[warp][lo], pr_rec1[warp][lo]);
          if (pass && s.rec_vt) {
            const uint2 tv = s.star_idx[pst];
            record_vt(s, index, __float_as_uint(pr_rec1[warp][lo].w), tv.x, tv.y);
          }
        }
        const uint32_t b = __ballot_sync(0xffffffffu, pass);
        if (pass) {
          const uint32_t kq = tqn + __popc(b & lt_mask);
          tq_slot[warp][kq] = ps;
          tq_st[warp][kq] = pst;
        }
        tqn += __popc(b);
        __syncwarp();
        if (tqn >= 32u) {
          vt_entry<true>(s, c, th, tq_slot[warp][lane], tq_st[warp][lane]);
          __syncwarp();
          tqn -= 32u;
          if (uint32_t(lane) < tqn) {
            tq_slot[warp][lane] = tq_slot[warp][32 + lane];
            tq_st[warp][lane] = tq_st[warp][32 + lane];
          }
          __syncwarp();
        }
      }
      __syncwarp();
    }
  }
  if (uint32_t(lane) < tqn) vt_entry<true>(s, c, th, tq_slot[warp][lane], tq_st[warp][lane]);
  if (c.track) {
    for (int o = 16; o > 0; o >>= 1) {
      const float ob = __shfl_xor_sync(0xffffffffu, best_in, o);
      const uint32_t ot = __shfl_xor_sync(0xffffffffu, best_t, o);
      const uint32_t oj = __shfl_xor_sync(0xffffffffu, best_j, o);
      if (ob < best_in || (ob == best_in && ot < best_t)) { best_in = ob; best_t = ot; best_j = oj; }
    }
    if (lane == 0 && best_j < 0x3FFFFEu) s.acc[(size_t)index * A_N + A_UT] = (int32_t)(best_j + 1u);
  }
}

// ---------------- sc_untangle: shaders/self_collision_untangle.wgsl:199-394
__device__ __forceinline__ bool th_range_has(const SCArgs& s, uint32_t b0, uint32_t e0, uint32_t v) {
  if (b0 >= e0) return false;
  uint32_t lo = b0, hi = e0;
  while (lo < hi) {
    const uint32_t mid = lo + (hi - lo) / 2u;
    const uint32_t x = s.th_idx[mid];
    if (x == v) return true;
    if (x < v) lo = mid + 1u; else hi = mid;
  }
  return false;
}

__global__ void k_untangle(SCArgs s) {
  const uint32_t index = blockIdx.x * blockDim.x + threadIdx.x;
  if (index >= s.n || !s.untangle) return;
  int32_t* ai = s.acc + (size_t)index * A_N;
  const uint32_t cand = (uint32_t)ai[A_UT];
  if (cand == 0u) return;
  ai[A_UT] = 0;
  const float wi = s.x4[index].w;
  const uint32_t li = layer_of(s.v4, index);
  if (wi <= 0.0f || li == 0u) return;
  const uint32_t j1e = cand & 0x3FFFFFu;
  if (j1e == 0u) return;
  const uint32_t j1 = j1e - 1u;
  if (j1 >= s.n || j1 == index) return;
  const float4 pi4 = s.p4[index];
  const V3 pi = mk(pi4);
  const float thi = pi4.w, lli = s.local_len[index];
  const uint32_t ts = s.th_off[index], te = s.th_off[index + 1];
  uint32_t j2 = 0xFFFFFFFFu;
  float bnd = 1e20f;
  for (uint32_t a = s.adj_off[j1]; a < s.adj_off[j1 + 1]; ++a) {
    const uint32_t nb = s.adj_idx[a];
    if (nb < s.n && nb != index && layer_of(s.v4, nb) < li) {
      const V3 dn = pi - mk(s.p4[nb]);
      const float dns = dot(dn, dn);
      if (dns < bnd && !th_range_has(s, ts, te, nb)) { bnd = dns; j2 = nb; }
    }
  }
  float bd2 = 1e20f, bh = 0.0f;
  uint32_t bj = 0xFFFFFFFFu, bv0 = 0, bv1 = 0;
  for (int ci = 0; ci < 2; ++ci) {
    const uint32_t j = ci == 0 ? j1 : j2;
    if (j == 0xFFFFFFFFu) continue;
    const float4 pj4 = s.p4[j];
    const V3 pj = mk(pj4);
    const float eth = fmaxf(thi + pj4.w, fminf(lli, s.local_len[j]) * 0.06f);
    const float capt = eth * 2.5f;
    const float capsq = capt * capt;
    for (uint32_t st = s.star_off[j]; st < s.star_off[j + 1]; ++st) {
      const uint2 pr = s.star_idx[st];
      const uint32_t v0 = pr.x, v1 = pr.y;
      if (v0 == index || v1 == index) continue;
      if (ci == 1 && (v0 == j1 || v1 == j1)) continue;
      const V3 pv0 = mk(s.p4[v0]), pv1 = mk(s.p4[v1]);
      const V3 tmin = vmin(vmin(pj, pv0), pv1), tmax = vmax(vmax(pj, pv0), pv1);
      const V3 z = mk(0.f, 0.f, 0.f);
      const V3 ad = vmax(tmin - pi, z) + vmax(pi - tmax, z);
      const float lim = fminf(capsq, bd2 + 1e-10f);
      if (dot(ad, ad) >= lim) continue;
      bool isf;
      V3 bary;
      const V3 pt = closest_tri(pi, pj, pv0, pv1, isf, bary);
      const V3 du = pi - pt;
      const float dsu = dot(du, du);
      if (dsu >= capsq) continue;
      if (bj != 0xFFFFFFFFu && dsu > bd2 + 1e-10f) continue;
      const V3 tc = cross(pv0 - pj, pv1 - pj);
      const float tl = length(tc);
      if (tl <= kEps) continue;
      const float hu = dot(du, tc / tl);
      const bool same = fabsf(dsu - bd2) <= 1e-10f;
      const bool better = (hu >= 0.0f && bh < 0.0f) || (((hu >= 0.0f) == (bh >= 0.0f)) && fabsf(hu) > fabsf(bh));
      if (bj == 0xFFFFFFFFu || dsu < bd2 - 1e-10f || (same && better)) {
        if (th_range_has(s, ts, te, j) || th_range_has(s, ts, te, v0) || th_range_has(s, ts, te, v1)) continue;
        bd2 = dsu; bh = hu; bj = j; bv0 = v0; bv1 = v1;
      }
    }
  }
  if (bj != 0xFFFFFFFFu && bh < 0.0f) {
    const float4 qj = s.p4[bj], q0 = s.p4[bv0], q1 = s.p4[bv1];
    const V3 upj = mk(qj), up0 = mk(q0), up1 = mk(q1);
    const float wj = s.x4[bj].w, w0 = s.x4[bv0].w, w1 = s.x4[bv1].w;
    bool isf;
    V3 bary;
    const V3 pt = closest_tri(pi, upj, up0, up1, isf, bary);
    const V3 du = pi - pt;
    const float dl = length(du);
    const V3 tc = cross(up0 - upj, up1 - upj);
    const float tl = length(tc);
    if (tl > kEps && dl > kEps) {
      const V3 tn = tc / tl;
      const float hu = dot(du, tn);
      if (hu < 0.0f) {
        const V3 ni = mk(s.nrm[index]);
        const float nil = length(ni);
        const bool tpin = (wj <= 0.0f) || (w0 <= 0.0f) || (w1 <= 0.0f);
        const bool allow = tpin || (nil <= 0.5f) || (dot(ni / fmaxf(nil, kEps), tn) > 0.0f);
        const float etu = fmaxf(thi + qj.w, fminf(lli, s.local_len[bj]) * 0.06f);
        const float cb = -hu / dl;
        const float rt = sqrtf(fmaxf(dl * dl - hu * hu, 0.0f));
        const float rl = fmaxf(etu * 0.5f, kEps);
        if (allow && cb > 0.707f && rt < rl) {
          const V3 ni2 = (mk(s.nrm[bj]) * bary.x + mk(s.nrm[bv0]) * bary.y) + mk(s.nrm[bv1]) * bary.z;
          const float nl = length(ni2);
          const bool behind = (nl <= 0.5f) || (dot(du, ni2) < 0.0f);
          if (behind) {
            const float cw = clampf((cb - 0.707f) / 0.2f, 0.0f, 1.0f);
            const float rw = clampf(1.0f - rt / rl, 0.0f, 1.0f);
            const float pen = fminf(etu - hu, etu * 2.0f) * cw * rw;
            if (pen > kEps) {
              if (tpin) {
                add_disp(s.acc, index, tn * pen);
              } else {
                const float wt = bary.x * bary.x * wj + bary.y * bary.y * w0 + bary.z * bary.z * w1;
                const float wtot = wi + wt;
                if (wtot > kEps) {
                  const V3 disp = tn * (pen * 0.5f);
                  add_disp(s.acc, index, disp * (wi / wtot));
                  if (wj > 0.0f) add_disp(s.acc, bj, (-disp) * (bary.x * wj / wtot));
                  if (w0 > 0.0f) add_disp(s.acc, bv0, (-disp) * (bary.y * w0 / wtot));
                  if (w1 > 0.0f) add_disp(s.acc, bv1, (-disp) * (bary.z * w1 / wtot));
                }
              }
            }
          }
        }
      }
    }
  }
}

// ---------------- sc_solve_ee: shaders/self_collision_ee_direct.wgsl:266-776
__device__ __forceinline__ float seg_eval(V3 a0o, V3 a0, V3 a1o, V3 a1, V3 b0o, V3 b0, V3 b1o, V3 b1, float tau,
                                          float& so, float& to) {
  const V3 A0 = vmix(a0o, a0, tau), A1 = vmix(a1o, a1, tau), B0 = vmix(b0o, b0, tau), B1 = vmix(b1o, b1, tau);
  seg_seg(A0, A1, B0, B1, so, to);
  const V3 d = vmix(A0, A1, so) - vmix(B0, B1, to);
  return dot(d, d);
}
__device__ __forceinline__ float seg_vol(V3 a0o, V3 a0, V3 a1o, V3 a1, V3 b0o, V3 b0, V3 b1o, V3 b1, float tau) {
  const V3 A0 = vmix(a0o, a0, tau), A1 = vmix(a1o, a1, tau), B0 = vmix(b0o, b0, tau), B1 = vmix(b1o, b1, tau);
  return dot(cross(A1 - A0, B1 - B0), B0 - A0);
}
__device__ __forceinline__ bool outer_behind(const SCArgs& s, uint32_t la, uint32_t lb, uint32_t a0, uint32_t a1,
                                             uint32_t b0, uint32_t b1, bool afix, bool bfix, V3 dab) {
  if (la == lb) return false;
  const V3 na = mk(s.nrm[a0]) + mk(s.nrm[a1]), nb = mk(s.nrm[b0]) + mk(s.nrm[b1]);
  const float nal = length(na), nbl = length(nb);
  if (la > lb) {
    if (nbl <= 0.5f) return false;
    const V3 ni = nb / nbl;
    const bool allow = bfix || (nal <= 0.5f) || (dot(na / fmaxf(nal, kEps), ni) > 0.0f);
    return allow && (dot(dab, ni) < 0.0f);
  }
  if (nal <= 0.5f) return false;
  const V3 ni = na / nal;
  const bool allow = afix || (nbl <= 0.5f) || (dot(nb / fmaxf(nbl, kEps), ni) > 0.0f);
  return allow && (dot(-dab, ni) < 0.0f);
}

struct EdgeCtx {
  uint32_t ei, u0, u1;
  float w_u0, w_u1;
  bool apin, bnda;
  V3 p_u0, p_u1, p_u0o, p_u1o;
  float thu0, thu1, mta;
  V3 amin, amax;
  uint32_t la;
  bool untangle;
};

// Contact work for one counted edge pair (shaders/self_collision_ee_direct.wgsl:356-774).
// defer_ccd: the warp pass hands pairs that need the CCD search to the
// one-thread-per-pair k_ee_ccd (inline when the queue is full).
__device__ __forceinline__ void ee_pair(const SCArgs& s, const EdgeCtx& c, const TwoHop& th0, const TwoHop& th1,
                                        uint32_t eb, uint32_t j, uint32_t vj, const float4& qj, const float4& qvj,
                                        const float4& xj, const float4& xvj, bool defer_ccd) {
  const uint32_t u0 = c.u0, u1 = c.u1;
  const float w_u0 = c.w_u0, w_u1 = c.w_u1;
  const bool apin = c.apin, bnda = c.bnda;
  const V3 p_u0 = c.p_u0, p_u1 = c.p_u1, p_u0o = c.p_u0o, p_u1o = c.p_u1o;
  const float thu0 = c.thu0, thu1 = c.thu1, mta = c.mta;
  const uint32_t la = c.la;
  const bool untangle = c.untangle;
  int32_t* acc = s.acc;
  const V3 p_j = mk(qj), p_vj = mk(qvj), p_jo = mk(xj), p_vjo = mk(xvj);
  const float w_j = xj.w, w_vj = xvj.w;
  const float thj = qj.w, thvj = qvj.w;
  const uint32_t lb = layer_of(s.v4, j);
  const bool bndb = ((s.edge_bits[eb >> 5] >> (eb & 31u)) & 1u) != 0u;
  const bool bpair = bnda || bndb;
  bool run_ccd = bpair, has1 = false;
  float s1 = 0.f, t1 = 0.f, d2c = 0.f, ethc = 0.f;
  V3 dl1 = mk(0.f, 0.f, 0.f);
  if (!run_ccd) {
    seg_seg(p_u0, p_u1, p_j, p_vj, s1, t1);
    dl1 = vmix(p_u0, p_u1, s1) - vmix(p_j, p_vj, t1);
    d2c = dot(dl1, dl1);
    ethc = mixf(thu0, thu1, s1) + mixf(thj, thvj, t1);
    const float meg = mta + fmaxf(thj, thvj);
    const V3 dv0 = p_u0 - p_u0o, dv1 = p_u1 - p_u1o, dvj = p_j - p_jo, dvvj = p_vj - p_vjo;
    const V3 va = (dv0 + dv1) * 0.5f, vb = (dvj + dvvj) * 0.5f;
    const float rdg = length(va - vb) + 0.5f * (length(dv1 - dv0) + length(dvvj - dvj));
    const float reach = meg + rdg;
    if (d2c > reach * reach) return;
    has1 = true;
    const V3 d0g = vmix(p_u0o, p_u1o, s1) - vmix(p_jo, p_vjo, t1);
    run_ccd = (rdg > ethc * 0.5f) || (dot(d0g, dl1) <= 0.0f);
  }
  if (run_ccd && defer_ccd) {
    const uint32_t q = atomicAdd(s.ccd_n, 1u);
    if (q < s.ccd_cap) {
      s.ccd_q[q] = make_uint2(c.ei, eb);
      return;
    }
  }
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
    float tstar = btau, dstar = msd, ss = ms, ts = mt;
    for (int it = 0; it < 6; ++it) {
      const float m1 = tlo + (thi - tlo) * (1.0f / 3.0f);
      const float mm2 = thi - (thi - tlo) * (1.0f / 3.0f);
      float e1s, e1t, e2s, e2t;
      const float e1 = seg_eval(p_u0o, p_u0, p_u1o, p_u1, p_jo, p_j, p_vjo, p_vj, m1, e1s, e1t);
      const float e2 = seg_eval(p_u0o, p_u0, p_u1o, p_u1, p_jo, p_j, p_vjo, p_vj, mm2, e2s, e2t);
      if (e1 < dstar) { dstar = e1; tstar = m1; ss = e1s; ts = e1t; }
      if (e2 < dstar) { dstar = e2; tstar = mm2; ss = e2s; ts = e2t; }
      if (e1 < e2) thi = mm2; else tlo = m1;
    }
    const float ets = mixf(thu0, thu1, ss) + mixf(thj, thvj, ts);
    if (dstar >= ets * ets) return;
    if (s.exclude_neighbors) {
      const V3 a0s = vmix(p_u0o, p_u0, tstar), a1s = vmix(p_u1o, p_u1, tstar);
      const V3 b0s = vmix(p_jo, p_j, tstar), b1s = vmix(p_vjo, p_vj, tstar);
      const V3 t0 = a0s - b0s, t1v = a0s - b1s, t2 = a1s - b0s, t3 = a1s - b1s;
      if (near_folded_sq_t(th0, u0, j, dot(t0, t0)) || near_folded_sq_t(th0, u0, vj, dot(t1v, t1v)) ||
          near_folded_sq_t(th1, u1, j, dot(t2, t2)) || near_folded_sq_t(th1, u1, vj, dot(t3, t3)))
        return;
    }
    bool utc = false;
    if (untangle && la != lb) {
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
      float s1b, t1b;
      seg_seg(p_u0, p_u1, p_j, p_vj, s1b, t1b);
      const V3 d1 = vmix(p_u0, p_u1, s1b) - vmix(p_j, p_vj, t1b);
      const float dist1 = length(d1);
      const V3 de = vmix(p_u0, p_u1, ss) - vmix(p_j, p_vj, ts);
      const float he = dot(de, n0);
      const bool crossed = (he <= 0.0f) || (dot(d1, n0) <= 0.0f) || (bpair && dist1 >= ets && tstar < 1.0f);
      if (he < ets && crossed) {
        const float pc = ets - he;
        const bool bpin = (w_j <= 0.0f) || (w_vj <= 0.0f);
        if (apin && bpin) return;
        const bool aall = (w_u0 == 0.0f) && (w_u1 == 0.0f);
        const bool ball = (w_j == 0.0f) && (w_vj == 0.0f);
        const bool cpe = !(aall || ball);
        if (bpin) {
          const V3 em = ((p_j - p_jo) + (p_vj - p_vjo)) * 0.5f;
          const float a = 1.0f - ss, b = ss;
          const float den = a * a * w_u0 + b * b * w_u1;
          if (den > kEps) {
            const V3 pb = n0 * pc + em * 0.5f;
            if (w_u0 > 0.0f) add_ccd(acc, u0, pb * fminf((a * w_u0) / den, 2.0f), cpe);
            if (w_u1 > 0.0f) add_ccd(acc, u1, pb * fminf((b * w_u1) / den, 2.0f), cpe);
          }
        } else if (apin) {
          const V3 em = ((p_u0 - p_u0o) + (p_u1 - p_u1o)) * 0.5f;
          const float a = 1.0f - ts, b = ts;
          const float den = a * a * w_j + b * b * w_vj;
          if (den > kEps) {
            const V3 pb = (-n0) * pc + em * 0.5f;
            if (w_j > 0.0f) add_ccd(acc, j, pb * fminf((a * w_j) / den, 2.0f), cpe);
            if (w_vj > 0.0f) add_ccd(acc, vj, pb * fminf((b * w_vj) / den, 2.0f), cpe);
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
  {
    float sst, tst, d2e, eth;
    V3 de;
    if (has1) {
      sst = s1; tst = t1; de = dl1; d2e = d2c; eth = ethc;
    } else {
      seg_seg(p_u0, p_u1, p_j, p_vj, sst, tst);
      de = (p_u0 + (p_u1 - p_u0) * sst) - (p_j + (p_vj - p_j) * tst);
      d2e = dot(de, de);
      eth = mixf(thu0, thu1, sst) + mixf(thj, thvj, tst);
    }
    if (d2e >= eth * eth || d2e <= kEps * kEps) return;
    if (s.exclude_neighbors) {
      const V3 e0 = p_u0 - p_j, e1 = p_u0 - p_vj, e2 = p_u1 - p_j, e3 = p_u1 - p_vj;
      if (near_folded_sq_t(th0, u0, j, dot(e0, e0)) || near_folded_sq_t(th0, u0, vj, dot(e1, e1)) ||
          near_folded_sq_t(th1, u1, j, dot(e2, e2)) || near_folded_sq_t(th1, u1, vj, dot(e3, e3)))
        return;
    }
    const float del = sqrtf(d2e);
    bool ute = false;
    if (untangle) {
      const bool afx = (w_u0 <= 0.0f) && (w_u1 <= 0.0f);
      const bool bfx = (w_j <= 0.0f) && (w_vj <= 0.0f);
      ute = outer_behind(s, la, lb, u0, u1, j, vj, afx, bfx, de);
    }
    if (!ute) {
      const V3 ne = de / del;
      const float pe = eth - del;
      const bool bpin = (w_j <= 0.0f) || (w_vj <= 0.0f);
      if (apin && bpin) return;
      if (bpin) {
        const V3 em = ((p_j - p_jo) + (p_vj - p_vjo)) * 0.5f;
        const float a = 1.0f - sst, b = sst;
        const float den = a * a * w_u0 + b * b * w_u1;
        if (den > kEps) {
          const V3 pb = ne * pe + em * 0.5f;
          if (w_u0 > 0.0f) add_pin(acc, u0, pb * fminf((a * w_u0) / den, 2.0f));
          if (w_u1 > 0.0f) add_pin(acc, u1, pb * fminf((b * w_u1) / den, 2.0f));
        }
      } else if (apin) {
        const V3 em = ((p_u0 - p_u0o) + (p_u1 - p_u1o)) * 0.5f;
        const float a = 1.0f - tst, b = tst;
        const float den = a * a * w_j + b * b * w_vj;
        if (den > kEps) {
          const V3 pb = (-ne) * pe + em * 0.5f;
          if (w_j > 0.0f) add_pin(acc, j, pb * fminf((a * w_j) / den, 2.0f));
          if (w_vj > 0.0f) add_pin(acc, vj, pb * fminf((b * w_vj) / den, 2.0f));
        }
      } else {
        const float we1 = (1.0f - sst) * (1.0f - sst) * w_u0 + sst * sst * w_u1;
        const float we2 = (1.0f - tst) * (1.0f - tst) * w_j + tst * tst * w_vj;
        const float wtot = we1 + we2;
        if (wtot > kEps) {
          const V3 td = ne * (pe * 0.6f);
          if (w_u0 > 0.0f) add_disp(acc, u0, td * ((1.0f - sst) * w_u0 / wtot));
          if (w_u1 > 0.0f) add_disp(acc, u1, td * (sst * w_u1 / wtot));
          if (w_j > 0.0f) add_disp(acc, j, (-td) * ((1.0f - tst) * w_j / wtot));
          if (w_vj > 0.0f) add_disp(acc, vj, (-td) * (tst * w_vj / wtot));
        }
      }
    }
  }
}

__device__ __forceinline__ EdgeCtx edge_ctx(const SCArgs& s, uint32_t ei) {
  EdgeCtx c;
  c.ei = ei;
  const uint2 ea = s.edges[ei];
  c.u0 = ea.x;
  c.u1 = ea.y;
  const float4 xu0 = s.x4[c.u0], xu1 = s.x4[c.u1], qu0 = s.p4[c.u0], qu1 = s.p4[c.u1];
  c.w_u0 = xu0.w;
  c.w_u1 = xu1.w;
  c.apin = (c.w_u0 <= 0.0f) || (c.w_u1 <= 0.0f);
  c.p_u0 = mk(qu0); c.p_u1 = mk(qu1); c.p_u0o = mk(xu0); c.p_u1o = mk(xu1);
  c.thu0 = qu0.w;
  c.thu1 = qu1.w;
  c.mta = fmaxf(c.thu0, c.thu1);
  c.bnda = ((s.edge_bits[ei >> 5] >> (ei & 31u)) & 1u) != 0u;
  const V3 m2 = mk(c.mta * 2.0f, c.mta * 2.0f, c.mta * 2.0f);
  c.amin = vmin(vmin(c.p_u0, c.p_u1), vmin(c.p_u0o, c.p_u1o)) - m2;
  c.amax = vmax(vmax(c.p_u0, c.p_u1), vmax(c.p_u0o, c.p_u1o)) + m2;
  c.la = layer_of(s.v4, c.u0);
  c.untangle = s.untangle != 0;
  return c;
}

// Contact work for a listed (edge, edge) pair, with the two-hop lists of
// the first edge's endpoints read from global memory.
__device__ __forceinline__ void ee_listed_pair(const SCArgs& s, uint2 pr, bool defer_ccd) {
  const EdgeCtx c = edge_ctx(s, pr.x);
  TwoHop th0, th1;
  th0.idx = s.th_idx + s.th_off[c.u0];
  th0.rest = s.th_rest + s.th_off[c.u0];
  th0.n = s.th_off[c.u0 + 1] - s.th_off[c.u0];
  th1.idx = s.th_idx + s.th_off[c.u1];
  th1.rest = s.th_rest + s.th_off[c.u1];
  th1.n = s.th_off[c.u1 + 1] - s.th_off[c.u1];
  const uint2 ebv = s.edges[pr.y];
  ee_pair(s, c, th0, th1, pr.y, ebv.x, ebv.y, s.p4[ebv.x], s.p4[ebv.y], s.x4[ebv.x], s.x4[ebv.y], defer_ccd);
}

// ee_listed_pair outside the caller's register allocation, for the rare
// pairs that do not fit the pair list.
__device__ __noinline__ void ee_listed_pair_call(const SCArgs& s, uint2 pr) { ee_listed_pair(s, pr, true); }

// Counted pairs listed by k_ee, one thread each: the CCD gate of
// shaders/self_collision_ee_direct.wgsl:361-403 and the discrete contact
// from :632 on; pairs that need the CCD search go on to k_ee_ccd.
// Grid: kEeSeg * kEePairBlocks blocks of 256 threads.
__global__ void __launch_bounds__(256, 4) k_ee_pairs(SCArgs s) {
  const uint32_t seg = blockIdx.x / kEePairBlocks, segcap = s.ee_cap / kEeSeg;
  const uint32_t total = min(s.ee_n[seg], segcap);
  const uint2* list = s.ee_q + size_t(seg) * segcap;
  for (uint32_t q = (blockIdx.x % kEePairBlocks) * blockDim.x + threadIdx.x; q < total;
       q += kEePairBlocks * blockDim.x) {
    const uint2 pr = list[q];
    if (s.rec_ee) record_ee(s, pr.x, pr.y);
    ee_listed_pair(s, pr, true);
  }
}

// Deferred CCD pairs, one thread each (the CCD search plus the discrete
// fall-through of shaders/self_collision_ee_direct.wgsl:404-774).
__global__ void __launch_bounds__(256, 3) k_ee_ccd(SCArgs s) {
  const uint32_t total = min(*s.ccd_n, s.ccd_cap);
  for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < total; q += gridDim.x * blockDim.x)
    ee_listed_pair(s, s.ccd_q[q], false);
}

// One warp per edge; candidates of the 27 cells around the edge midpoint are
// flattened in the reference's order (dz outer, dx inner) and visited 32 per
// round.  The per-edge cap on counted candidates (search_count >
// max_search_iterations, :356-359) is applied with a ballot prefix count, so
// exactly the reference's first max_search counted pairs are processed.
// kList: the counted pairs are appended to the pair list for k_ee_pairs
// (the two-hop lists are then not staged here); otherwise the warp does
// their contact work itself.
// (__grid_constant__: the overflow call takes the arguments' address without
// a per-thread copy.)  The filter alone is latency-bound and needs few
// registers, so list mode asks for 8 blocks (64 warps) per SM.
template <bool kList>
__global__ void __launch_bounds__(256, kList ? 8 : 4) k_ee(const __grid_constant__ SCArgs s) {
  __shared__ uint32_t sh_start[8][28], sh_end[8][28], sh_beg[8][28];
  __shared__ uint32_t sh_th[8][2][kTwoHopCache];
  __shared__ float sh_thr[8][2][kTwoHopCache];
  __shared__ uint32_t sh_q[8][32 * kRounds];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t ei = blockIdx.x * 8u + warp;
  if (ei >= s.ne) return;  // whole warp
  const EdgeCtx c = edge_ctx(s, ei);
  const int4 bc4 = s.ecell[ei];
  const I3 base = I3{bc4.x, bc4.y, bc4.z};
  TwoHop th0{}, th1{};
  if (!kList) {
    th0 = stage_two_hop(s.th_off, s.th_idx, s.th_rest, c.u0, sh_th[warp][0], sh_thr[warp][0], lane);
    th1 = stage_two_hop(s.th_off, s.th_idx, s.th_rest, c.u1, sh_th[warp][1], sh_thr[warp][1], lane);
  }
  // lane k = (dz+1)*9 + (dy+1)*3 + (dx+1)
  uint32_t cnt = 0, beg = 0;
  if (lane < 27) {
    const uint32_t h = hash3(base.x - 1 + lane % 3, base.y - 1 + (lane / 3) % 3, base.z - 1 + lane / 9, s.table);
    beg = s.ecs[h];
    const uint32_t en = s.ecs[h + 1];
    // buckets are in ascending edge order and a pair belongs to its smaller
    // edge index: skip straight to the first edge > ei (never counted before)
    uint32_t lo = beg, hi = en > beg ? en : beg;
    while (lo < hi) {
      const uint32_t mid = lo + (hi - lo) / 2u;
      if ((uint32_t)s.es_c[mid].w <= ei) lo = mid + 1u; else hi = mid;
    }
    beg = lo;
    cnt = en > beg ? en - beg : 0u;
  }
  uint32_t incl = cnt;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  if (lane < 27) {
    sh_start[warp][lane] = incl - cnt;
    sh_end[warp][lane] = incl;
    sh_beg[warp][lane] = beg;
  }
  __syncwarp();
  const uint32_t total = __shfl_sync(0xffffffffu, incl, 26);
  uint32_t counted = 0;
  int k = 0;
  uint32_t* queue = sh_q[warp];
  const uint32_t lt_mask = (1u << lane) - 1u;
  for (uint32_t chunk = 0; chunk < total && counted < s.max_search; chunk += 32u * kRounds) {
    // phase 1: counting filter; the first max_search counted pairs are queued
    uint32_t qn = 0;
    for (uint32_t r = 0; r < kRounds; ++r) {
      const uint32_t t = chunk + r * 32u + lane;
      bool pass = false;
      uint32_t slot = 0, eb_l = 0;
      if (t < total) {
        while (t >= sh_end[warp][k]) ++k;
        slot = sh_beg[warp][k] + (t - sh_start[warp][k]);
        // one level of loads for the whole filter
        const int4 bc = s.es_c[slot];
        const float4 bmin = s.es_lo[slot], bmax = s.es_hi[slot];
        const uint2 ebv = make_uint2(__float_as_uint(bmin.w), __float_as_uint(bmax.w));
        const uint32_t eb = (uint32_t)bc.w;
        eb_l = eb;
        pass = ei < eb && !(ebv.x == c.u0 || ebv.x == c.u1 || ebv.y == c.u0 || ebv.y == c.u1) &&
               bc.x == base.x - 1 + k % 3 && bc.y == base.y - 1 + (k / 3) % 3 && bc.z == base.z - 1 + k / 9 &&
               !(c.amin.x > bmax.x || c.amin.y > bmax.y || c.amin.z > bmax.z || c.amax.x < bmin.x ||
                 c.amax.y < bmin.y || c.amax.z < bmin.z);
      }
      const uint32_t b = __ballot_sync(0xffffffffu, pass);
      const uint32_t rank = counted + __popc(b & lt_mask);
      // list mode queues the edge index, otherwise the slot of its records
      if (pass && rank < s.max_search) queue[qn + __popc(b & lt_mask)] = kList ? eb_l : slot;
      const uint32_t nb = __popc(b);
      qn += counted + nb <= s.max_search ? nb : (counted < s.max_search ? s.max_search - counted : 0u);
      counted += nb;
    }
    __syncwarp();
    if constexpr (kList) {
      // phase 2: the queued pairs are appended to this block's segment of
      // the pair list of k_ee_pairs; those past its capacity get their
      // contact work here
      const uint32_t seg = blockIdx.x % kEeSeg, segcap = s.ee_cap / kEeSeg;
      uint32_t lbase = segcap;
      if (lane == 0 && qn && segcap) lbase = atomicAdd(s.ee_n + seg, qn);
      lbase = __shfl_sync(0xffffffffu, lbase, 0);
      for (uint32_t q = lane; q < qn; q += 32u) {
        const uint32_t eb = queue[q];
        if (lbase < segcap && q < segcap - lbase) {
          s.ee_q[size_t(seg) * segcap + lbase + q] = make_uint2(ei, eb);
        } else {
          if (s.rec_ee) record_ee(s, ei, eb);
          ee_listed_pair_call(s, make_uint2(ei, eb));
        }
      }
    } else {
      // phase 2: contact work on the queued pairs
      for (uint32_t q = lane; q < qn; q += 32u) {
        const uint32_t slot = queue[q];
        const uint32_t eb = (uint32_t)s.es_c[slot].w;
        const uint2 ebv = s.es_v[slot];
        const float4 qj = s.p4[ebv.x], qvj = s.p4[ebv.y], xj = s.x4[ebv.x], xvj = s.x4[ebv.y];
        if (s.rec_ee) record_ee(s, ei, eb);
        ee_pair(s, c, th0, th1, eb, ebv.x, ebv.y, qj, qvj, xj, xvj, true);
      }
    }
    __syncwarp();
  }
}

// Grouped variant of k_ee, one lane per edge.  A warp takes 32 consecutive
// slots of the hash-sorted edge order, which are mostly edges of one
// midpoint cell, so they share the reference's 27-cell candidate set.  For
// each distinct cell among its edges the warp builds the cell-matched
// candidates (es_* records) in shared memory, in the reference's visiting
// order (dz outer, dx inner, bucket order), up to kEeChunk at a time; every
// lane of that cell then walks them for its own edge with the reference's
// tests (e_a < e_b, no shared vertex, swept boxes) and per-edge count cap
// (search_count > max_search_iterations ends the edge's search,
// shaders/self_collision_ee_direct.wgsl:330-360).  Counted pairs go to a
// per-warp queue whose contact work (ee_pair) runs 32 pairs at a time.
// The set of counted pairs and the work on each are those of k_ee.
constexpr uint32_t kEeChunk = 128;
constexpr uint32_t kEeWarps = 4;
__global__ void __launch_bounds__(128) k_ee_grouped(SCArgs s) {
  __shared__ int4 ch_c[kEeWarps][kEeChunk];
  __shared__ uint2 ch_v[kEeWarps][kEeChunk];
  __shared__ float4 ch_lo[kEeWarps][kEeChunk], ch_hi[kEeWarps][kEeChunk];
  __shared__ uint32_t q_a[kEeWarps][64], q_b[kEeWarps][64];
  __shared__ uint32_t sh_start[kEeWarps][28], sh_end[kEeWarps][28], sh_beg[kEeWarps][28];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t slot0 = (blockIdx.x * kEeWarps + uint32_t(warp)) * 32u;
  if (slot0 >= s.ne) return;  // whole warp
  const uint32_t my = slot0 + uint32_t(lane);
  const bool valid = my < s.ne;
  // this lane's edge: what the filter needs
  uint32_t ei = 0, u0 = 0, u1 = 0;
  V3 amin = mk(0.f, 0.f, 0.f), amax = amin;
  int4 bc = make_int4(0, 0, 0, 0);
  if (valid) {
    ei = (uint32_t)s.es_c[my].w;
    const EdgeCtx c = edge_ctx(s, ei);
    u0 = c.u0;
    u1 = c.u1;
    amin = c.amin;
    amax = c.amax;
    bc = s.ecell[ei];
  }
  const uint32_t lt_mask = (1u << lane) - 1u;
  uint32_t qn = 0;
  // contact work on the first 32 queued pairs, one per lane
  auto drain32 = [&](uint32_t m) {
    if (uint32_t(lane) < m) {
      const uint32_t a = q_a[warp][lane], b = q_b[warp][lane];
      const EdgeCtx c = edge_ctx(s, a);
      TwoHop th0, th1;
      th0.idx = s.th_idx + s.th_off[c.u0];
      th0.rest = s.th_rest + s.th_off[c.u0];
      th0.n = s.th_off[c.u0 + 1] - s.th_off[c.u0];
      th1.idx = s.th_idx + s.th_off[c.u1];
      th1.rest = s.th_rest + s.th_off[c.u1];
      th1.n = s.th_off[c.u1 + 1] - s.th_off[c.u1];
      const uint2 ebv = s.edges[b];
      if (s.rec_ee) record_ee(s, a, b);
      ee_pair(s, c, th0, th1, b, ebv.x, ebv.y, s.p4[ebv.x], s.p4[ebv.y], s.x4[ebv.x], s.x4[ebv.y], true);
    }
    __syncwarp();
  };
  uint32_t todo = __ballot_sync(0xffffffffu, valid);
  while (todo) {
    const int leader = __ffs(todo) - 1;
    const int32_t cx = __shfl_sync(0xffffffffu, bc.x, leader);
    const int32_t cy = __shfl_sync(0xffffffffu, bc.y, leader);
    const int32_t cz = __shfl_sync(0xffffffffu, bc.z, leader);
    const bool mine = valid && bc.x == cx && bc.y == cy && bc.z == cz;
    todo &= ~__ballot_sync(0xffffffffu, mine);
    // bucket ranges of the cell's 27 neighbours, lane k = (dz+1)*9 + (dy+1)*3 + (dx+1)
    uint32_t cnt = 0, beg = 0;
    if (lane < 27) {
      const uint32_t h = hash3(cx - 1 + lane % 3, cy - 1 + (lane / 3) % 3, cz - 1 + lane / 9, s.table);
      beg = s.ecs[h];
      cnt = s.ecs[h + 1] - beg;
    }
    uint32_t incl = cnt;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    if (lane < 27) {
      sh_start[warp][lane] = incl - cnt;
      sh_end[warp][lane] = incl;
      sh_beg[warp][lane] = beg;
    }
    __syncwarp();
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 26);
    uint32_t counted = 0;
    bool active = mine;
    int k = 0;
    for (uint32_t t0 = 0; t0 < total && __any_sync(0xffffffffu, active);) {
      // the next cell-matched candidates, in order, into the chunk
      uint32_t nch = 0;
      while (t0 < total && nch + 32u <= kEeChunk) {
        const uint32_t t = t0 + uint32_t(lane);
        bool keep = false;
        uint32_t slot = 0;
        int4 c4 = make_int4(0, 0, 0, 0);
        if (t < total) {
          while (t >= sh_end[warp][k]) ++k;
          slot = sh_beg[warp][k] + (t - sh_start[warp][k]);
          c4 = s.es_c[slot];
          keep = c4.x == cx - 1 + k % 3 && c4.y == cy - 1 + (k / 3) % 3 && c4.z == cz - 1 + k / 9;
        }
        const uint32_t b = __ballot_sync(0xffffffffu, keep);
        if (keep) {
          const uint32_t o = nch + __popc(b & lt_mask);
          ch_c[warp][o] = c4;
          ch_v[warp][o] = s.es_v[slot];
          ch_lo[warp][o] = s.es_lo[slot];
          ch_hi[warp][o] = s.es_hi[slot];
        }
        nch += __popc(b);
        t0 += 32u;
      }
      __syncwarp();
      // every lane of the cell walks the chunk for its own edge
      for (uint32_t j = 0; j < nch; ++j) {
        bool pass = false;
        uint32_t eb = 0;
        if (active) {
          const int4 c4 = ch_c[warp][j];
          const uint2 v = ch_v[warp][j];
          eb = (uint32_t)c4.w;
          const float4 lo = ch_lo[warp][j], hi = ch_hi[warp][j];
          pass = ei < eb && !(v.x == u0 || v.x == u1 || v.y == u0 || v.y == u1) &&
                 !(amin.x > hi.x || amin.y > hi.y || amin.z > hi.z || amax.x < lo.x || amax.y < lo.y ||
                   amax.z < lo.z);
          if (pass && ++counted > s.max_search) {
            pass = false;
            active = false;
          }
        }
        const uint32_t b = __ballot_sync(0xffffffffu, pass);
        if (pass) {
          const uint32_t o = qn + __popc(b & lt_mask);
          q_a[warp][o] = ei;
          q_b[warp][o] = eb;
        }
        qn += __popc(b);
        __syncwarp();
        if (qn >= 32u) {
          drain32(32u);
          qn -= 32u;
          if (uint32_t(lane) < qn) {
            q_a[warp][lane] = q_a[warp][32 + lane];
            q_b[warp][lane] = q_b[warp][32 + lane];
          }
          __syncwarp();
        }
      }
      __syncwarp();
    }
  }
  if (qn) drain32(qn);
}

// ---------------- edge colliders: shaders/edge_collision.wgsl:82-276
// Collider edge (mesh.rs:1503-1565): endpoints, the largest thickness and the
// mean friction of its triangles, their summed then normalised normals, and
// bit 0 set when every triangle is single-sided.
struct ColEdge {
  float4 p0t;  // p0, thickness
  float4 p1f;  // p1, friction
  float4 nfl;  // normal, flags bits
};
struct EdgeColArgs {
  uint32_t ne, nce;            // cloth edges, collider edges
  const uint2* edges;
  const float4* x4;
  const float4* p4;
  const ColEdge* ce;
  const uint32_t* cs;          // collider-edge grid: cell starts [table + 1]
  const uint32_t* srt;         // and edge indices
  float cell;
  uint32_t table;
  float mscale, moff;          // contact distance = thickness sum * mscale + moff
  int32_t* acc;
};
// closest points of segments p0-p1 and q0-q1 (edge_collision.wgsl:96-149)
__device__ __forceinline__ float seg_closest(V3 p0, V3 p1, V3 q0, V3 q1, float& s, float& t) {
  const V3 d1 = p1 - p0, d2 = q1 - q0, r = p0 - q0;
  const float a = dot(d1, d1), e = dot(d2, d2), f = dot(d2, r);
  s = 0.0f;
  t = 0.0f;
  if (a <= 1e-12f && e <= 1e-12f) return length(p0 - q0);
  if (a <= 1e-12f) {
    t = clampf(f / e, 0.0f, 1.0f);
  } else {
    const float c = dot(d1, r);
    if (e <= 1e-12f) {
      s = clampf(-c / a, 0.0f, 1.0f);
    } else {
      const float b = dot(d1, d2);
      const float denom = a * e - b * b;
      s = denom > a * e * 1e-7f ? clampf((b * f - c * e) / denom, 0.0f, 1.0f) : 0.0f;
      t = (b * s + f) / e;
      if (t < 0.0f) {
        t = 0.0f;
        s = clampf(-c / a, 0.0f, 1.0f);
      } else if (t > 1.0f) {
        t = 1.0f;
        s = clampf((b - c) / a, 0.0f, 1.0f);
      }
    }
  }
  return length((p0 + d1 * s) - (q0 + d2 * t));
}
// One thread per cloth edge: collider edges of the 27 cells around its
// midpoint; a contact pushes both endpoints out (collider edges do not move)
// through the pin channel of the self-collision accumulator.
__global__ void __launch_bounds__(256) k_edge_collision(EdgeColArgs a) {
  const uint32_t ei = blockIdx.x * blockDim.x + threadIdx.x;
  if (ei >= a.ne || a.nce == 0u) return;
  const uint2 e = a.edges[ei];
  const uint32_t u0 = e.x, u1 = e.y;
  const float w0 = a.x4[u0].w, w1 = a.x4[u1].w;
  if (w0 + w1 <= kEps) return;
  const float4 q0v = a.p4[u0], q1v = a.p4[u1];
  const V3 p0 = mk(q0v), p1 = mk(q1v);
  const V3 pmid = (p0 + p1) * 0.5f;
  const float cth = fmaxf(q0v.w, q1v.w);
  const I3 cc = cell_of(pmid, a.cell);
  const V3 lo = vmin(p0, p1), hi = vmax(p0, p1);
  for (int dz = -1; dz <= 1; ++dz)
    for (int dy = -1; dy <= 1; ++dy)
      for (int dx = -1; dx <= 1; ++dx) {
        const uint32_t h = hash3(cc.x + dx, cc.y + dy, cc.z + dz, a.table);
        const uint32_t st = a.cs[h], en = a.cs[h + 1];
        for (uint32_t k = st; k < en; ++k) {
          const ColEdge ce = a.ce[a.srt[k]];
          const V3 c0 = mk(ce.p0t), c1 = mk(ce.p1f);
          const float tgt = (cth + ce.p0t.w) * a.mscale + a.moff;
          const V3 clo = vmin(c0, c1), chi = vmax(c0, c1);
          if (hi.x + tgt < clo.x || lo.x - tgt > chi.x || hi.y + tgt < clo.y || lo.y - tgt > chi.y ||
              hi.z + tgt < clo.z || lo.z - tgt > chi.z)
            continue;
          float s, t;
          const float dist = seg_closest(p0, p1, c0, c1, s, t);
          if (!(dist < tgt)) continue;
          const V3 diff = (p0 + (p1 - p0) * s) - (c0 + (c1 - c0) * t);
          const V3 en_ = mk(ce.nfl);
          const bool single = (__float_as_uint(ce.nfl.w) & 1u) != 0u;
          const bool has_n = dot(en_, en_) > 0.25f;
          V3 nrm = mk(0.0f, 0.0f, 1.0f);
          float pen = tgt - dist;
          if (single && has_n) {
            const float sp = dot(diff, en_);
            if (sp >= 0.0f) {
              nrm = dist > kEps ? diff / dist : en_;
              pen = tgt - dist;
            } else {
              nrm = en_;
              pen = fminf(tgt - sp, tgt * 2.0f);
            }
          } else if (dist > kEps) {
            nrm = diff / dist;
          } else {
            const V3 cr = cross(p1 - p0, c1 - c0);
            const float cl = length(cr);
            if (cl > kEps) nrm = cr / cl;
          }
          const V3 push = nrm * pen;
          const float ca = 1.0f - s, cb = s;
          const float den = ca * ca * w0 + cb * cb * w1;
          if (den > kEps) {
            const float f0 = fminf((ca * w0) / den, 2.0f), f1 = fminf((cb * w1) / den, 2.0f);
            if (w0 > 0.0f) add_pin(a.acc, u0, push * f0);
            if (w1 > 0.0f) add_pin(a.acc, u1, push * f1);
          }
        }
      }
}

// ---------------- sc_apply: shaders/self_collision_apply.wgsl:57-177
__global__ void k_apply(uint32_t n, const float4* __restrict__ x4, float4* __restrict__ p4,
                        const float* __restrict__ local_len, int32_t* __restrict__ acc, float relief, int enable_relief,
                        float max_disp_ratio) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int4* a4 = reinterpret_cast<int4*>(acc + (size_t)i * A_N);
  const int4 r0 = a4[0], r1 = a4[1], r2 = a4[2], r3 = a4[3];
  const bool pinned = x4[i].w <= 0.0f;
  V3 fd = mk(0.f, 0.f, 0.f);
  const uint32_t cnt = (uint32_t)r0.w;
  if (cnt > 0u && !pinned) {
    const V3 tdp = mk((float)r0.x, (float)r0.y, (float)r0.z) * (1.0f / 1000000.0f);
    V3 ed = tdp / fmaxf(1.0f, sqrtf((float)cnt));
    if (enable_relief) ed = ed * relief;
    const float pl = length(ed);
    const float ratio = max_disp_ratio > 0.0f ? max_disp_ratio : 0.50f;
    const float ms = fminf(local_len[i] * ratio, 0.10f);
    if (pl > ms && pl > kEps) ed = (ed / pl) * ms;
    fd = fd + ed;
  }
  const uint32_t pc = (uint32_t)r1.w;
  V3 avg = mk(0.f, 0.f, 0.f);
  if (pc > 0u && !pinned) avg = (mk((float)r1.x, (float)r1.y, (float)r1.z) * (1.0f / 1000000.0f)) / (float)pc;
  const uint32_t eec = (uint32_t)r3.w;
  if (!pinned) {
    const V3 cp = mk((float)r2.x, (float)r2.y, (float)r2.z) * (1.0f / 1000000.0f);
    const V3 cn = mk((float)r2.w, (float)r3.x, (float)r3.y) * (1.0f / 1000000.0f);
    V3 env = cp + cn;
    if (eec >= 4u) env = env * fmaxf(0.5f, sqrtf(3.0f / (float)eec));
    const V3 z = mk(0.f, 0.f, 0.f);
    fd = fd + (vmax(vmax(env, z), vmax(avg, z)) + vmin(vmin(env, z), vmin(avg, z)));
  }
  const int4 zero = make_int4(0, 0, 0, 0);
  a4[0] = zero; a4[1] = zero; a4[2] = zero; a4[3] = zero;
  if (length(fd) > kEps) {
    float4 p = p4[i];
    p.x += fd.x; p.y += fd.y; p.z += fd.z;
    p4[i] = p;
  }
}

}  // namespace tcloth
