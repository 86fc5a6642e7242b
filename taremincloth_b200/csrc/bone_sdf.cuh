// Bone SDF collider: linear-blend skinning, bone-local triangle preparation,
// the per-bone signed-distance bake into an fp16 x 2 atlas, and the collision
// phase that samples it.
//
// Restates skinning.wgsl:16-43, prep_bone_triangles.wgsl:30-67,
// bake_sdf.wgsl:33-196 and collision.wgsl:116-265 (crates/cloth_core/src/shaders).
// Matrices are stored as the reference's GpuBoneTransform: 16 floats,
// column-major (element (row j, column k) at [k * 4 + j]).
//
// The atlas is a plain device array [depth][height][width] of packed half2
// (distance in the low half, alpha in the high half), the reference's
// Rg16Float texture layout.  Sampling is trilinear with clamp-to-edge in fp32
// (the reference's hardware sampler filters with 8-bit weights; no fixture
// pins either, so this row is parity unpinned against the reference and
// bit-exact against the oracle).
//
// The bake reproduces, per voxel, the reference's sequential scan of a bone's
// triangles (the first triangle within the tie tolerance of the running
// minimum with a larger |projection| wins, so the result depends on the
// order).  It runs in two passes: an order-free search for the minimum
// squared distance m, then the sequential rule over the triangles within a
// small window above m, started at a triangle where the full scan provably
// resets its state (k_bone_bake states the argument).  A triangle, or a tile
// of 32, is skipped only when a conservative bounding-sphere lower bound on
// its squared distance shows that it cannot matter.
#pragma once
#include <cuda_fp16.h>

#include "vmath.cuh"

namespace tcloth {

struct BoneInfo {    // the reference's GpuBoneInfo (collision.wgsl:50-56), 80 B
  float4 aabb_min;   // .w: world bounding-sphere centre x
  float4 aabb_max;   // .w: centre y
  float4 uvw_scale;  // .w: centre z (the bake writes blend_k here)
  float4 uvw_offset; // .w: world bounding-sphere radius
  float4 params;     // friction, thickness, restitution, weight threshold
};
struct BoneXform {   // world and inverse world, column-major
  float m[16];
  float inv[16];
};
struct BakeParams {  // GpuBakeParams (sdf_baker.rs:12-25), 64 B
  float lmin[3];
  uint32_t tri_start;
  float lmax[3];
  uint32_t tri_count;
  uint32_t tile_col, tile_row, tile_layer, res;
  uint32_t total_w, total_h, total_d, row_pitch;
};
struct BakeTri {     // GpuBakeTriangle (sdf_baker.rs:29-38), 64 B
  float4 p0w0, p1w1, p2w2;
  float4 n_bmask;    // normal, open-boundary bit mask (as float)
};

// ((m0 x + m4 y) + m8 z) + m12: column-major matrix times (x, y, z, 1)
__device__ __forceinline__ V3 xform_point(const float* m, V3 p) {
  return mk(((m[0] * p.x + m[4] * p.y) + m[8] * p.z) + m[12], ((m[1] * p.x + m[5] * p.y) + m[9] * p.z) + m[13],
            ((m[2] * p.x + m[6] * p.y) + m[10] * p.z) + m[14]);
}
__device__ __forceinline__ V3 xform_dir(const float* m, V3 p) {
  return mk((m[0] * p.x + m[4] * p.y) + m[8] * p.z, (m[1] * p.x + m[5] * p.y) + m[9] * p.z,
            (m[2] * p.x + m[6] * p.y) + m[10] * p.z);
}

// ---- skinning.wgsl:16-43: rest (pos, normal) + 4 bone indices / weights
__global__ void k_bone_skin(uint32_t nv, const float4* __restrict__ rest_pos, const uint4* __restrict__ bidx,
                            const float4* __restrict__ bw, const float* __restrict__ skin_mats,
                            float4* __restrict__ out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nv) return;
  const V3 pos = mk(rest_pos[i]);
  const uint4 bi = bidx[i];
  const float4 w4 = bw[i];
  const uint32_t ids[4] = {bi.x, bi.y, bi.z, bi.w};
  const float ws[4] = {w4.x, w4.y, w4.z, w4.w};
  V3 p = mk(0.f, 0.f, 0.f);
  float wsum = 0.f;
  for (int k = 0; k < 4; ++k) {
    const float w = ws[k];
    if (w > 0.f) {
      p = p + xform_point(skin_mats + 16 * size_t(ids[k]), pos) * w;
      wsum += w;
    }
  }
  if (wsum <= 1e-6f) p = pos;
  out[i] = make_float4(p.x, p.y, p.z, 1.f);
}

// ---- prep_bone_triangles.wgsl:30-67: world triangle -> bone-local BakeTri
// src = (i0, i1, i2, bone), srcw = (w0, w1, w2, open-boundary mask)
__global__ void k_bone_prep(uint32_t nt, const float4* __restrict__ skinned, const float* __restrict__ inv_mats,
                            const uint4* __restrict__ src, const float4* __restrict__ srcw,
                            BakeTri* __restrict__ out) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  const uint4 s = src[t];
  const float4 w = srcw[t];
  const float* inv = inv_mats + 16 * size_t(s.w);
  const V3 p0 = xform_point(inv, mk(skinned[s.x]));
  const V3 p1 = xform_point(inv, mk(skinned[s.y]));
  const V3 p2 = xform_point(inv, mk(skinned[s.z]));
  const V3 cr = cross(p1 - p0, p2 - p0);
  const float l2 = dot(cr, cr);
  V3 n = mk(0.f, 1.f, 0.f);
  if (l2 > 1e-12f) n = cr * (1.0f / sqrtf(l2));
  out[t] = BakeTri{make_float4(p0.x, p0.y, p0.z, w.x), make_float4(p1.x, p1.y, p1.z, w.y),
                   make_float4(p2.x, p2.y, p2.z, w.z), make_float4(n.x, n.y, n.z, w.w)};
}

// Conservative bounding spheres: per triangle (centroid, max vertex distance),
// and per tile of 32 consecutive triangles of one bone (tiles listed by the
// host: tile k covers [tile_first[k], tile_first[k] + tile_cnt[k])).  Radii are
// widened (x 1.001 + 1e-5) so that fp32 rounding cannot make a bound exceed a
// computed distance.
__global__ void k_bone_tri_spheres(uint32_t nt, const BakeTri* __restrict__ tris, float4* __restrict__ sph) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  const BakeTri q = tris[t];
  const V3 a = mk(q.p0w0), b = mk(q.p1w1), c = mk(q.p2w2);
  const V3 m = (a + b + c) / 3.0f;
  const float r = sqrtf(fmaxf(fmaxf(dot(a - m, a - m), dot(b - m, b - m)), dot(c - m, c - m)));
  sph[t] = make_float4(m.x, m.y, m.z, r * 1.001f + 1e-5f);
}
__global__ void k_bone_tile_spheres(uint32_t ntiles, const uint32_t* __restrict__ tile_first,
                                    const uint32_t* __restrict__ tile_cnt, const float4* __restrict__ sph,
                                    float4* __restrict__ tsph) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ntiles) return;
  const uint32_t f = tile_first[k], c = tile_cnt[k];
  V3 m = mk(0.f, 0.f, 0.f);
  for (uint32_t i = 0; i < c; ++i) m = m + mk(sph[f + i]);
  m = m / float(max(c, 1u));
  float r = 0.f;
  for (uint32_t i = 0; i < c; ++i) {
    const float4 s = sph[f + i];
    r = fmaxf(r, length(mk(s) - m) + s.w);
  }
  tsph[k] = make_float4(m.x, m.y, m.z, r * 1.001f + 1e-5f);
}

__global__ void k_bake_perm_spheres(uint32_t nt, const uint32_t* __restrict__ perm, const float4* __restrict__ sph,
                                    float4* __restrict__ psph) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nt) psph[i] = sph[perm[i]];
}

__device__ __forceinline__ uint32_t pack_half2(float lo, float hi) {
  return (uint32_t)__half_as_ushort(__float2half_rn(lo)) | ((uint32_t)__half_as_ushort(__float2half_rn(hi)) << 16);
}

// Voxel state of the sequential nearest-triangle rule (bake_sdf.wgsl:71-183)
struct BakeState {
  float min_d2, best_abs_proj, best_signed, best_alpha;
  float reach;  // sqrt((min_d2 + tolerance) * 1.0001), refreshed when min_d2 changes
};
__device__ __forceinline__ float bake_reach(float min_d2) {
  return sqrtf((min_d2 + 1e-7f * fmaxf(1.0f, min_d2)) * 1.0001f);
}
// Closest point of the triangle to p (bake_sdf.wgsl:71-130): returns the squared
// distance and leaves p - closest point in `diff` and the barycentrics in `bary`.
__device__ __forceinline__ float bake_closest(V3 p, const BakeTri& tri, V3& diff, V3& bary_out) {
  const V3 a = mk(tri.p0w0), b = mk(tri.p1w1), c = mk(tri.p2w2);
  const V3 ab = b - a, ac = c - a, ap = p - a;
  const float d1 = dot(ab, ap), d2 = dot(ac, ap);
  V3 cp = a;
  V3 bary = mk(1.f, 0.f, 0.f);
  if (d1 <= 0.f && d2 <= 0.f) {
  } else {
    const V3 bp = p - b;
    const float d3 = dot(ab, bp), d4 = dot(ac, bp);
    if (d3 >= 0.f && d4 <= d3) {
      cp = b;
      bary = mk(0.f, 1.f, 0.f);
    } else {
      const float vc = d1 * d4 - d3 * d2;
      if (vc <= 0.f && d1 >= 0.f && d3 <= 0.f) {
        const float v = d1 / (d1 - d3);
        cp = a + ab * v;
        bary = mk(1.f - v, v, 0.f);
      } else {
        const V3 cpv = p - c;
        const float d5 = dot(ab, cpv), d6 = dot(ac, cpv);
        if (d6 >= 0.f && d5 <= d6) {
          cp = c;
          bary = mk(0.f, 0.f, 1.f);
        } else {
          const float vb = d5 * d2 - d1 * d6;
          if (vb <= 0.f && d2 >= 0.f && d6 <= 0.f) {
            const float w = d2 / (d2 - d6);
            cp = a + ac * w;
            bary = mk(1.f - w, 0.f, w);
          } else {
            const float va = d3 * d6 - d5 * d4;
            if (va <= 0.f && (d4 - d3) >= 0.f && (d5 - d6) >= 0.f) {
              const float w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
              cp = b + (c - b) * w;
              bary = mk(0.f, 1.f - w, w);
            } else {
              const float denom = 1.0f / ((va + vb) + vc);
              const float v = vb * denom, w = vc * denom;
              const float u = (1.0f - v) - w;
              cp = (a + ab * v) + ac * w;
              bary = mk(u, v, w);
            }
          }
        }
      }
    }
  }
  diff = p - cp;
  bary_out = bary;
  return dot(diff, diff);
}
// The sequential rule for one triangle whose closest point is known
// (bake_sdf.wgsl:131-183): accepted when closer by more than the tolerance, or
// within it with a larger |projection|.
__device__ __forceinline__ void bake_accept(BakeState& s, const BakeTri& tri, V3 diff, V3 bary, float d_sq) {
  const V3 a = mk(tri.p0w0), b = mk(tri.p1w1), c = mk(tri.p2w2);
  const V3 nrm = mk(tri.n_bmask);
  const float proj = dot(diff, nrm);
  const float aproj = fabsf(proj);
  const float eps_sq = 1e-7f * fmaxf(1.0f, s.min_d2);
  const bool closer = d_sq + eps_sq < s.min_d2;
  const bool tie = fabsf(d_sq - s.min_d2) <= eps_sq && aproj > s.best_abs_proj;
  if (closer || tie) {
    if (d_sq < s.min_d2) {
      s.min_d2 = d_sq;
      s.reach = bake_reach(d_sq);
    }
    s.best_abs_proj = aproj;
    const float d = sqrtf(d_sq);
    float sign = proj >= 0.f ? 1.f : -1.f;
    const uint32_t bmask = uint32_t(tri.n_bmask.w + 0.5f);
    if (bmask != 0u && sign < 0.f) {
      float out_proj = -1.f;
      if ((bmask & 1u) && bary.z <= 1e-5f) {
        const V3 e = cross(b - a, nrm);
        out_proj = fmaxf(out_proj, dot(diff, e / length(e)));
      }
      if ((bmask & 2u) && bary.x <= 1e-5f) {
        const V3 e = cross(c - b, nrm);
        out_proj = fmaxf(out_proj, dot(diff, e / length(e)));
      }
      if ((bmask & 4u) && bary.y <= 1e-5f) {
        const V3 e = cross(a - c, nrm);
        out_proj = fmaxf(out_proj, dot(diff, e / length(e)));
      }
      if (out_proj > 0.f && out_proj >= aproj * 0.25f) sign = 1.f;
    }
    s.best_signed = d * sign;
    s.best_alpha = (bary.x * tri.p0w0.w + bary.y * tri.p1w1.w) + bary.z * tri.p2w2.w;
  }
}
__device__ __forceinline__ void bake_visit(BakeState& s, V3 p, const BakeTri& tri) {
  V3 diff, bary;
  const float d_sq = bake_closest(p, tri, diff, bary);
  bake_accept(s, tri, diff, bary, d_sq);
}
// true when nothing in the sphere can be accepted for this voxel state
// |p - c| - r > reach, tested on squares with a 1e-5 relative margin for
// rounding (no square root per test)
__device__ __forceinline__ bool bake_far_r(float reach, V3 p, float4 sph) {
  const V3 d = p - mk(sph);
  const float rr = sph.w + reach;
  return dot(d, d) > (rr * rr) * 1.00001f;
}
__device__ __forceinline__ bool bake_far(const BakeState& s, V3 p, float4 sph) { return bake_far_r(s.reach, p, sph); }

// ---- bake_sdf.wgsl:33-196.  Block = 8 warps = an 8 x 8 x 4 voxel region of
// one bone; each warp owns a 4 x 4 x 2 brick, a lane one voxel.
// blockIdx.y = entry of `params`.
//
// Per voxel the reference keeps, in triangle order, the state (running
// minimum R of the accepted squared distances, the last accepted triangle),
// accepting d when d + eps(R) < R, or when |d - R| <= eps(R) with a larger
// |projection| (eps(R) = 1e-7 max(1, R)).  The kernel gets the same state
// without an ordered walk over every triangle:
//  A. a first bound on m, the minimum squared distance, from the spatial
//     tile (`perm`, tile spheres `stsph`, sub-tiles of 8 with spheres
//     `ssph8`) nearest to the brick;
//  B. one order-free pass over the spatial tiles, in rings of growing
//     distance from the brick: (voxel, triangle) pairs that the sphere bounds
//     (tile, sub-tile, triangle) cannot rule out are queued and evaluated 32
//     at a time, lowering m by a shared-memory atomic min and listing every
//     triangle with d <= m + W (W = 4e-6 max(1, m)) for its voxel;
//  C. per voxel, the listed window G = {d <= T}, T = m + W, sorted by
//     triangle index, runs through the rule from its first "hard record": a
//     member below T and below every earlier member by more than
//     gap = 1e-6 max(1, qmin).
// Exact: every triangle outside G has d > T, so at a hard record the full
// scan's running minimum is >= qmin and the rule resets the state to that
// triangle alone (closer by more than eps, with room for fp32 rounding); after
// it R < T - gap, so every triangle outside G is rejected.  The full scan thus
// ends in the state of the windowed scan.  A voxel whose list overflowed, or
// whose window holds no hard record, collects its window again in rounds of
// kBakeList sorted indices (retried four times wider, since any T is valid),
// and after three retries takes the ordered full scan over the
// triangle-order tiles (`tsph`).
constexpr uint32_t kBakeList = 16;
constexpr uint32_t kBakeCol = 256;  // threads (voxels) per block: 8 warps, an 8 x 8 x 4 region
__device__ __forceinline__ float bake_window(float m) { return 4.0e-6f * fmaxf(1.0f, m); }
__device__ __forceinline__ V3 bake_voxel(const BakeParams& P, float fr, uint32_t vx, uint32_t vy, uint32_t vz) {
  const V3 uvw = mk((float(vx) + 0.5f) / fr, (float(vy) + 0.5f) / fr, (float(vz) + 0.5f) / fr);
  return mk(P.lmin[0] + uvw.x * (P.lmax[0] - P.lmin[0]), P.lmin[1] + uvw.y * (P.lmax[1] - P.lmin[1]),
            P.lmin[2] + uvw.z * (P.lmax[2] - P.lmin[2]));
}
__device__ __forceinline__ void bake_list_insert(uint32_t* lst, uint32_t& n, bool& more, uint32_t o) {
  // ascending list in shared memory, stride kBakeCol (one column per thread)
  uint32_t j;
  if (n < kBakeList) {
    j = n++;
  } else {
    more = true;
    if (o > lst[(kBakeList - 1) * kBakeCol]) return;
    j = kBakeList - 1;
  }
  while (j > 0 && lst[(j - 1) * kBakeCol] > o) {
    lst[j * kBakeCol] = lst[(j - 1) * kBakeCol];
    --j;
  }
  lst[j * kBakeCol] = o;
}
__device__ __forceinline__ BakeTri bake_tri(const BakeTri* __restrict__ tris, uint32_t o) {
  return BakeTri{__ldg(&tris[o].p0w0), __ldg(&tris[o].p1w1), __ldg(&tris[o].p2w2), __ldg(&tris[o].n_bmask)};
}
// pair evaluation of phase B: voxel slot `slot` of this block at p
__device__ __forceinline__ void bake_pair(const BakeTri* __restrict__ tris, V3 p, uint32_t o, uint32_t slot,
                                          uint32_t* sh_m, uint32_t* sh_cnt, uint32_t* sh_ct, float* sh_cd) {
  V3 diff, bary;
  const float d = bake_closest(p, bake_tri(tris, o), diff, bary);
  if (!(d <= 3.0e38f)) return;  // NaN or inf: never accepted by the rule
  atomicMin(&sh_m[slot], __float_as_uint(d));
  const float mv = __uint_as_float(sh_m[slot]);
  if (d <= mv + bake_window(mv)) {
    const uint32_t c = atomicAdd(&sh_cnt[slot], 1u);
    if (c < kBakeList) {
      sh_ct[c * kBakeCol + slot] = o;
      sh_cd[c * kBakeCol + slot] = d;
    }
  }
}
__global__ void __launch_bounds__(kBakeCol, 3) k_bone_bake(const BakeParams* __restrict__ params, const BakeTri* __restrict__ tris,
                                                   const float4* __restrict__ sph, const float4* __restrict__ tsph,
                                                   const uint32_t* __restrict__ perm, const float4* __restrict__ psph,
                                                   const float4* __restrict__ stsph,
                                                   const float4* __restrict__ ssph8,
                                                   const uint32_t* __restrict__ bone_tile_off,
                                                   const uint32_t* __restrict__ bone_sub_off,
                                                   const uint32_t* __restrict__ param_bone,
                                                   uint32_t* __restrict__ atlas) {
  __shared__ uint32_t sh_list[kBakeList * kBakeCol];  // phase-B candidate indices, then the rounds' lists
  __shared__ float sh_cd[kBakeList * kBakeCol];       // phase-B candidate squared distances
  __shared__ uint32_t sh_m[kBakeCol], sh_cnt[kBakeCol];  // per voxel: running minimum (bits), candidates
  __shared__ uint32_t sh_qv[8][64], sh_qt[8][64];       // per warp: queued (voxel lane, triangle) pairs
  __shared__ float4 sh_sph[8][32];                       // per warp: the current tile's triangle spheres
  __shared__ uint32_t sh_tri[8][32];                     // and triangle indices
  const BakeParams P = params[blockIdx.y];
  const uint32_t res = P.res;
  const uint32_t nbx = (res + 7) / 8, nby = (res + 7) / 8;
  const uint32_t blk = blockIdx.x;
  const uint32_t ox = (blk % nbx) * 8, oy = ((blk / nbx) % nby) * 8, oz = (blk / (nbx * nby)) * 4;
  if (oz >= res) return;  // whole block
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t bx0 = ox + (warp & 1) * 4, by0 = oy + ((warp >> 1) & 1) * 4, bz0 = oz + (warp >> 2) * 2;
  const uint32_t vx = bx0 + (lane & 3), vy = by0 + ((lane >> 2) & 3), vz = bz0 + (lane >> 4);
  const bool valid = vx < res && vy < res && vz < res;
  const float fr = float(res);
  const V3 p = bake_voxel(P, fr, vx, vy, vz);
  const uint32_t t0 = P.tri_start, tn = P.tri_count;
  const uint32_t tile0 = bone_tile_off[param_bone[blockIdx.y]];
  const uint32_t sub0 = bone_sub_off[param_bone[blockIdx.y]];
  const uint32_t ntile = (tn + 31u) / 32u;
  const uint32_t me = threadIdx.x;  // this voxel's slot
  uint32_t* lst = sh_list + me;
  const uint32_t lt_mask = (1u << lane) - 1u;

  // A. first bound on m from the spatial tile nearest to the brick
  uint32_t bt = 0;
  {
    const V3 pc = bake_voxel(P, fr, bx0 + 1, by0 + 1, bz0);
    float bk = 1.0e30f;
    for (uint32_t k = lane; k < ntile; k += 32u) {
      const float4 ts = __ldg(stsph + tile0 + k);
      const float key = length(pc - mk(ts)) - ts.w;
      if (key < bk) { bk = key; bt = k; }
    }
    for (int o = 16; o > 0; o >>= 1) {
      const float ok = __shfl_xor_sync(0xffffffffu, bk, o);
      const uint32_t ot = __shfl_xor_sync(0xffffffffu, bt, o);
      if (ok < bk || (ok == bk && ot < bt)) { bk = ok; bt = ot; }
    }
  }
  float m = 1.0e30f;
  if (valid && bt < ntile) {
    const uint32_t e = min(32u, tn - bt * 32u);
    for (uint32_t q = 0; q < e; ++q) {
      V3 diff, bary;
      const float d = bake_closest(p, bake_tri(tris, __ldg(perm + t0 + bt * 32u + q)), diff, bary);
      m = fminf(m, d);
    }
  }
  sh_m[me] = __float_as_uint(m);
  sh_cnt[me] = 0u;
  __syncwarp();

  // B. order-free pass over the spatial tiles in rings of growing distance
  // from the brick, nearest first, so that m tightens early: (voxel,
  // triangle) pairs that the sphere bound cannot rule out are queued and
  // evaluated 32 at a time, lowering m by a shared-memory atomic min and
  // listing every triangle with d <= m + W for its voxel.  A tile is left out
  // of a ring only when its sphere lies farther from every voxel of the brick
  // than the largest reach sqrt((m + W) * 1.0001) of the brick.
  {
    uint32_t* qv = sh_qv[warp];
    uint32_t* qt = sh_qt[warp];
    float4* ssph = sh_sph[warp];
    uint32_t* stri = sh_tri[warp];
    uint32_t qn = 0;
    const V3 ca = bake_voxel(P, fr, bx0, by0, bz0), cb = bake_voxel(P, fr, bx0 + 3, by0 + 3, bz0 + 1);
    const V3 pc = (ca + cb) * 0.5f;
    const float brad = length(cb - ca) * 0.5f * 1.001f + 1e-5f;  // every voxel of the brick lies within brad of pc
    float lim = -INFINITY;
    while (true) {
      float rmax = 0.f;
      if (valid) {
        const float mv = __uint_as_float(sh_m[me]);
        rmax = sqrtf((mv + bake_window(mv)) * 1.0001f);
      }
      for (int o = 16; o > 0; o >>= 1) rmax = fmaxf(rmax, __shfl_xor_sync(0xffffffffu, rmax, o));
      const float cut = rmax * 1.0001f + 1e-5f;
      float next = 3.0e38f;
      for (uint32_t k = lane; k < ntile; k += 32u) {
        const float4 ts = __ldg(stsph + tile0 + k);
        float key = length(pc - mk(ts)) - ts.w - brad;
        if (!(key == key)) key = -3.0e38f;  // a tile with a NaN sphere goes first
        if (key > lim && key < next) next = key;
      }
      for (int o = 16; o > 0; o >>= 1) next = fminf(next, __shfl_xor_sync(0xffffffffu, next, o));
      if (!(next <= cut)) break;
      const float hi = fminf(cut, next + fmaxf(2.0f * brad, 0.5f * (cut - next)));
      for (uint32_t kb = 0; kb < ntile; kb += 32u) {
        bool sel = false;
        if (kb + lane < ntile) {
          const float4 ts = __ldg(stsph + tile0 + kb + lane);
          float key = length(pc - mk(ts)) - ts.w - brad;
          if (!(key == key)) key = -3.0e38f;
          sel = key > lim && key <= hi;
        }
        uint32_t bm = __ballot_sync(0xffffffffu, sel);
        while (bm) {
          const uint32_t k = kb + uint32_t(__ffs(bm) - 1);
          bm &= bm - 1u;
          const uint32_t e = min(32u, tn - k * 32u);
          __syncwarp();
          if (lane < e) {
            ssph[lane] = __ldg(psph + t0 + k * 32u + lane);
            stri[lane] = __ldg(perm + t0 + k * 32u + lane);
          }
          const uint32_t nsubk = (e + 7u) / 8u;
          float4 s8 = make_float4(0.f, 0.f, 0.f, -1.f);
          if (lane < nsubk) s8 = __ldg(ssph8 + sub0 + k * 4u + lane);
          __syncwarp();
          uint32_t mask = 0u;
          float reach = 0.f;
          if (valid) {
            const float mv = __uint_as_float(sh_m[me]);
            reach = sqrtf((mv + bake_window(mv)) * 1.0001f);
          }
          // sub-tiles of 8 that no voxel of the brick can use are skipped
          uint32_t subs = 0u;
          for (uint32_t u = 0; u < nsubk; ++u) {
            const float4 su = make_float4(__shfl_sync(0xffffffffu, s8.x, u), __shfl_sync(0xffffffffu, s8.y, u),
                                          __shfl_sync(0xffffffffu, s8.z, u), __shfl_sync(0xffffffffu, s8.w, u));
            if (__any_sync(0xffffffffu, valid && !bake_far_r(reach, p, su))) subs |= 1u << u;
          }
          if (valid) {
            for (uint32_t u = 0; u < nsubk; ++u) {
              if (!((subs >> u) & 1u)) continue;
              const uint32_t qe = min(e, 8u * u + 8u);
              for (uint32_t q = 8u * u; q < qe; ++q)
                if (!bake_far_r(reach, p, ssph[q])) mask |= 1u << q;
            }
          }
          while (__any_sync(0xffffffffu, mask != 0u)) {
            const bool has = mask != 0u;
            const uint32_t q = has ? uint32_t(__ffs(mask) - 1) : 0u;
            mask &= mask - 1u;
            const uint32_t b = __ballot_sync(0xffffffffu, has);
            if (has) {
              const uint32_t at = qn + __popc(b & lt_mask);
              qv[at] = lane;
              qt[at] = stri[q];
            }
            qn += __popc(b);
            if (qn >= 32u) {
              __syncwarp();
              const uint32_t v = qv[lane];
              bake_pair(tris, bake_voxel(P, fr, bx0 + (v & 3), by0 + ((v >> 2) & 3), bz0 + (v >> 4)), qt[lane],
                        warp * 32u + v, sh_m, sh_cnt, sh_list, sh_cd);
              __syncwarp();
              qn -= 32u;
              if (lane < qn) {
                qv[lane] = qv[32 + lane];
                qt[lane] = qt[32 + lane];
              }
              // drop candidates above this voxel's window
              const float mv = __uint_as_float(sh_m[me]);
              const uint32_t c = sh_cnt[me];
              if (c > kBakeList / 2 && c <= kBakeList) {
                uint32_t kept = 0;
                for (uint32_t i = 0; i < c; ++i) {
                  const float d = sh_cd[i * kBakeCol + me];
                  if (d <= mv + bake_window(mv)) {
                    lst[kept * kBakeCol] = lst[i * kBakeCol];
                    sh_cd[kept * kBakeCol + me] = d;
                    ++kept;
                  }
                }
                sh_cnt[me] = kept;
              }
              __syncwarp();
            }
          }
        }
      }
      lim = hi;
    }
    __syncwarp();
    if (lane < qn) {
      const uint32_t v = qv[lane];
      bake_pair(tris, bake_voxel(P, fr, bx0 + (v & 3), by0 + ((v >> 2) & 3), bz0 + (v >> 4)), qt[lane],
                warp * 32u + v, sh_m, sh_cnt, sh_list, sh_cd);
    }
    __syncwarp();
  }

  // C. the listed window in the reference's order
  m = __uint_as_float(sh_m[me]);
  const float T0 = m + bake_window(m);
  BakeState s{1e10f, -1.0f, 10.0f, 0.0f, bake_reach(1e10f)};
  bool started = false;
  {
    const uint32_t c = sh_cnt[me];
    if (valid && c <= kBakeList) {
      uint32_t n = 0;
      for (uint32_t i = 0; i < c; ++i) {  // members of G, insertion-sorted by index
        if (!(sh_cd[i * kBakeCol + me] <= T0)) continue;
        const uint32_t o = lst[i * kBakeCol];
        uint32_t j = n++;
        while (j > 0 && lst[(j - 1) * kBakeCol] > o) {
          lst[j * kBakeCol] = lst[(j - 1) * kBakeCol];
          --j;
        }
        lst[j * kBakeCol] = o;
      }
      float qmin = T0;
      for (uint32_t i = 0; i < n; ++i) {
        const uint32_t o = lst[i * kBakeCol];
        const BakeTri tri = bake_tri(tris, o);
        V3 diff, bary;
        const float d_sq = bake_closest(p, tri, diff, bary);
        if (started) {
          bake_accept(s, tri, diff, bary, d_sq);
        } else if (d_sq + 1.0e-6f * fmaxf(1.0f, qmin) < qmin) {
          started = true;
          bake_accept(s, tri, diff, bary, d_sq);
        } else {
          qmin = fminf(qmin, d_sq);
        }
      }
    }
  }
  __syncwarp();

  // the window again in rounds, for voxels whose list overflowed or held no
  // hard record
  float W = bake_window(m);
  float T = m + W;
  float qmin = T;
  uint32_t lo = t0, retries = 0;
  bool need = valid && !started, full = false;
  if (need) s = BakeState{1e10f, -1.0f, 10.0f, 0.0f, bake_reach(1e10f)};
  while (__any_sync(0xffffffffu, need)) {
    const float rT = sqrtf(T * 1.0001f);
    uint32_t n = 0;
    bool more = false;
    for (uint32_t k = 0; k < ntile; ++k) {
      const float r = started ? fminf(rT, s.reach) : rT;
      const bool skip_tile = !need || bake_far_r(r, p, __ldg(stsph + tile0 + k));
      if (__all_sync(0xffffffffu, skip_tile)) continue;
      const uint32_t e = min(32u, tn - k * 32u);
      for (uint32_t q = 0; q < e; ++q) {
        const uint32_t pos = t0 + k * 32u + q;
        if (skip_tile || bake_far_r(started ? fminf(rT, s.reach) : rT, p, __ldg(psph + pos))) continue;
        const uint32_t o = __ldg(perm + pos);
        if (o < lo) continue;
        V3 diff, bary;
        if (bake_closest(p, bake_tri(tris, o), diff, bary) <= T) bake_list_insert(lst, n, more, o);
      }
    }
    if (need) {
      for (uint32_t i = 0; i < n; ++i) {
        const uint32_t o = lst[i * kBakeCol];
        const BakeTri tri = bake_tri(tris, o);
        V3 diff, bary;
        const float d_sq = bake_closest(p, tri, diff, bary);
        if (started) {
          bake_accept(s, tri, diff, bary, d_sq);
        } else if (d_sq + 1.0e-6f * fmaxf(1.0f, qmin) < qmin) {
          started = true;
          bake_accept(s, tri, diff, bary, d_sq);
        } else {
          qmin = fminf(qmin, d_sq);
        }
      }
      if (more) {
        lo = lst[(kBakeList - 1) * kBakeCol] + 1u;
      } else if (started) {
        need = false;
      } else if (retries < 3) {
        ++retries;
        W *= 4.0f;
        T = m + W;
        qmin = T;
        lo = t0;
      } else {
        need = false;
        full = true;
      }
    }
  }

  // the ordered full scan for voxels whose windows held no hard record
  if (__any_sync(0xffffffffu, full)) {
    if (full) s = BakeState{1e10f, -1.0f, 10.0f, 0.0f, bake_reach(1e10f)};
    for (uint32_t k = 0; k < ntile; ++k) {
      const bool skip_tile = !full || bake_far(s, p, __ldg(tsph + tile0 + k));
      if (__all_sync(0xffffffffu, skip_tile)) continue;
      const uint32_t e = min(32u, tn - k * 32u);
      for (uint32_t q = 0; q < e; ++q) {
        const uint32_t t = t0 + k * 32u + q;
        if (skip_tile || bake_far(s, p, __ldg(sph + t))) continue;
        bake_visit(s, p, bake_tri(tris, t));
      }
    }
  }
  if (!valid) return;
  const uint32_t gx = P.tile_col * res + vx, gy = P.tile_row * res + vy, gz = P.tile_layer * res + vz;
  const uint32_t pitch = P.row_pitch > 0u ? P.row_pitch : P.total_w;
  atlas[(size_t(gz) * P.total_h + gy) * pitch + gx] = pack_half2(s.best_signed, s.best_alpha);
}

// ---- single-mesh SDF (bake_mesh_sdf.wgsl:1-121; sdf_baker.rs:1114-1326):
// per voxel the signed distance to the nearest triangle, the first of equal
// distances winning (strict <), the sign from the triangle's normal; alpha 1.
// Voxel centres at local_min + ((i + 0.5) * (1 / dim)) * (local_max - local_min).
// Same brick layout and conservative sphere culling as k_bone_bake (a triangle
// is skipped only when no point of its sphere can come closer).
struct MeshBakeParams {
  float lmin[3], lmax[3];
  uint32_t w, h, d, ntri;
};
__device__ __forceinline__ void mesh_visit(BakeState& s, V3 p, const BakeTri& tri) {
  const V3 a = mk(tri.p0w0), b = mk(tri.p1w1), c = mk(tri.p2w2);
  const V3 ab = b - a, ac = c - a, ap = p - a;
  const float d1 = dot(ab, ap), d2 = dot(ac, ap);
  V3 cp;
  if (d1 <= 0.f && d2 <= 0.f) {
    cp = a;
  } else {
    const V3 bp = p - b;
    const float d3 = dot(ab, bp), d4 = dot(ac, bp);
    const float vc = d1 * d4 - d3 * d2;
    if (d3 >= 0.f && d4 <= d3) {
      cp = b;
    } else if (vc <= 0.f && d1 >= 0.f && d3 <= 0.f) {
      cp = a + ab * (d1 / (d1 - d3));
    } else {
      const V3 cpv = p - c;
      const float d5 = dot(ab, cpv), d6 = dot(ac, cpv);
      const float vb = d5 * d2 - d1 * d6;
      const float va = d3 * d6 - d5 * d4;
      if (d6 >= 0.f && d5 <= d6) {
        cp = c;
      } else if (vb <= 0.f && d2 >= 0.f && d6 <= 0.f) {
        cp = a + ac * (d2 / (d2 - d6));
      } else if (va <= 0.f && (d4 - d3) >= 0.f && (d5 - d6) >= 0.f) {
        cp = b + (c - b) * ((d4 - d3) / ((d4 - d3) + (d5 - d6)));
      } else {
        const float denom = 1.0f / ((va + vb) + vc);
        cp = (a + ab * (vb * denom)) + ac * (vc * denom);
      }
    }
  }
  const V3 diff = p - cp;
  const float d_sq = dot(diff, diff);
  if (d_sq < s.min_d2) {
    s.min_d2 = d_sq;
    s.reach = bake_reach(d_sq);
    s.best_signed = sqrtf(d_sq) * (dot(diff, mk(tri.n_bmask)) >= 0.0f ? 1.0f : -1.0f);
  }
}
__global__ void __launch_bounds__(256) k_mesh_bake(MeshBakeParams P, const BakeTri* __restrict__ tris,
                                                   const float4* __restrict__ sph, const float4* __restrict__ tsph,
                                                   uint32_t* __restrict__ out) {
  const uint32_t bx = (P.w + 7) / 8, by = (P.h + 7) / 8;
  const uint32_t blk = blockIdx.x;
  const uint32_t ox = (blk % bx) * 8, oy = ((blk / bx) % by) * 8, oz = (blk / (bx * by)) * 4;
  if (oz >= P.d) return;  // whole block
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t vx = ox + (warp & 1) * 4 + (lane & 3);
  const uint32_t vy = oy + ((warp >> 1) & 1) * 4 + ((lane >> 2) & 3);
  const uint32_t vz = oz + (warp >> 2) * 2 + (lane >> 4);
  const bool valid = vx < P.w && vy < P.h && vz < P.d;
  const V3 inv = mk(1.0f / float(P.w), 1.0f / float(P.h), 1.0f / float(P.d));
  const V3 uvw = mk((float(vx) + 0.5f) * inv.x, (float(vy) + 0.5f) * inv.y, (float(vz) + 0.5f) * inv.z);
  const V3 p = mk(P.lmin[0] + uvw.x * (P.lmax[0] - P.lmin[0]), P.lmin[1] + uvw.y * (P.lmax[1] - P.lmin[1]),
                  P.lmin[2] + uvw.z * (P.lmax[2] - P.lmin[2]));
  BakeState s{1e10f, -1.0f, 10.0f, 1.0f, bake_reach(1e10f)};
  for (uint32_t k = 0; k * 32u < P.ntri; ++k) {
    const bool skip_tile = !valid || bake_far(s, p, __ldg(tsph + k));
    if (__all_sync(0xffffffffu, skip_tile)) continue;
    const uint32_t e = min(32u, P.ntri - k * 32u);
    for (uint32_t q = 0; q < e; ++q) {
      const uint32_t t = k * 32u + q;
      if (skip_tile || bake_far(s, p, __ldg(sph + t))) continue;
      const BakeTri tri{__ldg(&tris[t].p0w0), __ldg(&tris[t].p1w1), __ldg(&tris[t].p2w2), __ldg(&tris[t].n_bmask)};
      mesh_visit(s, p, tri);
    }
  }
  if (!valid) return;
  out[(size_t(vz) * P.h + vy) * P.w + vx] = pack_half2(s.best_signed, 1.0f);
}

// Point-triangle closest point of bake_mesh_sdf_hier_common.wgsl:30-78 (the
// legacy bake's formula): squared distance and the distance signed by the
// triangle normal.
__device__ __forceinline__ float mesh_tri_dist(V3 p, const BakeTri& tri, float& signed_d) {
  const V3 a = mk(tri.p0w0), b = mk(tri.p1w1), c = mk(tri.p2w2);
  const V3 ab = b - a, ac = c - a, ap = p - a;
  const float d1 = dot(ab, ap), d2 = dot(ac, ap);
  V3 cp;
  if (d1 <= 0.f && d2 <= 0.f) {
    cp = a;
  } else {
    const V3 bp = p - b;
    const float d3 = dot(ab, bp), d4 = dot(ac, bp);
    const float vc = d1 * d4 - d3 * d2;
    if (d3 >= 0.f && d4 <= d3) {
      cp = b;
    } else if (vc <= 0.f && d1 >= 0.f && d3 <= 0.f) {
      cp = a + ab * (d1 / (d1 - d3));
    } else {
      const V3 cpv = p - c;
      const float d5 = dot(ab, cpv), d6 = dot(ac, cpv);
      const float vb = d5 * d2 - d1 * d6;
      const float va = d3 * d6 - d5 * d4;
      if (d6 >= 0.f && d5 <= d6) {
        cp = c;
      } else if (vb <= 0.f && d2 >= 0.f && d6 <= 0.f) {
        cp = a + ac * (d2 / (d2 - d6));
      } else if (va <= 0.f && (d4 - d3) >= 0.f && (d5 - d6) >= 0.f) {
        cp = b + (c - b) * ((d4 - d3) / ((d4 - d3) + (d5 - d6)));
      } else {
        const float denom = 1.0f / ((va + vb) + vc);
        cp = (a + ab * (vb * denom)) + ac * (vc * denom);
      }
    }
  }
  const V3 diff = p - cp;
  const float d_sq = dot(diff, diff);
  signed_d = sqrtf(d_sq) * (dot(diff, mk(tri.n_bmask)) >= 0.0f ? 1.0f : -1.0f);
  return d_sq;
}

// ---- hierarchical bake pass 1, the coarse grid
// (bake_mesh_sdf_hier_coarse_main.wgsl; sdf_baker.rs:1328-1600): per coarse
// voxel the 8 nearest triangles by an in-order insertion with strict <
// (equal distances keep the earlier triangle), the signed distance of the
// first packed as fp16 (distance, 1), the 8 indices at voxel * 8 + k.
// Voxels are linear (z, y, x).  The brick layout and sphere culling of
// k_mesh_bake skip a triangle only when no point of its sphere can come
// under the 8th distance, which the insertion needs.
__global__ void __launch_bounds__(256) k_mesh_bake_coarse(MeshBakeParams P, const BakeTri* __restrict__ tris,
                                                          const float4* __restrict__ sph,
                                                          const float4* __restrict__ tsph,
                                                          uint32_t* __restrict__ dist, uint32_t* __restrict__ near8) {
  const uint32_t bx = (P.w + 7) / 8, by = (P.h + 7) / 8;
  const uint32_t blk = blockIdx.x;
  const uint32_t ox = (blk % bx) * 8, oy = ((blk / bx) % by) * 8, oz = (blk / (bx * by)) * 4;
  if (oz >= P.d) return;  // whole block
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t vx = ox + (warp & 1) * 4 + (lane & 3);
  const uint32_t vy = oy + ((warp >> 1) & 1) * 4 + ((lane >> 2) & 3);
  const uint32_t vz = oz + (warp >> 2) * 2 + (lane >> 4);
  const bool valid = vx < P.w && vy < P.h && vz < P.d;
  const V3 inv = mk(1.0f / float(P.w), 1.0f / float(P.h), 1.0f / float(P.d));
  const V3 uvw = mk((float(vx) + 0.5f) * inv.x, (float(vy) + 0.5f) * inv.y, (float(vz) + 0.5f) * inv.z);
  const V3 p = mk(P.lmin[0] + uvw.x * (P.lmax[0] - P.lmin[0]), P.lmin[1] + uvw.y * (P.lmax[1] - P.lmin[1]),
                  P.lmin[2] + uvw.z * (P.lmax[2] - P.lmin[2]));
  float bsq[8], bsg[8];
  uint32_t bid[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) { bsq[k] = 1e10f; bsg[k] = 10.0f; bid[k] = 0u; }
  BakeState s{1e10f, -1.0f, 10.0f, 1.0f, bake_reach(1e10f)};
  for (uint32_t k = 0; k * 32u < P.ntri; ++k) {
    const bool skip_tile = !valid || bake_far(s, p, __ldg(tsph + k));
    if (__all_sync(0xffffffffu, skip_tile)) continue;
    const uint32_t e = min(32u, P.ntri - k * 32u);
    for (uint32_t q = 0; q < e; ++q) {
      const uint32_t t = k * 32u + q;
      if (skip_tile || bake_far(s, p, __ldg(sph + t))) continue;
      const BakeTri tri{__ldg(&tris[t].p0w0), __ldg(&tris[t].p1w1), __ldg(&tris[t].p2w2), __ldg(&tris[t].n_bmask)};
      float sd;
      const float dsq = mesh_tri_dist(p, tri, sd);
      if (dsq < bsq[7]) {
        float isq = dsq, isg = sd;
        uint32_t iid = t;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          if (isq < bsq[j]) {
            const float tq = bsq[j], ts = bsg[j];
            const uint32_t ti = bid[j];
            bsq[j] = isq; bsg[j] = isg; bid[j] = iid;
            isq = tq; isg = ts; iid = ti;
          }
        }
        s.min_d2 = bsq[7];
        s.reach = bake_reach(bsq[7]);
      }
    }
  }
  if (!valid) return;
  const size_t flat = (size_t(vz) * P.h + vy) * P.w + vx;
  dist[flat] = pack_half2(bsg[0], 1.0f);
#pragma unroll
  for (int k = 0; k < 8; ++k) near8[flat * 8 + k] = bid[k];
}

// ---- sampling: trilinear, clamp to edge, texel centres at (i + 0.5) / size
__device__ __forceinline__ float2 unpack_half2(uint32_t u) {
  return make_float2(__half2float(__ushort_as_half((unsigned short)(u & 0xFFFFu))),
                     __half2float(__ushort_as_half((unsigned short)(u >> 16))));
}
struct BoneSdfArgs {
  const BoneInfo* info;
  const BoneXform* xf;
  const uint32_t* atlas;
  uint32_t nbones, w, h, d;
};
__device__ __forceinline__ float2 atlas_fetch(const BoneSdfArgs& a, int x, int y, int z) {
  return unpack_half2(__ldg(a.atlas + (size_t(z) * a.h + y) * a.w + x));
}
__device__ __forceinline__ float2 sample_atlas(const BoneSdfArgs& a, V3 uvw) {
  const float fx = uvw.x * float(a.w) - 0.5f, fy = uvw.y * float(a.h) - 0.5f, fz = uvw.z * float(a.d) - 0.5f;
  const float flx = floorf(fx), fly = floorf(fy), flz = floorf(fz);
  const float tx = fx - flx, ty = fy - fly, tz = fz - flz;
  const int ix = int(flx), iy = int(fly), iz = int(flz);
  const int x0 = min(max(ix, 0), int(a.w) - 1), x1 = min(max(ix + 1, 0), int(a.w) - 1);
  const int y0 = min(max(iy, 0), int(a.h) - 1), y1 = min(max(iy + 1, 0), int(a.h) - 1);
  const int z0 = min(max(iz, 0), int(a.d) - 1), z1 = min(max(iz + 1, 0), int(a.d) - 1);
  auto lx = [&](int y, int z) {
    const float2 p = atlas_fetch(a, x0, y, z), q = atlas_fetch(a, x1, y, z);
    return make_float2(p.x * (1.f - tx) + q.x * tx, p.y * (1.f - tx) + q.y * tx);
  };
  auto ly = [&](int z) {
    const float2 p = lx(y0, z), q = lx(y1, z);
    return make_float2(p.x * (1.f - ty) + q.x * ty, p.y * (1.f - ty) + q.y * ty);
  };
  const float2 p = ly(z0), q = ly(z1);
  return make_float2(p.x * (1.f - tz) + q.x * tz, p.y * (1.f - tz) + q.y * tz);
}
__device__ __forceinline__ float smoothstep_f(float e0, float e1, float x) {
  const float t = clampf((x - e0) / (e1 - e0), 0.f, 1.f);
  return (t * t) * (3.0f - 2.0f * t);
}

// collision.wgsl:123-265 (solve_bone_sdf_collision).  Returns true with the
// best contact (target position, normal, friction, restitution) when the
// vertex penetrates target_dist of some bone.
__device__ __noinline__ bool bone_sdf_contact(const BoneSdfArgs& a, V3 p, float vth, bool has_mesh, V3& target,
                                              V3& nrm_out, float& fric, float& rest) {
  float best = 1e6f, best_target = 0.f;
  V3 best_n = mk(0.f, 0.f, 0.f);
  float bf = 0.f, br = 0.f;
  uint32_t hits = 0;
  for (uint32_t b = 0; b < a.nbones; ++b) {
    const BoneInfo info = a.info[b];
    const float wr = info.uvw_offset.w;
    if (wr > 0.f) {
      const V3 dw = p - mk(info.aabb_min.w, info.aabb_max.w, info.uvw_scale.w);
      const float rt = wr + vth;
      if (dot(dw, dw) > rt * rt) continue;
    }
    const BoneXform& X = a.xf[b];
    const V3 pl = xform_point(X.inv, p);
    const float target_dist = vth + info.params.y;
    const float margin = target_dist + 0.05f;
    if (pl.x < info.aabb_min.x - margin || pl.x > info.aabb_max.x + margin || pl.y < info.aabb_min.y - margin ||
        pl.y > info.aabb_max.y + margin || pl.z < info.aabb_min.z - margin || pl.z > info.aabb_max.z + margin)
      continue;
    const V3 sc = mk(info.uvw_scale), of = mk(info.uvw_offset);
    const V3 uvw = mk(pl.x * sc.x + of.x, pl.y * sc.y + of.y, pl.z * sc.z + of.z);
    const V3 umin = mk(info.aabb_min.x * sc.x + of.x, info.aabb_min.y * sc.y + of.y, info.aabb_min.z * sc.z + of.z);
    const V3 umax = mk(info.aabb_max.x * sc.x + of.x, info.aabb_max.y * sc.y + of.y, info.aabb_max.z * sc.z + of.z);
    if (uvw.x < umin.x || uvw.x > umax.x || uvw.y < umin.y || uvw.y > umax.y || uvw.z < umin.z || uvw.z > umax.z)
      continue;
    const V3 es = (umax - umin) * (a.nbones == 1u ? 0.002f : 0.015f);
    const V3 lo = umin + es, hi = umax - es;
    const V3 us = mk(clampf(uvw.x, lo.x, hi.x), clampf(uvw.y, lo.y, hi.y), clampf(uvw.z, lo.z, hi.z));
    const float2 sv = sample_atlas(a, us);
    const float raw = sv.x, alpha = sv.y;
    const float thr = fmaxf(info.params.w, 0.01f);
    float retract = 0.f;
    if (has_mesh) retract = (1.0f - smoothstep_f(thr, 0.7f, alpha)) * 0.06f;
    const float eff = alpha > thr ? raw + retract : 10.0f;
    if (eff < target_dist) {
      const V3 eu = sc * 0.005f;
      const float dxp = sample_atlas(a, mk(clampf(uvw.x + eu.x, lo.x, hi.x), us.y, us.z)).x;
      const float dxn = sample_atlas(a, mk(clampf(uvw.x - eu.x, lo.x, hi.x), us.y, us.z)).x;
      const float dyp = sample_atlas(a, mk(us.x, clampf(uvw.y + eu.y, lo.y, hi.y), us.z)).x;
      const float dyn = sample_atlas(a, mk(us.x, clampf(uvw.y - eu.y, lo.y, hi.y), us.z)).x;
      const float dzp = sample_atlas(a, mk(us.x, us.y, clampf(uvw.z + eu.z, lo.z, hi.z))).x;
      const float dzn = sample_atlas(a, mk(us.x, us.y, clampf(uvw.z - eu.z, lo.z, hi.z))).x;
      float dx = dxp - dxn, dy = dyp - dyn, dz = dzp - dzn;
      if (fabsf(dx) < 1e-6f) dx = uvw.x < (lo.x + hi.x) * 0.5f ? dxp - raw : raw - dxn;
      if (fabsf(dy) < 1e-6f) dy = uvw.y < (lo.y + hi.y) * 0.5f ? dyp - raw : raw - dyn;
      if (fabsf(dz) < 1e-6f) dz = uvw.z < (lo.z + hi.z) * 0.5f ? dzp - raw : raw - dzn;
      const V3 g = mk(dx, dy, dz);
      const float gl = length(g);
      V3 nl = mk(0.f, 0.f, 1.f);
      if (gl > 1e-6f) {
        nl = g / gl;
      } else {
        const V3 cl = (mk(info.aabb_min) + mk(info.aabb_max)) * 0.5f;
        const V3 dc = pl - cl;
        const float lc = length(dc);
        if (lc > 1e-6f) nl = dc / lc;
      }
      const V3 nwr = xform_dir(X.m, nl);
      const V3 nw = nwr / length(nwr);
      if (hits == 0u || eff < best) {
        best = eff;
        best_n = nw;
        bf = info.params.x;
        br = info.params.z;
        best_target = target_dist;
      }
      ++hits;
    }
  }
  if (hits > 0u && best < best_target) {
    target = p + best_n * (best_target - best);
    nrm_out = best_n;
    fric = bf;
    rest = br;
    return true;
  }
  return false;
}

// ---- hierarchical bake pass 2, the fine grid
// (bake_mesh_sdf_hier_fine_main.wgsl; sdf_baker.rs:1603-1900): a fine voxel
// whose parent coarse cell is at least band + half a cell diagonal from the
// surface copies the parent's packed value; else the candidates are the
// 8 nearest triangles of the 5 x 5 x 5 coarse cells around the parent
// (clamped), visited z, y, x, with an AABB lower bound that skips a triangle
// unable to enter the running top 2; when the top 2 lie within 0.2 mm with
// opposite signs the voxel is rescanned over every triangle in order.
struct HierFineParams {
  uint32_t cw, ch, cd;
  float band;
};
__device__ __forceinline__ void hier_eval(V3 p, const BakeTri* __restrict__ tris, uint32_t ntri, uint32_t ti,
                                          uint32_t& best_i, float& best_sq, float& best_sg, float& sec_sq,
                                          float& sec_sg) {
  if (ti >= ntri || ti == best_i) return;
  const BakeTri tri{__ldg(&tris[ti].p0w0), __ldg(&tris[ti].p1w1), __ldg(&tris[ti].p2w2), __ldg(&tris[ti].n_bmask)};
  const V3 a = mk(tri.p0w0), b = mk(tri.p1w1), c = mk(tri.p2w2);
  const V3 tmin = vmin(a, vmin(b, c)), tmax = vmax(a, vmax(b, c));
  const V3 z = mk(0.0f, 0.0f, 0.0f);
  const V3 dv = vmax(tmin - p, z) + vmax(p - tmax, z);
  if (dot(dv, dv) >= sec_sq) return;
  float sd;
  const float dsq = mesh_tri_dist(p, tri, sd);
  if (dsq < best_sq) {
    sec_sq = best_sq; sec_sg = best_sg;
    best_sq = dsq; best_sg = sd; best_i = ti;
  } else if (dsq < sec_sq) {
    sec_sq = dsq; sec_sg = sd;
  }
}
__global__ void __launch_bounds__(128) k_mesh_bake_fine(MeshBakeParams P, HierFineParams H,
                                                        const BakeTri* __restrict__ tris,
                                                        const uint32_t* __restrict__ cdist,
                                                        const uint32_t* __restrict__ cnear, uint32_t* __restrict__ out) {
  const size_t flat = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const size_t nvox = size_t(P.w) * P.h * P.d;
  if (flat >= nvox) return;
  const uint32_t vx = uint32_t(flat % P.w), vy = uint32_t((flat / P.w) % P.h), vz = uint32_t(flat / (size_t(P.w) * P.h));
  const V3 lmin = mk(P.lmin[0], P.lmin[1], P.lmin[2]);
  const V3 size = mk(P.lmax[0], P.lmax[1], P.lmax[2]) - lmin;
  const V3 inv = mk(1.0f / float(P.w), 1.0f / float(P.h), 1.0f / float(P.d));
  const V3 uvw = mk((float(vx) + 0.5f) * inv.x, (float(vy) + 0.5f) * inv.y, (float(vz) + 0.5f) * inv.z);
  const V3 p = mk(lmin.x + uvw.x * size.x, lmin.y + uvw.y * size.y, lmin.z + uvw.z * size.z);
  const V3 cdf = mk(float(H.cw), float(H.ch), float(H.cd));
  const V3 spacing = mk(size.x / cdf.x, size.y / cdf.y, size.z / cdf.z);
  const float halfdiag = 0.5f * length(spacing);
  const V3 rel = p - lmin;
  const int32_t hx = f2i(cdf.x) - 1, hy = f2i(cdf.y) - 1, hz = f2i(cdf.z) - 1;
  const int32_t px = min(max(f2i(floorf(rel.x / spacing.x)), 0), hx);
  const int32_t py = min(max(f2i(floorf(rel.y / spacing.y)), 0), hy);
  const int32_t pz = min(max(f2i(floorf(rel.z / spacing.z)), 0), hz);
  const uint32_t pidx = (uint32_t(pz) * H.ch + uint32_t(py)) * H.cw + uint32_t(px);
  const uint32_t dc_packed = cdist[pidx];
  const float dc = unpack_half2(dc_packed).x;
  if (fabsf(dc) - halfdiag >= H.band) {
    out[flat] = dc_packed;
    return;
  }
  uint32_t best_i = 0xFFFFFFFFu;
  float best_sq = 1e10f, best_sg = 10.0f, sec_sq = 1e10f, sec_sg = 10.0f;
  for (int dz = -2; dz <= 2; ++dz)
    for (int dy = -2; dy <= 2; ++dy)
      for (int dx = -2; dx <= 2; ++dx) {
        const int32_t cx = min(max(px + dx, 0), hx), cy = min(max(py + dy, 0), hy), cz = min(max(pz + dz, 0), hz);
        const size_t base = (size_t(uint32_t(cz) * H.ch + uint32_t(cy)) * H.cw + uint32_t(cx)) * 8u;
        for (uint32_t k = 0; k < 8u; ++k)
          hier_eval(p, tris, P.ntri, __ldg(cnear + base + k), best_i, best_sq, best_sg, sec_sq, sec_sg);
      }
  bool amb = (sqrtf(sec_sq) - sqrtf(best_sq) <= 0.0002f);
  if (amb) {
    const float sb = best_sg >= 0.0f ? 1.0f : -1.0f, ss = sec_sg >= 0.0f ? 1.0f : -1.0f;
    amb = sb != ss;
  }
  if (amb) {
    best_sq = 1e10f;
    best_sg = 10.0f;
    for (uint32_t t = 0; t < P.ntri; ++t) {
      const BakeTri tri{__ldg(&tris[t].p0w0), __ldg(&tris[t].p1w1), __ldg(&tris[t].p2w2), __ldg(&tris[t].n_bmask)};
      float sd;
      const float dsq = mesh_tri_dist(p, tri, sd);
      if (dsq < best_sq) { best_sq = dsq; best_sg = sd; }
    }
  }
  out[flat] = pack_half2(best_sg, 1.0f);
}

}  // namespace tcloth
