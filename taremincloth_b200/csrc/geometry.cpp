// Self-intersection search over a triangle mesh, host only.
//
// Same contract as the reference's find_triangle_intersections
// (crates/cloth_core/src/geometry.rs:506-633, exported by
// crates/cloth_py/src/lib.rs:856-879): all face pairs (f0 < f1, ascending)
// whose triangles share at least one point, skipping degenerate faces and,
// with ignore_adjacent, pairs that share a vertex -- or, with sewing springs,
// a vertex cluster joined by springs (union-find over the spring graph,
// geometry.rs:484-506).
//
// Broad phase: a uniform grid over the triangles' bounding boxes, cell size
// from the caller or max(2 x mean edge length, span / 128, 1e-4) as the
// reference's NumPy path chooses it (python/taremin_cloth/analysis.py:690-700);
// each triangle visits the cells its box covers and tests the later
// triangles found there once (a per-triangle stamp).  Narrow phase: the
// interval-overlap test of Moller, "A Fast Triangle-Triangle Intersection
// Test" (JGT 1997) in double precision: each triangle against the other's
// plane, then the two intervals the planes cut along their common line;
// coplanar pairs fall back to 2D edge crossings and containment.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <unordered_map>
#include <vector>

namespace tcloth {
namespace {

struct D3 {
  double x, y, z;
};
inline D3 sub(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline D3 crs(D3 a, D3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline double comp(D3 a, int k) { return k == 0 ? a.x : (k == 1 ? a.y : a.z); }

// the part of a triangle's edges that lies on the other triangle's plane,
// as an interval of the projection v along the planes' common line
bool plane_interval(const double v[3], const double d[3], double& lo, double& hi) {
  bool any = false;
  auto add = [&](double t) {
    if (!any) { lo = hi = t; any = true; }
    else { lo = std::min(lo, t); hi = std::max(hi, t); }
  };
  for (int i = 0; i < 3; ++i)
    if (d[i] == 0.0) add(v[i]);
  for (int i = 0; i < 3; ++i) {
    const int j = (i + 1) % 3;
    if ((d[i] < 0.0 && d[j] > 0.0) || (d[i] > 0.0 && d[j] < 0.0)) add(v[i] + (v[j] - v[i]) * d[i] / (d[i] - d[j]));
  }
  return any;
}

// 2D: do closed segments ab and cd share a point?
bool seg_seg_2d(const double a[2], const double b[2], const double c[2], const double d[2]) {
  auto orient = [](const double p[2], const double q[2], const double r[2]) {
    return (q[0] - p[0]) * (r[1] - p[1]) - (q[1] - p[1]) * (r[0] - p[0]);
  };
  auto on_seg = [](const double p[2], const double q[2], const double r[2]) {
    return std::min(p[0], q[0]) <= r[0] && r[0] <= std::max(p[0], q[0]) && std::min(p[1], q[1]) <= r[1] &&
           r[1] <= std::max(p[1], q[1]);
  };
  const double o1 = orient(a, b, c), o2 = orient(a, b, d), o3 = orient(c, d, a), o4 = orient(c, d, b);
  if (((o1 > 0 && o2 < 0) || (o1 < 0 && o2 > 0)) && ((o3 > 0 && o4 < 0) || (o3 < 0 && o4 > 0))) return true;
  if (o1 == 0 && on_seg(a, b, c)) return true;
  if (o2 == 0 && on_seg(a, b, d)) return true;
  if (o3 == 0 && on_seg(c, d, a)) return true;
  if (o4 == 0 && on_seg(c, d, b)) return true;
  return false;
}

bool point_in_tri_2d(const double p[2], const double t[3][2]) {
  double s[3];
  for (int i = 0; i < 3; ++i) {
    const double* a = t[i];
    const double* b = t[(i + 1) % 3];
    s[i] = (b[0] - a[0]) * (p[1] - a[1]) - (b[1] - a[1]) * (p[0] - a[0]);
  }
  return (s[0] >= 0 && s[1] >= 0 && s[2] >= 0) || (s[0] <= 0 && s[1] <= 0 && s[2] <= 0);
}

bool coplanar_overlap(const D3 p[3], const D3 q[3], D3 n) {
  // drop the axis along which the normal is largest
  const double ax = std::fabs(n.x), ay = std::fabs(n.y), az = std::fabs(n.z);
  const int drop = (ax >= ay && ax >= az) ? 0 : (ay >= az ? 1 : 2);
  const int i0 = drop == 0 ? 1 : 0, i1 = drop == 2 ? 1 : 2;
  double P[3][2], Q[3][2];
  for (int k = 0; k < 3; ++k) {
    P[k][0] = comp(p[k], i0); P[k][1] = comp(p[k], i1);
    Q[k][0] = comp(q[k], i0); Q[k][1] = comp(q[k], i1);
  }
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b)
      if (seg_seg_2d(P[a], P[(a + 1) % 3], Q[b], Q[(b + 1) % 3])) return true;
  return point_in_tri_2d(P[0], Q) || point_in_tri_2d(Q[0], P);
}

bool tri_tri(const D3 p[3], const D3 q[3]) {
  const D3 nq = crs(sub(q[1], q[0]), sub(q[2], q[0]));
  const double oq = dot(nq, q[0]);
  double dp[3];
  for (int i = 0; i < 3; ++i) dp[i] = dot(nq, p[i]) - oq;
  if ((dp[0] > 0 && dp[1] > 0 && dp[2] > 0) || (dp[0] < 0 && dp[1] < 0 && dp[2] < 0)) return false;
  const D3 np_ = crs(sub(p[1], p[0]), sub(p[2], p[0]));
  const double op = dot(np_, p[0]);
  double dq[3];
  for (int i = 0; i < 3; ++i) dq[i] = dot(np_, q[i]) - op;
  if ((dq[0] > 0 && dq[1] > 0 && dq[2] > 0) || (dq[0] < 0 && dq[1] < 0 && dq[2] < 0)) return false;
  if (dp[0] == 0 && dp[1] == 0 && dp[2] == 0) return coplanar_overlap(p, q, nq);
  const D3 L = crs(np_, nq);
  const double lx = std::fabs(L.x), ly = std::fabs(L.y), lz = std::fabs(L.z);
  const int k = (lx >= ly && lx >= lz) ? 0 : (ly >= lz ? 1 : 2);
  const double vp[3] = {comp(p[0], k), comp(p[1], k), comp(p[2], k)};
  const double vq[3] = {comp(q[0], k), comp(q[1], k), comp(q[2], k)};
  double a0, a1, b0, b1;
  if (!plane_interval(vp, dp, a0, a1) || !plane_interval(vq, dq, b0, b1)) return false;
  return std::max(a0, b0) <= std::min(a1, b1);
}

uint32_t find_root(std::vector<uint32_t>& parent, uint32_t x) {
  while (parent[x] != x) {
    parent[x] = parent[parent[x]];
    x = parent[x];
  }
  return x;
}

}  // namespace

std::vector<uint32_t> find_triangle_intersections(const float* pos, uint32_t n, const uint32_t* faces, uint32_t nf,
                                                  bool ignore_adjacent, float cell_size, const uint32_t* sew,
                                                  uint32_t nsew) {
  std::vector<uint32_t> out;
  // valid faces: in range and non-degenerate by index
  std::vector<uint32_t> fid;
  for (uint32_t f = 0; f < nf; ++f) {
    const uint32_t a = faces[3 * f], b = faces[3 * f + 1], c = faces[3 * f + 2];
    if (a >= n || b >= n || c >= n || a == b || b == c || a == c) continue;
    fid.push_back(f);
  }
  const size_t m = fid.size();
  if (m < 2) return out;
  std::vector<uint32_t> rep(n);
  for (uint32_t v = 0; v < n; ++v) rep[v] = v;
  if (ignore_adjacent && sew && nsew) {
    for (uint32_t s = 0; s < nsew; ++s) {
      const uint32_t a = sew[2 * s], b = sew[2 * s + 1];
      if (a >= n || b >= n) continue;
      const uint32_t ra = find_root(rep, a), rb = find_root(rep, b);
      if (ra != rb) rep[std::max(ra, rb)] = std::min(ra, rb);
    }
    for (uint32_t v = 0; v < n; ++v) rep[v] = find_root(rep, v);
  }
  std::vector<D3> tri(3 * m);
  std::vector<double> lo(3 * m), hi(3 * m);
  double gmin[3] = {INFINITY, INFINITY, INFINITY}, gmax[3] = {-INFINITY, -INFINITY, -INFINITY};
  double edge_sum = 0.0;
  for (size_t k = 0; k < m; ++k) {
    for (int c = 0; c < 3; ++c) {
      const float* p = pos + 3 * size_t(faces[3 * fid[k] + c]);
      tri[3 * k + c] = {p[0], p[1], p[2]};
    }
    for (int a = 0; a < 3; ++a) {
      double l = INFINITY, h = -INFINITY;
      for (int c = 0; c < 3; ++c) {
        const double v = comp(tri[3 * k + c], a);
        l = std::min(l, v);
        h = std::max(h, v);
      }
      lo[3 * k + a] = l;
      hi[3 * k + a] = h;
      gmin[a] = std::min(gmin[a], l);
      gmax[a] = std::max(gmax[a], h);
    }
    for (int c = 0; c < 3; ++c) {
      const D3 e = sub(tri[3 * k + (c + 1) % 3], tri[3 * k + c]);
      edge_sum += std::sqrt(dot(e, e)) / 3.0;
    }
  }
  const double span = std::max({gmax[0] - gmin[0], gmax[1] - gmin[1], gmax[2] - gmin[2]});
  double cell = cell_size > 0.f ? double(cell_size) : 2.0 * edge_sum / double(m);
  cell = std::max({cell, span / 128.0, 1e-4});
  auto key = [](int64_t x, int64_t y, int64_t z) {
    return (uint64_t(x & 0x1FFFFF) << 42) | (uint64_t(y & 0x1FFFFF) << 21) | uint64_t(z & 0x1FFFFF);
  };
  std::unordered_map<uint64_t, std::vector<uint32_t>> grid;
  grid.reserve(m * 2);
  auto cells_of = [&](size_t k, int64_t c0[3], int64_t c1[3]) {
    for (int a = 0; a < 3; ++a) {
      c0[a] = int64_t(std::floor(lo[3 * k + a] / cell));
      c1[a] = int64_t(std::floor(hi[3 * k + a] / cell));
    }
  };
  for (size_t k = 0; k < m; ++k) {
    int64_t c0[3], c1[3];
    cells_of(k, c0, c1);
    for (int64_t x = c0[0]; x <= c1[0]; ++x)
      for (int64_t y = c0[1]; y <= c1[1]; ++y)
        for (int64_t z = c0[2]; z <= c1[2]; ++z) grid[key(x, y, z)].push_back(uint32_t(k));
  }
  std::vector<uint32_t> stamp(m, UINT32_MAX);
  for (size_t k = 0; k < m; ++k) {
    int64_t c0[3], c1[3];
    cells_of(k, c0, c1);
    const uint32_t* fk = faces + 3 * size_t(fid[k]);
    for (int64_t x = c0[0]; x <= c1[0]; ++x)
      for (int64_t y = c0[1]; y <= c1[1]; ++y)
        for (int64_t z = c0[2]; z <= c1[2]; ++z) {
          auto it = grid.find(key(x, y, z));
          if (it == grid.end()) continue;
          for (uint32_t j : it->second) {
            if (j <= k || stamp[j] == uint32_t(k)) continue;
            stamp[j] = uint32_t(k);
            bool sep = false;
            for (int a = 0; a < 3 && !sep; ++a)
              sep = lo[3 * k + a] > hi[3 * size_t(j) + a] || lo[3 * size_t(j) + a] > hi[3 * k + a];
            if (sep) continue;
            if (ignore_adjacent) {
              const uint32_t* fj = faces + 3 * size_t(fid[j]);
              bool shared = false;
              for (int a = 0; a < 3 && !shared; ++a)
                for (int b = 0; b < 3 && !shared; ++b) shared = rep[fk[a]] == rep[fj[b]];
              if (shared) continue;
            }
            if (tri_tri(&tri[3 * k], &tri[3 * size_t(j)])) {
              out.push_back(fid[k]);
              out.push_back(fid[j]);
            }
          }
        }
  }
  // ascending (f0, f1); k < j and fid ascending already give f0 < f1
  std::vector<std::pair<uint32_t, uint32_t>> pr(out.size() / 2);
  for (size_t i = 0; i < pr.size(); ++i) pr[i] = {out[2 * i], out[2 * i + 1]};
  std::sort(pr.begin(), pr.end());
  for (size_t i = 0; i < pr.size(); ++i) {
    out[2 * i] = pr[i].first;
    out[2 * i + 1] = pr[i].second;
  }
  return out;
}

}  // namespace tcloth
