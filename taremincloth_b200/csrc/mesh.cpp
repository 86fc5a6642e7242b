// Host-side cloth topology and constraint builder (see mesh.hpp).
//
// Data structures: every "set of edges" / "map edge -> opposite vertices" of
// the reference is a sorted vector of 64-bit keys here; lookups are binary
// searches.  Insertion order is kept where the reference's output depends on
// it (constraint order, strand neighbour order).
#include "mesh.hpp"

#include <algorithm>
#include <cmath>
#include <numeric>
#include <stdexcept>

namespace tcloth {
namespace {

inline uint64_t key2(uint32_t a, uint32_t b) {
  return a < b ? (uint64_t(a) << 32 | b) : (uint64_t(b) << 32 | a);
}
inline uint32_t klo(uint64_t k) { return uint32_t(k >> 32); }
inline uint32_t khi(uint64_t k) { return uint32_t(k); }

inline float len3(const float* a, const float* b) {
  float dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
  return std::sqrt(dx * dx + dy * dy + dz * dz);
}

bool sorted_has(const std::vector<uint64_t>& v, uint64_t k) {
  return std::binary_search(v.begin(), v.end(), k);
}

// Growable open-addressing set of 64-bit keys (used where the reference
// inserts into a HashSet while iterating and tests the insert result).
class KeySet {
 public:
  explicit KeySet(size_t expect) { rehash(expect * 2 + 16); }
  bool insert(uint64_t k) {
    if ((n_ + 1) * 2 > slots_.size()) rehash(slots_.size() * 2);
    size_t m = slots_.size() - 1, h = mix(k) & m;
    while (slots_[h] != kEmpty) {
      if (slots_[h] == k) return false;
      h = (h + 1) & m;
    }
    slots_[h] = k;
    ++n_;
    return true;
  }

 private:
  static constexpr uint64_t kEmpty = ~uint64_t(0);
  static size_t mix(uint64_t k) {
    k ^= k >> 31; k *= 0x7fb5d329728ea185ULL; k ^= k >> 27; k *= 0x81dadef4bc2dd44dULL; k ^= k >> 33;
    return size_t(k);
  }
  void rehash(size_t want) {
    size_t c = 16;
    while (c < want) c <<= 1;
    std::vector<uint64_t> old;
    old.swap(slots_);
    slots_.assign(c, kEmpty);
    n_ = 0;
    for (uint64_t k : old)
      if (k != kEmpty) insert(k);
  }
  std::vector<uint64_t> slots_;
  size_t n_ = 0;
};

// Welsh-Powell: order by (degree desc, index asc), first-fit colour.
// conflict[i] lists the vertices whose constraint lists make up i's
// neighbourhood and degree; reg[i] lists where i registers itself.
// Returns number of colours.
uint32_t welsh_powell(uint32_t nv, const std::vector<std::vector<uint32_t>>& deg_verts,
                      const std::vector<std::vector<uint32_t>>& reg, std::vector<uint32_t>& color) {
  const size_t nc = reg.size();
  std::vector<uint32_t> off(nv + 1, 0);
  for (const auto& r : reg)
    for (uint32_t v : r) off[v + 1]++;
  for (uint32_t v = 0; v < nv; ++v) off[v + 1] += off[v];
  std::vector<uint32_t> fill(off.begin(), off.end() - 1), v2c(off[nv]);
  for (size_t i = 0; i < nc; ++i)
    for (uint32_t v : reg[i]) v2c[fill[v]++] = uint32_t(i);
  std::vector<std::pair<int64_t, uint32_t>> order(nc);
  for (size_t i = 0; i < nc; ++i) {
    int64_t d = 0;
    for (uint32_t v : deg_verts[i])
      if (v < nv) d += off[v + 1] - off[v];
    order[i] = {-d, uint32_t(i)};
  }
  std::sort(order.begin(), order.end());
  color.assign(nc, UINT32_MAX);
  std::vector<uint32_t> stamp(64, 0);
  uint32_t ncol = 0, tick = 0;
  for (const auto& oi : order) {
    const uint32_t i = oi.second;
    ++tick;
    for (uint32_t v : deg_verts[i]) {
      if (v >= nv) continue;
      for (uint32_t q = off[v]; q < off[v + 1]; ++q) {
        uint32_t a = v2c[q];
        if (a == i || color[a] == UINT32_MAX) continue;
        if (color[a] >= stamp.size()) stamp.resize(color[a] * 2 + 2, 0);
        stamp[color[a]] = tick;
      }
    }
    uint32_t c = 0;
    while (c < stamp.size() && stamp[c] == tick) ++c;
    color[i] = c;
    ncol = std::max(ncol, c + 1);
  }
  return ncol;
}

// stable bucket reorder: perm[sorted] = original index
void bucket(const std::vector<uint32_t>& color, uint32_t ncol, std::vector<uint32_t>& off,
            std::vector<uint32_t>& cnt, std::vector<uint32_t>& perm) {
  cnt.assign(ncol, 0);
  for (uint32_t c : color) cnt[c]++;
  off.assign(ncol, 0);
  uint32_t acc = 0;
  for (uint32_t c = 0; c < ncol; ++c) { off[c] = acc; acc += cnt[c]; }
  std::vector<uint32_t> f(off);
  perm.assign(color.size(), 0);
  for (size_t i = 0; i < color.size(); ++i) perm[f[color[i]]++] = uint32_t(i);
}

inline uint32_t expand10(uint32_t v) {
  v = (v * 0x00010001u) & 0xFF0000FFu;
  v = (v * 0x00000101u) & 0x0F00F00Fu;
  v = (v * 0x00000011u) & 0xC30C30C3u;
  v = (v * 0x00000005u) & 0x49249249u;
  return v;
}
inline uint32_t sat_u32(float f) {
  if (!(f > 0.f)) return 0;
  if (f >= 4294967295.f) return UINT32_MAX;
  return uint32_t(f);
}
inline float clamp01(float x) { return std::fmin(std::fmax(x, 0.f), 1.f); }

}  // namespace

float stiffness_to_compliance(float k) {
  if (k >= 5000.f) return 0.f;   // inextensible (mesh.rs:450-472)
  if (k > 0.f) return 1.f / k;
  return 1e10f;
}

uint32_t morton3(float px, float py, float pz, const float bmin[3], const float inv[3]) {
  uint32_t x = sat_u32(clamp01((px - bmin[0]) * inv[0]) * 1023.f);
  uint32_t y = sat_u32(clamp01((py - bmin[1]) * inv[1]) * 1023.f);
  uint32_t z = sat_u32(clamp01((pz - bmin[2]) * inv[2]) * 1023.f);
  return (expand10(x) << 2) | (expand10(y) << 1) | expand10(z);
}

// |(projection of p - e0 onto the edge e0->e1, distance from the edge line)|,
// the in-plane coordinates used to unfold two triangles about a seam
// (mesh.rs:795-809, :1436-1454).  ok = false for a degenerate edge.
struct EdgeFrame { float s, h; bool ok; };
EdgeFrame edge_frame(const float* e0, const float* e1, const float* p) {
  const float ev[3] = {e1[0] - e0[0], e1[1] - e0[1], e1[2] - e0[2]};
  const float len = std::sqrt(ev[0] * ev[0] + ev[1] * ev[1] + ev[2] * ev[2]);
  if (len <= 1e-6f) return {0.f, 0.f, false};
  const float u[3] = {ev[0] / len, ev[1] / len, ev[2] / len};
  const float d[3] = {p[0] - e0[0], p[1] - e0[1], p[2] - e0[2]};
  const float s = d[0] * u[0] + d[1] * u[1] + d[2] * u[2];
  const float q[3] = {d[0] - s * u[0], d[1] - s * u[1], d[2] - s * u[2]};
  return {s, std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]), true};
}
// distance of the opposite vertices with both triangles unfolded flat about
// the seam: sqrt((sa - sb)^2 + (ha + hb)^2)
inline float unfolded(const EdgeFrame& a, const EdgeFrame& b) {
  const float ds = a.s - b.s, dh = a.h + b.h;
  return std::sqrt(ds * ds + dh * dh);
}

// Rest length of a two-hop pair that is two-hop only through a sewing
// group (mesh.rs:1382-1488): the smallest of, over relay groups reached
// from both i and nbr, the direct distance (same relay vertex), the
// unfolded distance across a shared seam edge, or the two edge lengths
// summed (no shared seam edge); 0 when none is above 1e-5.
float seam_two_hop_rest(uint32_t i, uint32_t nbr, const float* P, const std::vector<uint32_t>& off,
                        const std::vector<uint32_t>& idx, const std::vector<uint32_t>& rep) {
  auto pv = [&](uint32_t v) { return P + 3 * size_t(v); };
  const uint32_t ri = rep[i], rn = rep[nbr];
  float best = 3.4028235e38f;
  for (uint32_t q1 = off[i]; q1 < off[i + 1]; ++q1) {
    const uint32_t m1 = idx[q1], rm1 = rep[m1];
    if (rm1 == ri || rm1 == rn) continue;
    for (uint32_t q2 = off[nbr]; q2 < off[nbr + 1]; ++q2) {
      const uint32_t m2 = idx[q2];
      if (rep[m2] != rm1) continue;
      if (m1 == m2) {
        best = std::fmin(best, len3(pv(i), pv(nbr)));
        continue;
      }
      bool seam = false;
      for (uint32_t k1q = off[m1]; k1q < off[m1 + 1]; ++k1q) {
        const uint32_t k1 = idx[k1q], rk1 = rep[k1];
        if (rk1 == rm1) continue;
        for (uint32_t k2q = off[m2]; k2q < off[m2 + 1]; ++k2q) {
          const uint32_t k2 = idx[k2q];
          if (rep[k2] != rk1) continue;
          const EdgeFrame fa = edge_frame(pv(m1), pv(k1), pv(i)), fb = edge_frame(pv(m2), pv(k2), pv(nbr));
          if (!fa.ok || !fb.ok) continue;
          const float fl = unfolded(fa, fb);
          if (fl < best) { best = fl; seam = true; }
        }
      }
      if (!seam) best = std::fmin(best, len3(pv(i), pv(m1)) + len3(pv(nbr), pv(m2)));
    }
  }
  return (best < 3.4028235e38f && std::isfinite(best) && best > 1e-5f) ? best : 0.f;
}

MeshData build_mesh(const MeshInput& in) {
  MeshData m;
  const uint32_t n = in.n;
  m.n = n;
  const float* P = in.pos;
  auto pv = [&](uint32_t i) { return P + 3 * size_t(i); };
  m.pos.assign(P, P + 3 * size_t(n));
  m.inv_mass.resize(n);
  m.layer.resize(n);
  m.thickness.resize(n);
  for (uint32_t i = 0; i < n; ++i) {
    m.inv_mass[i] = in.inv_masses ? in.inv_masses[i] : 1.f;
    m.layer[i] = in.layer_ids ? in.layer_ids[i] : in.layer_id;
    m.thickness[i] = in.thicknesses ? in.thicknesses[i] : in.thickness;
  }
  // valid faces
  std::vector<uint32_t> vf;
  vf.reserve(size_t(in.nf) * 3);
  for (uint32_t f = 0; f < in.nf; ++f) {
    const uint32_t* t = in.faces + 3 * size_t(f);
    if (t[0] < n && t[1] < n && t[2] < n) vf.insert(vf.end(), t, t + 3);
  }
  const size_t nfv = vf.size() / 3;

  // ---- stretch (mesh.rs:476-499)
  const float tc = stiffness_to_compliance(in.tension_k), cc = stiffness_to_compliance(in.compression_k),
              shc = stiffness_to_compliance(in.shear_k);
  std::vector<DistC> dl;
  dl.reserve(size_t(in.ne) * 3);
  std::vector<int64_t> raw_edge_to_dist(in.ne, -1);
  std::vector<uint64_t> orig;
  orig.reserve(in.ne);
  for (uint32_t e = 0; e < in.ne; ++e) {
    uint32_t a = in.edges[2 * size_t(e)], b = in.edges[2 * size_t(e) + 1];
    if (a < n && b < n && a != b) {
      raw_edge_to_dist[e] = int64_t(dl.size());
      dl.push_back({a, b, len3(pv(a), pv(b)), tc, cc, 0u});
      orig.push_back(key2(a, b));
    }
  }
  std::sort(orig.begin(), orig.end());
  orig.erase(std::unique(orig.begin(), orig.end()), orig.end());

  // edge -> opposite vertices, in face order (sorted by key, stable)
  struct Opp { uint64_t key; uint32_t opp; uint32_t ord; };
  std::vector<Opp> eo;
  eo.reserve(nfv * 3);
  for (size_t f = 0; f < nfv; ++f) {
    uint32_t f0 = vf[3 * f], f1 = vf[3 * f + 1], f2 = vf[3 * f + 2];
    uint32_t o = uint32_t(eo.size());
    eo.push_back({key2(f0, f1), f2, o});
    eo.push_back({key2(f1, f2), f0, o + 1});
    eo.push_back({key2(f2, f0), f1, o + 2});
  }
  std::sort(eo.begin(), eo.end(), [](const Opp& x, const Opp& y) {
    return x.key != y.key ? x.key < y.key : x.ord < y.ord;
  });

  // ---- shear on non-original triangle edges + their cross pair (mesh.rs:508-560)
  if (in.nf > 0) {
    KeySet exist(orig.size() + eo.size());
    for (uint64_t k : orig) exist.insert(k);
    for (size_t i = 0; i < eo.size();) {
      size_t j = i;
      while (j < eo.size() && eo[j].key == eo[i].key) ++j;
      if (!sorted_has(orig, eo[i].key) && j - i == 2) {
        uint32_t o0 = eo[i].opp, o1 = eo[i + 1].opp;
        uint64_t pairs[2] = {eo[i].key, (uint64_t(std::min(o0, o1)) << 32) | std::max(o0, o1)};
        for (uint64_t k : pairs) {
          uint32_t a = klo(k), b = khi(k);
          if (a != b && exist.insert(k)) dl.push_back({a, b, len3(pv(a), pv(b)), shc, shc, 1u});
        }
      }
      i = j;
    }
  }
  // colouring of distance constraints (coloring.rs:6-79)
  {
    std::vector<std::vector<uint32_t>> verts(dl.size());
    for (size_t i = 0; i < dl.size(); ++i) verts[i] = {dl[i].v0, dl[i].v1};
    std::vector<uint32_t> color, perm;
    uint32_t ncol = dl.empty() ? 0 : welsh_powell(n, verts, verts, color);
    bucket(color, ncol, m.dist_off, m.dist_cnt, perm);
    m.dist.resize(dl.size());
    std::vector<int64_t> remap(dl.size());
    for (size_t s = 0; s < perm.size(); ++s) { m.dist[s] = dl[perm[s]]; remap[perm[s]] = int64_t(s); }
    m.orig_edge_to_dist.resize(in.ne);
    for (uint32_t e = 0; e < in.ne; ++e)
      m.orig_edge_to_dist[e] = raw_edge_to_dist[e] < 0 ? -1 : remap[size_t(raw_edge_to_dist[e])];
  }

  // ---- bending across original edges with two triangles (mesh.rs:632-704)
  const float bcomp = in.bending_k > 0.f ? 1.f / in.bending_k : 1e10f;
  std::vector<BendC> bl;
  if (in.nf > 0) {
    for (size_t i = 0; i < eo.size();) {
      size_t j = i;
      while (j < eo.size() && eo[j].key == eo[i].key) ++j;
      if (sorted_has(orig, eo[i].key) && j - i == 2 && eo[i].opp != eo[i + 1].opp) {
        uint32_t v2 = eo[i].opp, v3 = eo[i + 1].opp;
        bl.push_back({klo(eo[i].key), khi(eo[i].key), v2, v3, len3(pv(v2), pv(v3)), bcomp, 0.f, 0.f});
      }
      i = j;
    }
  }
  // ---- sewing groups (mesh.rs:706-737, :990-1024): union-find over the
  //      springs, each group represented by its smallest vertex index
  std::vector<uint32_t>& rep = m.sew_rep;
  rep.resize(n);
  std::vector<uint8_t> has_sew(n, 0);
  for (uint32_t i = 0; i < n; ++i) rep[i] = i;
  auto find = [&](uint32_t i) {
    uint32_t r = i;
    while (r != rep[r]) r = rep[r];
    while (i != r) { const uint32_t nx = rep[i]; rep[i] = r; i = nx; }
    return r;
  };
  for (uint32_t k = 0; k < in.nsew; ++k) {
    const uint32_t u = in.sew[2 * size_t(k)], v = in.sew[2 * size_t(k) + 1];
    if (u < n && v < n && u != v) {
      has_sew[u] = has_sew[v] = 1;
      const uint32_t ru = find(u), rv = find(v);
      if (ru != rv) rep[std::max(ru, rv)] = std::min(ru, rv);
    }
  }
  for (uint32_t i = 0; i < n; ++i) rep[i] = find(i);
  // ---- seam-gated bending across sewn boundary edges (mesh.rs:706-838):
  //      two boundary edges (one triangle each) whose endpoints fall in the
  //      same two sewing groups get a bending constraint between their
  //      opposite vertices, rest = the distance with both triangles unfolded
  //      flat, gated on the seam closing to max(rest / 2, 0.01).  Within a
  //      group pair the two edges are taken in face order (the reference
  //      takes them in hash-map order; the constraint acts the same either
  //      way round).
  if (in.nsew > 0 && in.nf > 0) {
    struct Seam { uint64_t key; uint32_t a, b, opp, ord; };
    std::vector<Seam> se;
    for (size_t i = 0; i < eo.size();) {
      size_t j = i;
      while (j < eo.size() && eo[j].key == eo[i].key) ++j;
      const uint32_t ea = klo(eo[i].key), eb = khi(eo[i].key);
      if (j - i == 1 && has_sew[ea] && has_sew[eb] && rep[ea] != rep[eb]) {
        const bool fwd = rep[ea] < rep[eb];
        se.push_back({key2(rep[ea], rep[eb]), fwd ? ea : eb, fwd ? eb : ea, eo[i].opp, uint32_t(se.size())});
      }
      i = j;
    }
    std::sort(se.begin(), se.end(), [](const Seam& x, const Seam& y) {
      return x.key != y.key ? x.key < y.key : x.ord < y.ord;
    });
    for (size_t i = 0; i < se.size();) {
      size_t j = i;
      while (j < se.size() && se[j].key == se[i].key) ++j;
      if (j - i == 2) {
        const Seam &A = se[i], &B = se[i + 1];
        const uint32_t v2 = A.opp, v3 = B.opp;
        if (!(A.a == B.a || A.b == B.b || v2 == v3 || rep[v2] == rep[v3])) {
          const EdgeFrame fa = edge_frame(pv(A.a), pv(A.b), pv(v2)), fb = edge_frame(pv(B.a), pv(B.b), pv(v3));
          if (fa.ok && fb.ok) {
            const float flat = unfolded(fa, fb);
            if (flat > 1e-5f) bl.push_back({A.a, B.a, v2, v3, flat, bcomp, 1.f, std::fmax(flat * 0.5f, 0.01f)});
          }
        }
      }
      i = j;
    }
  }
  // ---- 1D strand bending (mesh.rs:840-905)
  {
    std::vector<uint64_t> fe;
    fe.reserve(size_t(in.nf) * 3);
    for (uint32_t f = 0; f < in.nf; ++f) {
      const uint32_t* t = in.faces + 3 * size_t(f);
      fe.push_back(key2(t[0], t[1]));
      fe.push_back(key2(t[1], t[2]));
      fe.push_back(key2(t[2], t[0]));
    }
    std::sort(fe.begin(), fe.end());
    std::vector<std::vector<uint32_t>> sadj;
    bool any = false;
    for (uint32_t e = 0; e < in.ne; ++e) {
      uint32_t a = in.edges[2 * size_t(e)], b = in.edges[2 * size_t(e) + 1];
      if (a < n && b < n && a != b && !sorted_has(fe, key2(a, b))) {
        if (!any) { sadj.resize(n); any = true; }
        sadj[a].push_back(b);
        sadj[b].push_back(a);
      }
    }
    if (any) {
      KeySet seen(bl.size() + 16);
      for (const auto& c : bl) seen.insert(key2(c.v2, c.v3));
      const float scomp = std::fmax(bcomp * 10.f, 0.5f);
      for (uint32_t u = 0; u < n; ++u) {
        const auto& nb = sadj[u];
        if (nb.size() < 2) continue;
        for (size_t i = 0; i < nb.size(); ++i)
          for (size_t j = i + 1; j < nb.size(); ++j) {
            uint32_t a = nb[i], b = nb[j];
            if (a != b && seen.insert(key2(a, b))) bl.push_back({u, u, a, b, len3(pv(a), pv(b)), scomp, 2.f, 0.f});
          }
      }
    }
  }
  // colouring of bending constraints (coloring.rs:82-173)
  {
    std::vector<std::vector<uint32_t>> dv(bl.size()), rg(bl.size());
    for (size_t i = 0; i < bl.size(); ++i) {
      const BendC& c = bl[i];
      rg[i] = {c.v2, c.v3};
      if (c.pad0 > 0.5f) {
        if (c.v0 < n && c.v0 != c.v2 && c.v0 != c.v3) rg[i].push_back(c.v0);
        if (c.v1 < n && c.v1 != c.v2 && c.v1 != c.v3 && c.v1 != c.v0) rg[i].push_back(c.v1);
        dv[i] = {c.v2, c.v3, c.v0, c.v1};
      } else {
        dv[i] = {c.v2, c.v3};
      }
    }
    std::vector<uint32_t> color, perm;
    uint32_t ncol = bl.empty() ? 0 : welsh_powell(n, dv, rg, color);
    bucket(color, ncol, m.bend_off, m.bend_cnt, perm);
    m.bend.resize(bl.size());
    for (size_t s = 0; s < perm.size(); ++s) m.bend[s] = bl[perm[s]];
  }

  // ---- sewing constraints and their colouring (mesh.rs:904-936,
  //      coloring.rs:236-300: Welsh-Powell as for distance constraints)
  {
    const float sk = in.sew_stiffness;
    const float comp = sk >= 5000.f ? 0.f : (sk > 0.f ? 1.f / sk : 1e10f);
    std::vector<SewC> sl;
    for (uint32_t k = 0; k < in.nsew; ++k) {
      const uint32_t a = in.sew[2 * size_t(k)], b = in.sew[2 * size_t(k) + 1];
      if (a < n && b < n && a != b)
        sl.push_back({a, b, len3(pv(a), pv(b)), 0.f, std::fmax(in.sew_shrink_speed, 0.f), comp, in.sew_lock ? 1.f : 0.f});
    }
    std::vector<std::vector<uint32_t>> verts(sl.size());
    for (size_t i = 0; i < sl.size(); ++i) verts[i] = {sl[i].v0, sl[i].v1};
    std::vector<uint32_t> color, perm;
    const uint32_t ncol = sl.empty() ? 0 : welsh_powell(n, verts, verts, color);
    bucket(color, ncol, m.sew_off, m.sew_cnt, perm);
    m.sew.resize(sl.size());
    for (size_t s2 = 0; s2 < perm.size(); ++s2) m.sew[s2] = sl[perm[s2]];
  }

  // ---- adjacency and local edge length (mesh.rs:949-1090)
  std::vector<uint32_t> deg(n + 1, 0);
  std::vector<float> lsum(n, 0.f);
  std::vector<uint32_t> lcnt(n, 0);
  float total = 0.f, maxe = 0.f;
  uint32_t valid = 0;
  for (uint32_t e = 0; e < in.ne; ++e) {
    uint32_t a = in.edges[2 * size_t(e)], b = in.edges[2 * size_t(e) + 1];
    if (a < n && b < n && a != b) {
      float L = len3(pv(a), pv(b));
      total += L;
      if (L > maxe) maxe = L;
      ++valid;
      deg[a + 1]++; deg[b + 1]++;
      lsum[a] += L; lcnt[a]++; lsum[b] += L; lcnt[b]++;
    }
  }
  m.mean_edge = valid ? total / float(valid) : 0.f;
  m.max_edge = maxe;
  m.local_len.resize(n);
  for (uint32_t i = 0; i < n; ++i)
    m.local_len[i] = lcnt[i] ? lsum[i] / float(lcnt[i]) : std::fmax(in.thickness, 0.01f);
  {
    std::vector<uint32_t> off(deg);
    for (uint32_t i = 0; i < n; ++i) off[i + 1] += off[i];
    std::vector<uint32_t> raw(off[n]), f(off.begin(), off.end() - 1);
    for (uint32_t e = 0; e < in.ne; ++e) {
      uint32_t a = in.edges[2 * size_t(e)], b = in.edges[2 * size_t(e) + 1];
      if (a < n && b < n && a != b) { raw[f[a]++] = b; raw[f[b]++] = a; }
    }
    m.adj_off.assign(n + 1, 0);
    m.adj_idx.clear();
    m.adj_idx.reserve(raw.size());
    for (uint32_t i = 0; i < n; ++i) {
      auto b = raw.begin() + off[i], e = raw.begin() + off[i + 1];
      std::sort(b, e);
      auto u = std::unique(b, e);
      m.adj_off[i] = uint32_t(m.adj_idx.size());
      m.adj_idx.insert(m.adj_idx.end(), b, u);
    }
    m.adj_off[n] = uint32_t(m.adj_idx.size());
  }
  // the adjacency of the input edges alone (sorted): two-hop rest lengths
  // and the sewing contraction read it
  const std::vector<uint32_t> orig_off = m.adj_off, orig_idx = m.adj_idx;
  bool sewn = false;
  for (uint32_t i = 0; i < n && !sewn; ++i) sewn = rep[i] != i;
  // ---- sewing extends the adjacency (mesh.rs:990-1060): the members of a
  //      group become neighbours of each other and of every neighbour of
  //      any member, symmetrically
  if (sewn) {
    std::vector<std::vector<uint32_t>> lists(n), groups(n);
    for (uint32_t i = 0; i < n; ++i) {
      lists[i].assign(orig_idx.begin() + orig_off[i], orig_idx.begin() + orig_off[i + 1]);
      groups[rep[i]].push_back(i);
    }
    for (const auto& g : groups)
      if (g.size() > 1)
        for (uint32_t u : g)
          for (uint32_t v : g)
            if (u != v) lists[u].push_back(v);
    const std::vector<std::vector<uint32_t>> base = lists;
    std::vector<uint32_t> shared;
    for (const auto& g : groups) {
      if (g.size() < 2) continue;
      shared.clear();
      for (uint32_t u : g)
        for (uint32_t w : base[u])
          if (rep[w] != rep[g[0]]) shared.push_back(w);
      std::sort(shared.begin(), shared.end());
      shared.erase(std::unique(shared.begin(), shared.end()), shared.end());
      for (uint32_t u : g)
        for (uint32_t w : shared) { lists[u].push_back(w); lists[w].push_back(u); }
    }
    m.adj_idx.clear();
    for (uint32_t i = 0; i < n; ++i) {
      auto& l = lists[i];
      std::sort(l.begin(), l.end());
      l.erase(std::unique(l.begin(), l.end()), l.end());
      m.adj_off[i] = uint32_t(m.adj_idx.size());
      m.adj_idx.insert(m.adj_idx.end(), l.begin(), l.end());
    }
    m.adj_off[n] = uint32_t(m.adj_idx.size());
  }
  // ---- two-hop CSR with rest lengths for true two-hop face pairs (mesh.rs:1092-1199).
  //      With sewing, a pair is true two-hop when neither the same group
  //      nor adjacent in the input mesh or in the group-contracted mesh; its
  //      rest length is the plain distance when it is within two hops in
  //      the input mesh, else the seam-unfolded one (seam_two_hop_rest).
  {
    // one-hop sets of the contracted mesh, indexed by group
    std::vector<std::vector<uint32_t>> chop;
    if (sewn) {
      chop.resize(n);
      for (uint32_t e = 0; e < in.ne; ++e) {
        const uint32_t a = in.edges[2 * size_t(e)], b = in.edges[2 * size_t(e) + 1];
        if (a < n && b < n && a != b && rep[a] != rep[b]) {
          chop[rep[a]].push_back(rep[b]);
          chop[rep[b]].push_back(rep[a]);
        }
      }
      for (auto& l : chop) {
        std::sort(l.begin(), l.end());
        l.erase(std::unique(l.begin(), l.end()), l.end());
      }
    }
    std::vector<uint32_t> orig2;
    std::vector<uint8_t> isface(n, 0);
    for (uint32_t f = 0; f < in.nf; ++f)
      for (int k = 0; k < 3; ++k) {
        uint32_t v = in.faces[3 * size_t(f) + k];
        if (v < n) isface[v] = 1;
      }
    m.th_off.assign(n + 1, 0);
    std::vector<uint32_t> tmp;
    for (uint32_t i = 0; i < n; ++i) {
      tmp.clear();
      tmp.push_back(i);
      for (uint32_t k = m.adj_off[i]; k < m.adj_off[i + 1]; ++k) {
        uint32_t u = m.adj_idx[k];
        tmp.push_back(u);
        tmp.insert(tmp.end(), m.adj_idx.begin() + m.adj_off[u], m.adj_idx.begin() + m.adj_off[u + 1]);
      }
      std::sort(tmp.begin(), tmp.end());
      tmp.erase(std::unique(tmp.begin(), tmp.end()), tmp.end());
      m.th_off[i] = uint32_t(m.th_idx.size());
      const uint32_t* ab = orig_idx.data() + orig_off[i];
      const uint32_t* ae = orig_idx.data() + orig_off[i + 1];
      if (sewn) {  // the input mesh's 0/1/2-hop set of i
        orig2.assign(1, i);
        for (const uint32_t* q = ab; q < ae; ++q) {
          orig2.push_back(*q);
          orig2.insert(orig2.end(), orig_idx.begin() + orig_off[*q], orig_idx.begin() + orig_off[*q + 1]);
        }
        std::sort(orig2.begin(), orig2.end());
        orig2.erase(std::unique(orig2.begin(), orig2.end()), orig2.end());
      }
      for (uint32_t nbr : tmp) {
        bool two = nbr != i && isface[i] && isface[nbr] && !std::binary_search(ab, ae, nbr);
        if (sewn)
          two = two && rep[i] != rep[nbr] &&
                !std::binary_search(chop[rep[i]].begin(), chop[rep[i]].end(), rep[nbr]);
        float rest = 0.f;
        if (two)
          rest = (!sewn || std::binary_search(orig2.begin(), orig2.end(), nbr))
                     ? len3(pv(i), pv(nbr))
                     : seam_two_hop_rest(i, nbr, P, orig_off, orig_idx, rep);
        m.th_idx.push_back(nbr);
        m.th_rest.push_back(rest);
      }
    }
    m.th_off[n] = uint32_t(m.th_idx.size());
  }
  // ---- star pairs (mesh.rs:1201-1221)
  {
    std::vector<uint32_t> c(n + 1, 0);
    for (size_t f = 0; f < nfv; ++f)
      for (int k = 0; k < 3; ++k) c[vf[3 * f + k] + 1]++;
    for (uint32_t i = 0; i < n; ++i) c[i + 1] += c[i];
    m.star_off = c;
    m.star_idx.assign(size_t(c[n]) * 2, 0);
    std::vector<uint32_t> f(c.begin(), c.end() - 1);
    for (size_t t = 0; t < nfv; ++t) {
      uint32_t f0 = vf[3 * t], f1 = vf[3 * t + 1], f2 = vf[3 * t + 2];
      uint32_t s;
      s = f[f0]++; m.star_idx[2 * s] = f1; m.star_idx[2 * s + 1] = f2;
      s = f[f1]++; m.star_idx[2 * s] = f2; m.star_idx[2 * s + 1] = f0;
      s = f[f2]++; m.star_idx[2 * s] = f0; m.star_idx[2 * s + 1] = f1;
    }
  }
  // ---- islands (mesh.rs:1233-1256)
  {
    m.island.assign(n, UINT32_MAX);
    std::vector<uint32_t> q(n);
    uint32_t cur = 0;
    for (uint32_t i = 0; i < n; ++i) {
      if (m.island[i] != UINT32_MAX) continue;
      size_t h = 0, t = 0;
      m.island[i] = cur;
      q[t++] = i;
      while (h < t) {
        uint32_t u = q[h++];
        for (uint32_t k = m.adj_off[u]; k < m.adj_off[u + 1]; ++k) {
          uint32_t v = m.adj_idx[k];
          if (m.island[v] == UINT32_MAX) { m.island[v] = cur; q[t++] = v; }
        }
      }
      ++cur;
    }
  }
  // ---- unique edges sorted by midpoint Morton code (mesh.rs:1258-1289)
  {
    std::vector<uint64_t> ge;
    {
      KeySet es(in.ne + 1);
      for (uint32_t e = 0; e < in.ne; ++e) {
        uint32_t a = in.edges[2 * size_t(e)], b = in.edges[2 * size_t(e) + 1];
        if (a < n && b < n && a != b && es.insert(key2(a, b))) ge.push_back(key2(a, b));
      }
    }
    if (!ge.empty() && n > 0) {
      float bmin[3] = {3.4028235e38f, 3.4028235e38f, 3.4028235e38f}, bmax[3] = {-3.4028235e38f, -3.4028235e38f, -3.4028235e38f};
      for (uint32_t i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a) {
          bmin[a] = std::fmin(bmin[a], P[3 * size_t(i) + a]);
          bmax[a] = std::fmax(bmax[a], P[3 * size_t(i) + a]);
        }
      float inv[3];
      for (int a = 0; a < 3; ++a) inv[a] = 1.f / std::fmax(bmax[a] - bmin[a], 1e-5f);
      std::vector<std::pair<uint32_t, uint32_t>> ki(ge.size());
      for (size_t e = 0; e < ge.size(); ++e) {
        const float *p0 = pv(klo(ge[e])), *p1 = pv(khi(ge[e]));
        ki[e] = {morton3((p0[0] + p1[0]) * 0.5f, (p0[1] + p1[1]) * 0.5f, (p0[2] + p1[2]) * 0.5f, bmin, inv),
                 uint32_t(e)};
      }
      std::sort(ki.begin(), ki.end());  // (code, original position): stable
      std::vector<uint64_t> g2(ge.size());
      for (size_t e = 0; e < ge.size(); ++e) g2[e] = ge[ki[e].second];
      ge.swap(g2);
    }
    m.edges.resize(ge.size() * 2);
    for (size_t e = 0; e < ge.size(); ++e) { m.edges[2 * e] = klo(ge[e]); m.edges[2 * e + 1] = khi(ge[e]); }
    // open-boundary bits (mesh.rs:1291-1344): an edge with 0 or 1 incident triangles
    m.edge_bits.assign((ge.size() + 31) / 32, 0);
    if (in.nf > 0) {
      std::vector<uint64_t> tk;
      tk.reserve(size_t(in.nf) * 3);
      for (uint32_t f = 0; f < in.nf; ++f) {
        const uint32_t* t = in.faces + 3 * size_t(f);
        for (int k = 0; k < 3; ++k) {
          uint32_t a = t[k], b = t[(k + 1) % 3];
          if (a < n && b < n && a != b) tk.push_back(key2(a, b));
        }
      }
      std::sort(tk.begin(), tk.end());
      // face edges counted between sewing groups (the contracted mesh)
      std::vector<uint64_t> ck;
      ck.reserve(tk.size());
      for (uint64_t k : tk)
        if (rep[klo(k)] != rep[khi(k)]) ck.push_back(key2(rep[klo(k)], rep[khi(k)]));
      std::sort(ck.begin(), ck.end());
      for (size_t e = 0; e < ge.size(); ++e) {
        const uint32_t ra = rep[klo(ge[e])], rb = rep[khi(ge[e])];
        if (ra == rb) continue;  // an edge inside a sewing group
        auto r = std::equal_range(tk.begin(), tk.end(), ge[e]);
        bool open = r.second == r.first;  // a 1D strand edge
        if (r.second - r.first == 1) {
          auto c = std::equal_range(ck.begin(), ck.end(), key2(ra, rb));
          open = c.second - c.first == 1;  // not matched by a sewn edge of another panel
        }
        if (open) m.edge_bits[e >> 5] |= 1u << (e & 31);
      }
    } else {
      for (size_t e = 0; e < ge.size(); ++e)
        if (rep[klo(ge[e])] != rep[khi(ge[e])]) m.edge_bits[e >> 5] |= 1u << (e & 31);
    }
  }
  // ---- automatic layer per island by mean Z (pipelines.rs:131-167)
  if (n > 0) {
    bool same = std::all_of(m.layer.begin(), m.layer.end(), [&](uint32_t l) { return l == m.layer[0]; });
    uint32_t maxi = n ? *std::max_element(m.island.begin(), m.island.end()) : 0;
    if (same && maxi > 0) {
      std::vector<float> zs(maxi + 1, 0.f);
      std::vector<uint32_t> zc(maxi + 1, 0);
      for (uint32_t i = 0; i < n; ++i) { zs[m.island[i]] += P[3 * size_t(i) + 2]; zc[m.island[i]]++; }
      std::vector<std::pair<float, uint32_t>> im(maxi + 1);
      for (uint32_t k = 0; k <= maxi; ++k) im[k] = {zs[k] / float(std::max(zc[k], 1u)), k};
      std::stable_sort(im.begin(), im.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
      std::vector<uint32_t> rank(maxi + 1);
      for (uint32_t r = 0; r <= maxi; ++r) rank[im[r].second] = r;
      for (uint32_t i = 0; i < n; ++i) m.layer[i] = rank[m.island[i]];
    }
  }
  m.multi_layer = false;
  for (uint32_t i = 0; i < n; ++i)
    if (m.layer[i] != m.layer[0]) { m.multi_layer = true; break; }

  // ---- virtual-particle count, which only sizes the hash table
  //      (virtual_mesh.rs:75-190; pipelines.rs:170-228, :910-912)
  {
    uint64_t M = 0;
    const float dthick = n ? m.thickness[0] : 0.003f;
    const float spacing = dthick * 1.5f;
    if (!(spacing <= 1e-6f) && n > 0 && nfv > 0) {
      std::vector<uint64_t> fk;
      fk.reserve(nfv * 3);
      for (size_t f = 0; f < nfv; ++f) {
        fk.push_back(key2(vf[3 * f], vf[3 * f + 1]));
        fk.push_back(key2(vf[3 * f + 1], vf[3 * f + 2]));
        fk.push_back(key2(vf[3 * f + 2], vf[3 * f]));
      }
      std::sort(fk.begin(), fk.end());
      for (const auto& c : m.dist) {
        if (!sorted_has(fk, key2(c.v0, c.v1))) continue;
        uint32_t ke = sat_u32(std::ceil(len3(pv(c.v1), pv(c.v0)) / spacing));
        ke = std::min(ke, 16u);
        if (ke > 1) M += ke - 1;
      }
      for (size_t f = 0; f < nfv; ++f) {
        const float *a = pv(vf[3 * f]), *b = pv(vf[3 * f + 1]), *c = pv(vf[3 * f + 2]);
        float lmax = std::fmax(std::fmax(len3(b, a), len3(c, b)), len3(a, c));
        uint32_t k = std::min(sat_u32(std::ceil(lmax / spacing)), 16u);
        if (k >= 3) M += uint64_t(k - 1) * (k - 2) / 2;
      }
    }
    m.num_virtual = uint32_t(std::min<uint64_t>(M, 150000));
  }
  // ---- hash sizing (pipelines.rs:898-912)
  {
    const float th = n ? m.thickness[0] : 0.005f;
    const float eb = std::fmin(std::fmax(m.max_edge * 0.85f, m.mean_edge * 1.0f), 0.025f);
    m.cell = std::fmax(std::fmax(th * 4.f, eb), 0.01f);
    uint64_t cap = uint64_t(n + m.num_virtual) * 4u, t = 1;
    while (t < cap) t <<= 1;
    m.table = uint32_t(std::min<uint64_t>(std::max<uint64_t>(t, 1024), 65536));
  }
  return m;
}

// compute_combined_inv_masses (mesh.rs:237-312): a third of each valid
// triangle's area x areal density to each corner, half of each strand edge's
// length x linear density to each end, in input order; then
// w = (1 - pin) / max(mass, 1e-9), with pin clamped to [0, 1] (missing = 0)
// and 0 for pin >= 1.
std::vector<float> combined_inv_masses(const float* pos, uint32_t n, const uint32_t* faces, uint32_t nf,
                                       const uint32_t* strands, uint32_t ns, const float* pins, uint32_t npin,
                                       float areal_density, float linear_density) {
  std::vector<float> m(n, 0.f);
  if (areal_density > 0.f && faces) {
    for (uint32_t f = 0; f < nf; ++f) {
      const uint32_t a = faces[3 * f], b = faces[3 * f + 1], c = faces[3 * f + 2];
      if (a >= n || b >= n || c >= n || a == b || b == c || c == a) continue;
      const float* pa = pos + 3 * size_t(a);
      const float* pb = pos + 3 * size_t(b);
      const float* pc = pos + 3 * size_t(c);
      const float ab[3] = {pb[0] - pa[0], pb[1] - pa[1], pb[2] - pa[2]};
      const float ac[3] = {pc[0] - pa[0], pc[1] - pa[1], pc[2] - pa[2]};
      const float cr[3] = {ab[1] * ac[2] - ab[2] * ac[1], ab[2] * ac[0] - ab[0] * ac[2], ab[0] * ac[1] - ab[1] * ac[0]};
      const float area = 0.5f * std::sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
      const float share = area * areal_density / 3.0f;
      m[a] += share;
      m[b] += share;
      m[c] += share;
    }
  }
  if (linear_density > 0.f && strands) {
    for (uint32_t e = 0; e < ns; ++e) {
      const uint32_t a = strands[2 * e], b = strands[2 * e + 1];
      if (a >= n || b >= n || a == b) continue;
      const float* pa = pos + 3 * size_t(a);
      const float* pb = pos + 3 * size_t(b);
      const float dx = pa[0] - pb[0], dy = pa[1] - pb[1], dz = pa[2] - pb[2];
      const float len = std::sqrt(dx * dx + dy * dy + dz * dz);
      const float share = len * linear_density / 2.0f;
      m[a] += share;
      m[b] += share;
    }
  }
  std::vector<float> w(n);
  for (uint32_t i = 0; i < n; ++i) {
    float pin = (pins && i < npin) ? pins[i] : 0.f;
    if (!std::isnan(pin)) pin = std::min(std::max(pin, 0.f), 1.f);
    w[i] = pin >= 1.f ? 0.f : (1.f - pin) / std::fmax(m[i], 1e-9f);
  }
  return w;
}

// color_edge_pairs (coloring.rs:180-233): Welsh-Powell over vertex-sharing
// pairs, order (-degree, index), first free colour; a pair's out-of-range
// ends register nothing.
std::vector<uint32_t> color_edge_pairs(uint32_t nv, const uint32_t* pairs, uint32_t np) {
  std::vector<uint32_t> color(np, 0u);
  if (np == 0 || nv == 0) return color;
  std::vector<uint32_t> off(size_t(nv) + 1, 0u);
  for (uint32_t i = 0; i < np; ++i)
    for (int k = 0; k < 2; ++k)
      if (pairs[2 * i + k] < nv) ++off[pairs[2 * i + k] + 1];
  for (uint32_t v = 0; v < nv; ++v) off[v + 1] += off[v];
  std::vector<uint32_t> fill(off.begin(), off.end() - 1), v2c(off[nv]);
  for (uint32_t i = 0; i < np; ++i)
    for (int k = 0; k < 2; ++k)
      if (pairs[2 * i + k] < nv) v2c[fill[pairs[2 * i + k]]++] = i;
  auto deg = [&](uint32_t v) { return v < nv ? off[v + 1] - off[v] : 0u; };
  std::vector<uint32_t> order(np);
  for (uint32_t i = 0; i < np; ++i) order[i] = i;
  std::vector<uint32_t> key(np);
  for (uint32_t i = 0; i < np; ++i) key[i] = deg(pairs[2 * i]) + deg(pairs[2 * i + 1]);
  std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return key[a] > key[b]; });
  std::fill(color.begin(), color.end(), UINT32_MAX);
  std::vector<uint32_t> used_stamp;
  uint32_t stamp = 0;
  for (uint32_t i : order) {
    ++stamp;
    for (int k = 0; k < 2; ++k) {
      const uint32_t v = pairs[2 * i + k];
      if (v >= nv) continue;
      for (uint32_t q = off[v]; q < off[v + 1]; ++q) {
        const uint32_t adj = v2c[q];
        if (adj != i && color[adj] != UINT32_MAX) {
          if (color[adj] >= used_stamp.size()) used_stamp.resize(size_t(color[adj]) + 1, 0u);
          used_stamp[color[adj]] = stamp;
        }
      }
    }
    uint32_t c = 0;
    while (c < used_stamp.size() && used_stamp[c] == stamp) ++c;
    color[i] = c;
  }
  return color;
}

}  // namespace tcloth
