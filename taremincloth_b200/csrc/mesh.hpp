// Host-side cloth topology and constraint builder.
//
// Builds, once per simulator, everything the device substep reads: stretch
// and shear distance constraints, opposite-vertex (and 1D strand) bending
// constraints, their Welsh-Powell colouring, the adjacency / two-hop / star
// CSRs used by self-collision, the Morton-sorted unique edge list with its
// open-boundary bits, islands and automatic layers, and the spatial-hash
// sizing; with sewing springs also the sewing constraints, the seam-gated
// bending across sewn boundary edges, and the sewing-contracted adjacency,
// two-hop and boundary data.  Semantics follow crates/cloth_core/src/mesh.rs:407-1377,
// crates/cloth_core/src/coloring.rs:6-173 and
// crates/cloth_core/src/simulation/pipelines.rs:131-167, :898-912.
#pragma once
#include <cstdint>
#include <vector>

namespace tcloth {

struct DistC {       // 24 bytes on the host, split into two device arrays
  uint32_t v0, v1;
  float rest, tc, cc;
  uint32_t type;     // 0 stretch, 1 shear
};

struct BendC {
  uint32_t v0, v1, v2, v3;
  float rest, comp, pad0, pad1;  // pad0: 0 plain, 1 seam-gated, 2 strand
};

// Sewing spring (mesh.rs:904-933): pulled from its initial length towards
// target_rest (0) at shrink_speed m/s.  compliance and lock are stored as
// the reference stores them; the solve reads the simulator-level values.
struct SewC {
  uint32_t v0, v1;
  float cur_rest, target_rest, shrink_speed, compliance, lock;
};

struct MeshInput {
  const float* pos = nullptr;  // n*3
  uint32_t n = 0;
  const uint32_t* edges = nullptr;  // ne*2
  uint32_t ne = 0;
  const uint32_t* faces = nullptr;  // nf*3
  uint32_t nf = 0;
  const float* inv_masses = nullptr;
  const uint32_t* layer_ids = nullptr;
  const float* thicknesses = nullptr;
  uint32_t layer_id = 0;
  float thickness = 0.005f;
  float tension_k = 1000.f, compression_k = 1000.f, shear_k = 500.f, bending_k = 10.f;
  const uint32_t* sew = nullptr;  // nsew*2 sewing springs (pairs of vertices)
  uint32_t nsew = 0;
  float sew_shrink_speed = 1.f;
  float sew_stiffness = 10000.f;  // per-constraint compliance only
  bool sew_lock = true;           // per-constraint lock flag only
};

struct MeshData {
  uint32_t n = 0;
  std::vector<float> pos, inv_mass, thickness;
  std::vector<uint32_t> layer;
  std::vector<DistC> dist;             // colour-sorted
  std::vector<uint32_t> dist_off, dist_cnt;
  std::vector<int64_t> orig_edge_to_dist;  // input edge -> sorted constraint (-1 if none)
  std::vector<BendC> bend;             // colour-sorted
  std::vector<uint32_t> bend_off, bend_cnt;
  std::vector<SewC> sew;               // colour-sorted
  std::vector<uint32_t> sew_off, sew_cnt;
  std::vector<uint32_t> sew_rep;       // sewing group of each vertex (its smallest index)
  std::vector<uint32_t> adj_off, adj_idx;
  std::vector<uint32_t> th_off, th_idx;
  std::vector<float> th_rest, local_len;
  std::vector<uint32_t> star_off, star_idx;  // star_idx: pairs
  std::vector<uint32_t> edges;               // unique, Morton sorted, pairs (min,max)
  std::vector<uint32_t> edge_bits;
  std::vector<uint32_t> island;
  float mean_edge = 0.f, max_edge = 0.f;
  uint32_t num_virtual = 0;
  float cell = 0.01f;
  uint32_t table = 1024;
  bool multi_layer = false;
};

float stiffness_to_compliance(float k);
MeshData build_mesh(const MeshInput& in);
uint32_t morton3(float px, float py, float pz, const float bmin[3], const float inv[3]);
std::vector<float> combined_inv_masses(const float* pos, uint32_t n, const uint32_t* faces, uint32_t nf,
                                       const uint32_t* strands, uint32_t ns, const float* pins, uint32_t npin,
                                       float areal_density, float linear_density);
std::vector<uint32_t> color_edge_pairs(uint32_t nv, const uint32_t* pairs, uint32_t np);

// Face pairs (f0 < f1, ascending, flattened) whose triangles intersect,
// skipping pairs that share a vertex (or a sewn vertex cluster) when
// ignore_adjacent (geometry.rs:506-633); cell_size <= 0 picks one.
std::vector<uint32_t> find_triangle_intersections(const float* pos, uint32_t n, const uint32_t* faces, uint32_t nf,
                                                  bool ignore_adjacent, float cell_size, const uint32_t* sew,
                                                  uint32_t nsew);

}  // namespace tcloth
