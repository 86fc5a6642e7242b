// Simulator state, frame encoding and the C ABI (include/tcloth.h).
//
// One tc_sim owns all device buffers of one cloth.  A frame (substeps x
// iterations x colours of launches) is recorded once into a CUDA graph on the
// simulator's own stream and replayed while no parameter changes; any setter
// marks the graph stale.  Pass order follows encode_simulation_steps
// (crates/cloth_core/src/simulation/dispatch.rs:7-354) with the reference
// defaults: decoupled colliders (coupled when the auto-coupling test fires),
// self-collision once per substep after the final pin pass.
#include <cuda_runtime.h>
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <memory>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/tcloth.h"
#include "adaptive.hpp"
#include "config.hpp"
#include "mesh.hpp"
#include "selfcol_kernels.cuh"
#include "paircache_kernels.cuh"
#include "collider_prep.cuh"
#include "solver_kernels.cuh"
#include "warmstart.cuh"

namespace tcloth {

struct TcError : std::runtime_error {
  tc_status code;
  TcError(tc_status c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define TC_CK(expr)                                                                              \
  do {                                                                                           \
    cudaError_t e__ = (expr);                                                                    \
    if (e__ != cudaSuccess)                                                                      \
      throw TcError(e__ == cudaErrorMemoryAllocation ? TC_ERR_NOMEM : TC_ERR_CUDA,               \
                    std::string(#expr) + ": " + cudaGetErrorString(e__));                        \
  } while (0)

template <class T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  DBuf() = default;
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  ~DBuf() { if (p) cudaFree(p); }
  void alloc(size_t cnt) {
    if (cnt <= n && p) return;
    if (p) { cudaFree(p); p = nullptr; }
    n = std::max<size_t>(cnt, 1);
    TC_CK(cudaMalloc(&p, n * sizeof(T)));
  }
  void upload(const T* h, size_t cnt, cudaStream_t st) {
    alloc(cnt);
    if (cnt) TC_CK(cudaMemcpyAsync(p, h, cnt * sizeof(T), cudaMemcpyHostToDevice, st));
  }
  void upload(const std::vector<T>& v, cudaStream_t st) { upload(v.data(), v.size(), st); }
};

// positions x of every vertex packed as xyz (encode_extract_positions)
__global__ void k_extract_positions(uint32_t n, const float4* __restrict__ x4, float* __restrict__ out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 x = x4[i];
  out[3 * size_t(i)] = x.x;
  out[3 * size_t(i) + 1] = x.y;
  out[3 * size_t(i) + 2] = x.z;
}

// Adaptive feedback (update_feedback_from_floats, dispatch.rs:356-429): the
// largest per-axis displacement since the previous frame (max is order-free:
// atomicMax on the bits of non-negative floats), then prev = x.
__global__ void k_fb_disp(uint32_t n, const float4* __restrict__ x4, float4* __restrict__ prev, float* out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  float d = 0.f;
  if (i < n) {
    const float4 x = x4[i], q = prev[i];
    d = fmaxf(fmaxf(fabsf(x.x - q.x), fabsf(x.y - q.y)), fabsf(x.z - q.z));
    prev[i] = x;
  }
  for (int o = 16; o > 0; o >>= 1) d = fmaxf(d, __shfl_down_sync(0xffffffffu, d, o));
  if ((threadIdx.x & 31) == 0 && d > 0.f) atomicMax(reinterpret_cast<int*>(out), __float_as_int(d));
}
// Tensile strain of every `stride`-th distance constraint against its
// initial rest length, or -1 when not stretched.
__global__ void k_fb_strain(uint32_t ns, uint32_t stride, const uint2* __restrict__ ids, const float* __restrict__ rest0,
                            const float4* __restrict__ x4, float min_ref, float* __restrict__ out) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ns) return;
  const uint32_t c = k * stride;
  const float l0 = rest0[c];
  float r = -1.f;
  if (l0 > 1e-6f) {
    const uint2 e = ids[c];
    const float4 a = x4[e.x], b = x4[e.y];
    const float dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
    const float d2 = (dx * dx + dy * dy) + dz * dz;
    if (d2 > l0 * l0) {
      const float st = (sqrtf(d2) - l0) / fmaxf(l0, min_ref);
      if (st > 0.f) r = st;
    }
  }
  out[k] = r;
}

struct PinH {
  float target[3];
  float weight;
};

// The warm-start graph MLP: fp32 master parameters with Adam moments, bf16
// copies for the tensor cores, inference activations and (allocated on first
// use) the training buffers.  Forward and backward run over one graph (the
// adjacency CSR of the cloth) on the owner's stream.
struct Mlp {
  cudaStream_t st = nullptr;
  uint32_t n = 0;
  const uint32_t* adj_off = nullptr;
  const uint32_t* adj_idx = nullptr;
  DBuf<float> w, gw, am, av;
  DBuf<__nv_bfloat16> wb, wbt;
  DBuf<__nv_bfloat16> h0, h1, h2;
  DBuf<float> y;
  DBuf<__nv_bfloat16> x0, x1, x2, dz;
  DBuf<float> z0, z1, z2, dy, dh, dx;
  DBuf<uint32_t> ell;  // inference: [n][16] degree, first 15 neighbours
  unsigned mp_grid = 1;
  // message-passing inference on the tcgen05 tensor cores (k_mlp_infer_mp_tc)
  // or, with tc = false, on warp-level mma.sync (k_mlp_infer_mp); err: the
  // device word a timed-out tensor-core wait sets to 2
  bool tc = true;
  unsigned mp_grid_tc = 1, bwd_grid_tc = 1;
  int* err = nullptr;
  uint32_t adam_t = 0;

  static unsigned grid(size_t cnt, unsigned b) { return unsigned((cnt + b - 1) / b); }
  void setup(cudaStream_t s_, uint32_t n_, const uint32_t* ao, const uint32_t* ai) {
    st = s_; n = n_; adj_off = ao; adj_idx = ai;
    w.alloc(kP_N); gw.alloc(kP_N); am.alloc(kP_N); av.alloc(kP_N);
    wb.alloc(kP_N); wbt.alloc(kT_N);
    h0.alloc(size_t(n) * kWsH); h1.alloc(size_t(n) * kWsH); h2.alloc(size_t(n) * kWsH);
    y.alloc(size_t(n) * 3);
    int dev = 0, sms = 0, per_sm = 0;
    TC_CK(cudaGetDevice(&dev));
    TC_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const unsigned tiles = grid(n, kWsRows);
    TC_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_mlp_infer_mp, 256, 0));
    mp_grid = std::max(1u, std::min(tiles, unsigned(std::max(per_sm, 1) * sms)));
    // persistent tcgen05 CTAs: the launch bounds' 3 per SM (the occupancy
    // query reports a shared-memory limit of 0 blocks for this kernel,
    // although 3 x 51 KB fit the 233 KB carveout; CTAs never wait for one
    // another, so any that do not fit simply start later), and at most
    // 512 / 64 per SM so that every resident CTA's TMEM allocation succeeds
    TC_CK(cudaFuncSetAttribute(k_mlp_infer_mp_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kWsTcSmemMp)));
    TC_CK(cudaFuncSetAttribute(k_mlp_infer_mp_tc, cudaFuncAttributePreferredSharedMemoryCarveout,
                               int(cudaSharedmemCarveoutMaxShared)));
    TC_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_mlp_infer_mp_tc, kWsTcThreads, kWsTcSmemMp));
    per_sm = std::min(std::max(per_sm, kWsTcMinBlocks), int(512 / kWsTcCols));
    mp_grid_tc = std::max(1u, std::min(unsigned(grid(n, kWsTcRows)), unsigned(per_sm * sms)));
    // backward: 2 CTAs per SM (80 KB of shared memory and 256 TMEM columns each)
    TC_CK(cudaFuncSetAttribute(k_mlp_layer_bwd_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kWsBwdSmem)));
    TC_CK(cudaFuncSetAttribute(k_mlp_layer_bwd_tc, cudaFuncAttributePreferredSharedMemoryCarveout,
                               int(cudaSharedmemCarveoutMaxShared)));
    bwd_grid_tc = std::max(1u, std::min(unsigned(grid(n, 128)), unsigned(2 * sms)));
  }
  // the ELL table of the inference kernels from the host CSR
  void set_ell(const uint32_t* h_off, const uint32_t* h_idx) {
    std::vector<uint32_t> e(size_t(n) * kWsEll, 0u);
    for (uint32_t v = 0; v < n; ++v) {
      const uint32_t b = h_off[v], d = h_off[v + 1] - b;
      e[size_t(v) * kWsEll] = d;
      for (uint32_t q = 0; q < std::min(d, uint32_t(kWsEll - 1)); ++q) e[size_t(v) * kWsEll + 1 + q] = h_idx[b + q];
    }
    ell.upload(e, st);
  }
  void alloc_train() {
    x0.alloc(size_t(n) * kWsF); x1.alloc(size_t(n) * 128); x2.alloc(size_t(n) * 128); dz.alloc(size_t(n) * kWsH);
    z0.alloc(size_t(n) * kWsH); z1.alloc(size_t(n) * kWsH); z2.alloc(size_t(n) * kWsH);
    dy.alloc(size_t(n) * 3); dh.alloc(size_t(n) * kWsH); dx.alloc(size_t(n) * 128);
  }
  // seeded init: uniform(-1/sqrt(in), 1/sqrt(in)), the head scaled by 0.1 so
  // that an untrained network moves vertices by little; zero biases
  static std::vector<float> init_blob(uint64_t seed) {
    std::vector<float> h(kP_N, 0.f);
    uint64_t x = seed * 6364136223846793005ull + 1442695040888963407ull;
    auto uni = [&]() {
      x = x * 6364136223846793005ull + 1442695040888963407ull;
      return float((x >> 40) & 0xFFFFFF) / float(1 << 24) * 2.f - 1.f;
    };
    auto fill = [&](uint32_t off, uint32_t cnt, float sc) { for (uint32_t e = 0; e < cnt; ++e) h[off + e] = uni() * sc; };
    fill(kP_W0, kP_b0 - kP_W0, 1.f / std::sqrt(16.f));
    fill(kP_W1, kP_b1 - kP_W1, 1.f / std::sqrt(128.f));
    fill(kP_W2, kP_b2 - kP_W2, 1.f / std::sqrt(128.f));
    fill(kP_W3, kP_b3 - kP_W3, 0.1f / std::sqrt(64.f));
    for (uint32_t e = kP_FS; e < kP_N; ++e) h[e] = 1.f;  // identity normalizer
    return h;
  }
  void set_params(const float* h) {
    TC_CK(cudaMemcpyAsync(w.p, h, kP_N * sizeof(float), cudaMemcpyHostToDevice, st));
    TC_CK(cudaMemsetAsync(am.p, 0, kP_N * sizeof(float), st));
    TC_CK(cudaMemsetAsync(av.p, 0, kP_N * sizeof(float), st));
    adam_t = 0;
    refresh();
    TC_CK(cudaStreamSynchronize(st));
  }
  void get_params(float* h) {
    TC_CK(cudaMemcpyAsync(h, w.p, kP_N * sizeof(float), cudaMemcpyDeviceToHost, st));
    TC_CK(cudaStreamSynchronize(st));
  }
  void refresh() { k_ws_refresh<<<grid(kP_N, 256), 256, 0, st>>>(w.p, wb.p, wbt.p); }

  // Y = MLP(feat); with train, keeps X1, X2, Z0..Z2 and (with target) writes
  // dY and adds the loss to *loss.
  void forward(const __nv_bfloat16* feat, bool train, const float* target, const float* mask, float* loss) {
    if (!n) return;
    MlpLayerArgs a{};
    a.n = n; a.adj_off = adj_off; a.adj_idx = adj_idx;
    a.kin = kWsF; a.x_feat = feat; a.fscale = w.p + kP_FS; a.wt = wbt.p + kT_W0; a.bias = w.p + kP_b0;
    a.x_out = train ? x0.p : nullptr; a.z_out = train ? z0.p : nullptr; a.h_out = h0.p;
    k_mlp_layer_fwd<<<grid(n, kWsRows), kWsFwdThreads, 0, st>>>(a);
    if (tc) {  // the message-passing layers on tcgen05, with the training outputs
      MlpInferArgs b{};
      b.n = n; b.ell = ell.p; b.adj_off = adj_off; b.adj_idx = adj_idx; b.err = err;
      b.h_prev = h0.p; b.wt = wbt.p + kT_W1; b.bias = w.p + kP_b1; b.h_out = h1.p;
      b.x_out = train ? x1.p : nullptr; b.z_out = train ? z1.p : nullptr;
      k_mlp_infer_mp_tc<<<mp_grid_tc, kWsTcThreads, kWsTcSmemMp, st>>>(b);
      b.h_prev = h1.p; b.wt = wbt.p + kT_W2; b.bias = w.p + kP_b2; b.h_out = h2.p;
      b.x_out = train ? x2.p : nullptr; b.z_out = train ? z2.p : nullptr;
      k_mlp_infer_mp_tc<<<mp_grid_tc, kWsTcThreads, kWsTcSmemMp, st>>>(b);
    } else {
      a.kin = 128; a.x_feat = nullptr; a.fscale = nullptr; a.h_prev = h0.p; a.wt = wbt.p + kT_W1; a.bias = w.p + kP_b1;
      a.x_out = train ? x1.p : nullptr; a.z_out = train ? z1.p : nullptr; a.h_out = h1.p;
      k_mlp_layer_fwd<<<grid(n, kWsRows), kWsFwdThreads, 0, st>>>(a);
      a.h_prev = h1.p; a.wt = wbt.p + kT_W2; a.bias = w.p + kP_b2;
      a.x_out = train ? x2.p : nullptr; a.z_out = train ? z2.p : nullptr; a.h_out = h2.p;
      k_mlp_layer_fwd<<<grid(n, kWsRows), kWsFwdThreads, 0, st>>>(a);
    }
    k_mlp_head<<<grid(n, 256), 256, 0, st>>>(n, h2.p, wb.p + kP_W3, w.p + kP_b3, y.p, target, mask, w.p + kP_YS,
                                             1.0f / float(n), target ? dy.p : nullptr, loss);
  }
  // inference: layer 0 from the given features (feat) or computed from fa
  // (then p is kept in ppred first); the head is fused into the last layer,
  // which either writes Y (y_out) or moves p by Y YS L on free vertices
  void infer(const __nv_bfloat16* feat, const WsFeatArgs* fa, float4* ppred, float* y_out, const float4* x4,
             float4* p4, const float* local_len) {
    if (!n) return;
    MlpInferArgs a{};
    a.n = n; a.x_feat = feat; if (fa) a.fa = *fa; a.ppred = ppred; a.fscale = w.p + kP_FS;
    a.wt = wbt.p + kT_W0; a.bias = w.p + kP_b0; a.h_out = h0.p;
    k_mlp_infer_l0<<<grid(n, kWsL0Rows), kWsL0Rows, 0, st>>>(a);
    a.ell = ell.p; a.adj_off = adj_off; a.adj_idx = adj_idx; a.err = err;
    auto mp = [&]() {
      if (tc) k_mlp_infer_mp_tc<<<mp_grid_tc, kWsTcThreads, kWsTcSmemMp, st>>>(a);
      else k_mlp_infer_mp<<<mp_grid, 256, 0, st>>>(a);
    };
    a.h_prev = h0.p; a.wt = wbt.p + kT_W1; a.bias = w.p + kP_b1; a.h_out = h1.p;
    mp();
    a.h_prev = h1.p; a.wt = wbt.p + kT_W2; a.bias = w.p + kP_b2; a.h_out = nullptr;
    a.w3 = wb.p + kP_W3; a.b3 = w.p + kP_b3; a.yscale = w.p + kP_YS; a.y_out = y_out; a.x4 = x4; a.p4 = p4;
    a.local_len = local_len;
    mp();
  }
  // gradients of the loss of the last forward(train, target) into gw (layer
  // 0's input is the scaled copy x0 that forward kept)
  void backward() {
    TC_CK(cudaMemsetAsync(gw.p, 0, kP_N * sizeof(float), st));
    if (!n) return;
    const unsigned gh = grid(size_t(n) * kWsH, 256), gt = grid(n, kWsRows);
    k_mlp_head_bwd<<<grid(n, 256), 256, 0, st>>>(n, h2.p, wb.p + kP_W3, dy.p, dh.p, gw.p + kP_W3, gw.p + kP_b3);
    k_mlp_act_bwd<<<gh, 256, 0, st>>>(n, dh.p, z2.p, dz.p, gw.p + kP_b2);
    auto bwd128 = [&](const __nv_bfloat16* x, uint32_t wo) {
      if (tc)
        k_mlp_layer_bwd_tc<<<bwd_grid_tc, 256, kWsBwdSmem, st>>>(
            MlpBwdTcArgs{n, x, dz.p, wb.p + wo, gw.p + wo, dx.p, err});
      else
        k_mlp_layer_bwd<<<gt, 128, 0, st>>>(MlpBwdArgs{n, 128, x, dz.p, wb.p + wo, gw.p + wo, dx.p});
    };
    bwd128(x2.p, kP_W2);
    k_mlp_agg_bwd<<<gh, 256, 0, st>>>(n, dx.p, adj_off, adj_idx, dh.p);
    k_mlp_act_bwd<<<gh, 256, 0, st>>>(n, dh.p, z1.p, dz.p, gw.p + kP_b1);
    bwd128(x1.p, kP_W1);
    k_mlp_agg_bwd<<<gh, 256, 0, st>>>(n, dx.p, adj_off, adj_idx, dh.p);
    k_mlp_act_bwd<<<gh, 256, 0, st>>>(n, dh.p, z0.p, dz.p, gw.p + kP_b0);
    k_mlp_layer_bwd<<<gt, 128, 0, st>>>(MlpBwdArgs{n, kWsF, x0.p, dz.p, wb.p + kP_W0, gw.p + kP_W0, nullptr});
  }
  // Normalizer from `rows` recorded rows (features, targets, free mask): FS =
  // 1 / RMS of each feature, YS = RMS of the target components, over the
  // free rows; FS clamped to [1e-4, 1e4], 1 where a feature is all zero.
  void fit_normalizer(const __nv_bfloat16* feat, const float* target, const float* mask, size_t rows) {
    DBuf<float> part;
    part.alloc(size_t(kWsMomBlocks) * kWsMom);
    k_ws_moments<<<kWsMomBlocks, 256, 0, st>>>(rows, feat, target, mask, part.p);
    std::vector<float> h(size_t(kWsMomBlocks) * kWsMom), blob(kP_N);
    TC_CK(cudaMemcpyAsync(h.data(), part.p, h.size() * sizeof(float), cudaMemcpyDeviceToHost, st));
    TC_CK(cudaMemcpyAsync(blob.data(), w.p, kP_N * sizeof(float), cudaMemcpyDeviceToHost, st));
    TC_CK(cudaStreamSynchronize(st));
    double sum[kWsMom] = {};
    for (int b = 0; b < kWsMomBlocks; ++b)
      for (int c = 0; c < kWsMom; ++c) sum[c] += h[size_t(b) * kWsMom + c];
    const double cnt = sum[kWsF + 1];
    if (cnt <= 0.0) return;
    for (int c = 0; c < kWsF; ++c) {
      const double rms = std::sqrt(sum[c] / cnt);
      blob[kP_FS + c] = rms > 0.0 ? float(std::min(std::max(1.0 / rms, 1e-4), 1e4)) : 1.f;
    }
    const double yr = std::sqrt(sum[kWsF] / (3.0 * cnt));
    blob[kP_YS] = yr > 0.0 && std::isfinite(yr) ? float(yr) : 1.f;
    set_params(blob.data());
  }
  void adam(float lr) {
    ++adam_t;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, float(adam_t)), c2 = 1.f - std::pow(b2, float(adam_t));
    k_adam<<<grid(kP_N, 256), 256, 0, st>>>(kP_N, w.p, gw.p, am.p, av.p, lr, b1, b2, 1e-8f, c1, c2, nullptr, nullptr, 0, 0);
    refresh();
  }
};

// Tiles of 32 consecutive triangles per bone for the bake's sphere culling.
struct BakeTiles {
  std::vector<uint32_t> first, cnt, bone_off;  // per tile; per bone: first tile
};
static BakeTiles make_bake_tiles(const std::vector<uint32_t>& start, const std::vector<uint32_t>& count,
                                 uint32_t size = 32) {
  BakeTiles t;
  t.bone_off.resize(start.size() + 1);
  for (size_t b = 0; b < start.size(); ++b) {
    t.bone_off[b] = uint32_t(t.first.size());
    for (uint32_t k = 0; k < count[b]; k += size) {
      t.first.push_back(start[b] + k);
      t.cnt.push_back(std::min(size, count[b] - k));
    }
  }
  t.bone_off[start.size()] = uint32_t(t.first.size());
  return t;
}

// Spatial order of each bone's triangles for the bake's order-free passes:
// within [start[b], start[b] + count[b]) the triangle indices sorted by the
// 30-bit Morton code of their centroid in the bone range's bounding box
// (stable, so equal codes keep the triangle order).  Only the culling depends
// on this order, not the baked values.
static std::vector<uint32_t> bake_spatial_perm(const std::vector<float>& cent, const std::vector<uint32_t>& start,
                                               const std::vector<uint32_t>& count, uint32_t nt) {
  std::vector<uint32_t> perm(nt);
  for (uint32_t t = 0; t < nt; ++t) perm[t] = t;
  // ranges that overlap or leave [0, nt) keep the triangle order everywhere
  std::vector<std::pair<uint32_t, uint32_t>> rg;
  for (size_t b = 0; b < start.size(); ++b)
    if (count[b]) rg.emplace_back(start[b], count[b]);
  std::sort(rg.begin(), rg.end());
  for (size_t i = 0; i < rg.size(); ++i)
    if (uint64_t(rg[i].first) + rg[i].second > nt || (i && uint64_t(rg[i - 1].first) + rg[i - 1].second > rg[i].first))
      return perm;
  for (size_t b = 0; b < start.size(); ++b) {
    const uint32_t s0 = start[b], c = count[b];
    if (c < 2) continue;
    float lo[3] = {1e30f, 1e30f, 1e30f}, hi[3] = {-1e30f, -1e30f, -1e30f};
    for (uint32_t i = s0; i < s0 + c; ++i)
      for (int a = 0; a < 3; ++a) {
        const float v = cent[3 * size_t(i) + a];
        if (std::isfinite(v)) { lo[a] = std::min(lo[a], v); hi[a] = std::max(hi[a], v); }
      }
    std::vector<std::pair<uint32_t, uint32_t>> key(c);
    for (uint32_t i = 0; i < c; ++i) {
      uint32_t code = 0;
      for (int a = 0; a < 3; ++a) {
        const float span = hi[a] > lo[a] ? hi[a] - lo[a] : 1.f;
        const float v = cent[3 * size_t(s0 + i) + a];
        const float u = std::isfinite(v) ? (v - lo[a]) / span : 0.f;
        const uint32_t q = uint32_t(std::min(std::max(u, 0.f), 1.f) * 1023.f);
        for (int bit = 0; bit < 10; ++bit) code |= ((q >> bit) & 1u) << (3 * bit + a);
      }
      key[i] = {code, s0 + i};
    }
    std::stable_sort(key.begin(), key.end(), [](const auto& x, const auto& y) { return x.first < y.first; });
    for (uint32_t i = 0; i < c; ++i) perm[s0 + i] = key[i].second;
  }
  return perm;
}

// Device side of a bake: triangles, spheres, tiles, parameters.  Two tile
// sets share one layout (32 positions per tile, the same tiles per bone):
// triangle-order tiles over the triangles themselves (`tsph`) and spatial
// tiles over `perm` (`psph`, the triangle spheres in perm order; `stsph`).
struct BakeGpu {
  DBuf<BakeTri> tris;
  DBuf<float4> sph, tsph, psph, stsph, ssph;
  DBuf<uint32_t> tile_first, tile_cnt, tile_off, param_bone, perm, sub_first, sub_cnt, sub_off;
  DBuf<BakeParams> params;
  uint32_t nt = 0, ntiles = 0, nsub = 0;
  void setup_tiles(const BakeTiles& t, cudaStream_t st) {
    ntiles = uint32_t(t.first.size());
    tile_first.upload(t.first, st);
    tile_cnt.upload(t.cnt, st);
    tile_off.upload(t.bone_off, st);
    sph.alloc(std::max<uint32_t>(nt, 1));
    tsph.alloc(std::max<uint32_t>(ntiles, 1));
    psph.alloc(std::max<uint32_t>(nt, 1));
    stsph.alloc(std::max<uint32_t>(ntiles, 1));
  }
  // the bone bake needs the spatial order (bake_spatial_perm) as well, and
  // sub-tiles of 8 positions (`sub`, spheres `ssph`) within its spatial tiles
  void setup_spatial(const std::vector<uint32_t>& p, const std::vector<uint32_t>& start,
                     const std::vector<uint32_t>& count, cudaStream_t st) {
    if (p.size() != nt) throw std::runtime_error("bake permutation size");
    if (nt) perm.upload(p, st);
    const BakeTiles sub = make_bake_tiles(start, count, 8);
    nsub = uint32_t(sub.first.size());
    sub_first.upload(sub.first, st);
    sub_cnt.upload(sub.cnt, st);
    sub_off.upload(sub.bone_off, st);
    ssph.alloc(std::max<uint32_t>(nsub, 1));
  }
  // spheres of the current triangles, then the bake of the listed entries
  void bake(const std::vector<BakeParams>& ps, const std::vector<uint32_t>& bones, uint32_t* atlas, cudaStream_t st) {
    if (ps.empty()) return;
    if (nt && !perm.p) throw std::runtime_error("bone bake without its spatial order");
    if (nt) k_bone_tri_spheres<<<(nt + 255) / 256, 256, 0, st>>>(nt, tris.p, sph.p);
    if (nt) k_bake_perm_spheres<<<(nt + 255) / 256, 256, 0, st>>>(nt, perm.p, sph.p, psph.p);
    if (ntiles) k_bone_tile_spheres<<<(ntiles + 127) / 128, 128, 0, st>>>(ntiles, tile_first.p, tile_cnt.p, sph.p, tsph.p);
    if (ntiles)
      k_bone_tile_spheres<<<(ntiles + 127) / 128, 128, 0, st>>>(ntiles, tile_first.p, tile_cnt.p, psph.p, stsph.p);
    if (nsub) k_bone_tile_spheres<<<(nsub + 127) / 128, 128, 0, st>>>(nsub, sub_first.p, sub_cnt.p, psph.p, ssph.p);
    params.upload(ps, st);
    param_bone.upload(bones, st);
    uint32_t res = 0;
    for (const auto& q : ps) res = std::max(res, q.res);
    const uint32_t nblk = ((res + 7) / 8) * ((res + 7) / 8) * ((res + 3) / 4);  // 8 x 8 x 4 regions
    k_bone_bake<<<dim3(nblk, uint32_t(ps.size())), kBakeCol, 0, st>>>(params.p, tris.p, sph.p, tsph.p, perm.p, psph.p,
                                                                 stsph.p, ssph.p, tile_off.p, sub_off.p,
                                                                 param_bone.p, atlas);
  }
};

// Bone SDF colliders (simulation/mod.rs:1630-1960, :1998-2464): atlas,
// per-bone infos and transforms, and the dynamic path (skinning, triangle
// preparation and rebake of dirty bones before a frame).
struct BoneSdfState {
  std::vector<BoneInfo> info_h;
  std::vector<BoneXform> xf_h;
  DBuf<BoneInfo> info;
  DBuf<BoneXform> xf;
  DBuf<uint32_t> atlas;
  uint32_t w = 0, h = 0, d = 0;
  bool enabled = false;
  // dynamic
  bool dyn = false, dyn_on = false, baked = false;
  uint32_t interval = 1, res = 0, nv = 0, nb = 0;
  uint64_t counter = 0;
  bool dirty_set = false;
  std::vector<uint32_t> dirty;
  std::vector<float> bind_inv;  // nb x 16, row-major
  std::vector<BakeParams> params_h;
  DBuf<float4> rest, bw, skinned;
  DBuf<uint4> bidx, tsrc;
  DBuf<float4> tsrcw;
  DBuf<float> skin_m, inv_m;
  BakeGpu bake;
};

// Collider edges of the mesh-collider triangles (extract_collider_edges,
// mesh.rs:1503-1565) and their grid (build_collider_edge_grid,
// spatial_hash.rs:463-528): every cell an edge passes through, sampled at
// half-cell steps, registered once per distinct hash bucket.  Edges are kept
// in first-seen order (the reference's hash-map order differs; the contacts
// are integer sums with no cap, so the result does not depend on it).
constexpr uint32_t kColEdgeTable = 32768;
inline int32_t sat_i32(float f) {
  if (!(f == f)) return 0;
  if (f <= -2147483648.f) return INT32_MIN;
  if (f >= 2147483647.f) return INT32_MAX;
  return int32_t(f);
}
static void build_collider_edges(const std::vector<MeshTri>& tris, float cell, std::vector<ColEdge>& out,
                                 std::vector<uint32_t>& cs, std::vector<uint32_t>& srt) {
  out.clear();
  std::map<std::array<uint32_t, 6>, uint32_t> at;
  auto bits = [](const float* p, uint32_t* b) { std::memcpy(b, p, 12); };
  for (const MeshTri& t : tris) {
    const float* P[3] = {&t.p0f.x, &t.p1t.x, &t.p2r.x};
    const float e1[3] = {P[1][0] - P[0][0], P[1][1] - P[0][1], P[1][2] - P[0][2]};
    const float e2[3] = {P[2][0] - P[0][0], P[2][1] - P[0][1], P[2][2] - P[0][2]};
    const float cr[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
    const float cl = std::sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
    const float tn[3] = {cl > 1e-12f ? cr[0] / cl : 0.f, cl > 1e-12f ? cr[1] / cl : 0.f, cl > 1e-12f ? cr[2] / cl : 0.f};
    uint32_t tf;
    std::memcpy(&tf, &t.fl.x, 4);
    const uint32_t single = tf & 1u;
    for (int k = 0; k < 3; ++k) {
      const float *a = P[k], *b = P[(k + 1) % 3];
      std::array<uint32_t, 6> key;
      uint32_t ba[3], bb[3];
      bits(a, ba);
      bits(b, bb);
      const bool a_first = std::lexicographical_compare(ba, ba + 3, bb, bb + 3);
      for (int j = 0; j < 3; ++j) { key[j] = a_first ? ba[j] : bb[j]; key[3 + j] = a_first ? bb[j] : ba[j]; }
      auto it = at.find(key);
      if (it == at.end()) {
        at.emplace(key, uint32_t(out.size()));
        float fb;
        std::memcpy(&fb, &single, 4);
        out.push_back(ColEdge{make_float4(a[0], a[1], a[2], t.p1t.w), make_float4(b[0], b[1], b[2], t.p0f.w),
                              make_float4(tn[0], tn[1], tn[2], fb)});
      } else {
        ColEdge& c = out[it->second];
        c.p0t.w = std::fmax(c.p0t.w, t.p1t.w);
        c.p1f.w = (c.p1f.w + t.p0f.w) * 0.5f;
        c.nfl.x += tn[0]; c.nfl.y += tn[1]; c.nfl.z += tn[2];
        uint32_t f;
        std::memcpy(&f, &c.nfl.w, 4);
        f &= single;
        std::memcpy(&c.nfl.w, &f, 4);
      }
    }
  }
  for (ColEdge& c : out) {
    const float nl = std::sqrt(c.nfl.x * c.nfl.x + c.nfl.y * c.nfl.y + c.nfl.z * c.nfl.z);
    if (nl > 1e-6f) { c.nfl.x /= nl; c.nfl.y /= nl; c.nfl.z /= nl; }
    else { c.nfl.x = c.nfl.y = c.nfl.z = 0.f; }
  }
  const float safe = std::fmax(cell, 1e-4f), pitch = safe * 0.5f;
  const uint32_t T = kColEdgeTable;
  std::vector<uint32_t> cnt(T, 0), hs;
  std::vector<std::pair<uint32_t, uint32_t>> ent;
  for (uint32_t ei = 0; ei < out.size(); ++ei) {
    const ColEdge& c = out[ei];
    const float dx = c.p1f.x - c.p0t.x, dy = c.p1f.y - c.p0t.y, dz = c.p1f.z - c.p0t.z;
    const float len = std::sqrt(dx * dx + dy * dy + dz * dz);
    const float sf = std::ceil(len / pitch);
    size_t steps = (sf == sf && sf > 0.f) ? (sf >= 4096.f ? 4096 : size_t(sf)) : 0;
    steps = std::min<size_t>(std::max<size_t>(steps, 1), 4096);
    hs.clear();
    for (size_t k = 0; k <= steps; ++k) {
      const float t = float(k) / float(steps);
      const float px = c.p0t.x + dx * t, py = c.p0t.y + dy * t, pz = c.p0t.z + dz * t;
      const uint32_t h = ((uint32_t)sat_i32(std::floor(px / safe)) * 73856093u ^
                          (uint32_t)sat_i32(std::floor(py / safe)) * 19349663u ^
                          (uint32_t)sat_i32(std::floor(pz / safe)) * 83492791u) % T;
      hs.push_back(h);
    }
    std::sort(hs.begin(), hs.end());
    hs.erase(std::unique(hs.begin(), hs.end()), hs.end());
    for (uint32_t h : hs) { cnt[h]++; ent.push_back({h, ei}); }
  }
  cs.assign(T + 1, 0);
  for (uint32_t i = 0; i < T; ++i) cs[i + 1] = cs[i] + cnt[i];
  std::vector<uint32_t> cur(cs.begin(), cs.end() - 1);
  srt.assign(ent.size(), 0);
  for (const auto& e : ent) srt[cur[e.first]++] = e.second;
}

// Learned warm start state of one simulator: the network, the correction of
// the previous substep, the in-kernel residual judge and the recorded
// training snapshots (features, target correction / L, free mask).
struct WarmStart {
  Mlp net;
  bool ready = false;  // buffers allocated
  bool normalized = false;  // the network's normalizer is set (fitted or loaded)
  bool on = false;
  uint32_t k = 1;
  float res_thresh = 0.f;
  float res_ratio = 0.f;  // > 0: threshold = res_ratio x residual of the predicted positions
  DBuf<float4> ppred, dprev;
  DBuf<float> adj_rest, res_max, res_part, res_pred;
  DBuf<unsigned int> fallbacks, gate;
  uint64_t substeps_run = 0;
  // recording
  uint32_t rec_cap = 0, rec_count = 0, rec_every = 1, rec_phase = 0;
  DBuf<__nv_bfloat16> rec_feat;
  DBuf<float> rec_target, rec_mask, losses;
};

struct Sim {
  int device = 0;
  uint64_t epoch = 0;       // device-context epoch at creation (device health below)
  bool nonfinite_check = false;  // read-backs refuse non-finite positions
  cudaStream_t st = nullptr;
  MeshData m;
  uint32_t n = 0, nd = 0, nb = 0, ne = 0;
  // host mirrors
  std::vector<float> orig_w, init_w, init_pos;
  std::vector<int64_t> orig_edge_to_dist;
  std::vector<float> mult;  // per sorted distance constraint
  std::vector<DistC> dist_h;
  std::vector<BendC> bend_h;
  std::vector<float> base_rest;
  float base_tc = 0, base_cc = 0, base_shc = 0, base_bk = 0;
  // device state
  DBuf<float4> x4, p4, v4;
  DBuf<float> local_len, dlam, blam, th_rest;
  DBuf<uint2> dist_ids, star_idx, edges;
  DBuf<float4> dist_par, bend_par;
  DBuf<uint4> bend_ids;
  DBuf<uint32_t> adj_off, adj_idx, th_off, th_idx, star_off, edge_bits;
  DBuf<uint32_t> keys, counts, cursor, cs, srt, ekeys, ecs, esrt, ecounts, ecursor, etile_sum;
  cudaStream_t st2 = nullptr;  // edge side of self-collision
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  DBuf<float4> nrm;
  DBuf<int32_t> acc;
  DBuf<int4> vcell, ecell;
  DBuf<float4> sbox;
  DBuf<float> mlen;
  DBuf<float4> eamin, eamax;
  DBuf<float4> vs_p, vs_q, es_lo, es_hi;
  DBuf<uint32_t> tile_sum;
  DBuf<int4> vs_c, es_c;
  DBuf<uint2> es_v, ccd_q, ee_q;
  DBuf<uint32_t> ccd_n;  // [0] deferred CCD pairs, [1 + g] listed E-E pairs of segment g
  // contact-pair cache (self-collision algorithm 1; simulation/mod.rs:582-600,
  // :799-893, dispatch.rs:1540-1670), off by default; buffers on first use
  bool pair_cache = false, pair_final_fallback = true;
  uint32_t sc_algorithm = 0;
  uint32_t pair_max_vt = 0, pair_max_ee = 0, pair_qvt = 1, pair_qee = 1;
  uint32_t pair_margin_mode = 1;
  float pair_safety = 0.005f, pair_hscale = 1.3f, pair_max_h = 0.02f;
  DBuf<uint4> pair_vt, pair_ee;
  DBuf<uint32_t> pair_cnt, island_d;
  DBuf<float> pair_hz;
  // quota_for_budget (simulation/mod.rs:36-41)
  static uint32_t quota_for_budget(uint32_t budget, uint32_t nv) {
    return nv == 0 ? 1u : std::min(std::max(budget / nv, 1u), kPairQuotaMax);
  }
  void pair_defaults() {
    pair_max_vt = pair_max_ee = std::min(std::max(n * 8u, 8192u), 262144u);
    pair_qvt = quota_for_budget(pair_max_vt, n);
    pair_qee = quota_for_budget(pair_max_ee, n);
  }
  void ensure_pair_buffers() {
    if (pair_vt.p) return;
    const size_t slots = std::max<size_t>(size_t(n) * kPairQuotaMax, 64);
    pair_vt.alloc(slots);
    pair_ee.alloc(slots);
    pair_cnt.alloc(4);
    pair_hz.alloc(n);
    island_d.upload(m.island, st);
    TC_CK(cudaMemsetAsync(pair_vt.p, 0xFF, slots * sizeof(uint4), st));
    TC_CK(cudaMemsetAsync(pair_ee.p, 0xFF, slots * sizeof(uint4), st));
    TC_CK(cudaMemsetAsync(pair_cnt.p, 0, 4 * sizeof(uint32_t), st));
    TC_CK(cudaStreamSynchronize(st));
  }
  void set_pair_cache(bool on) {
    if (on) ensure_pair_buffers();
    pair_cache = on;
    mark();
  }
  // colliders
  std::vector<Prim> prims_h;
  std::vector<MeshTri> tris_h;
  // edge colliders (edge_collision.wgsl; simulation/mod.rs:1007-1025): off by default
  bool edge_collision = false;
  float edge_mscale = 1.f, edge_moff = 0.f;
  std::vector<ColEdge> cedges_h;
  DBuf<ColEdge> cedges;
  DBuf<uint32_t> ce_cs, ce_srt;
  float ce_cell = 0.01f;  // the grid's cell, fixed when it is built (the reference's is fixed at creation)
  bool ce_stale = true;   // triangles changed since the collider edges were built
  bool edge_active() const { return edge_collision && has_colliders() && ne > 0; }
  // built when first needed after the triangles change: frames without edge
  // collision never pay for it (the reference extracts on every upload)
  void ensure_collider_edges() {
    if (ce_stale) rebuild_collider_edges();
  }
  void rebuild_collider_edges() {
    ce_stale = false;
    std::vector<uint32_t> cs, srt;
    ce_cell = m.cell;
    const size_t n_before = cedges_h.size();
    build_collider_edges(host_tris(), ce_cell, cedges_h, cs, srt);
    const void* before[3] = {cedges.p, ce_cs.p, ce_srt.p};
    cedges.upload(cedges_h, st);
    ce_cs.upload(cs, st);
    ce_srt.upload(srt, st);
    TC_CK(cudaStreamSynchronize(st));
    // a recorded frame holds the pointers and the edge count only
    const void* after[3] = {cedges.p, ce_cs.p, ce_srt.p};
    if (cedges_h.size() != n_before || std::memcmp(before, after, sizeof before) != 0) mark();
  }
  // edge colliders after the final pins, then the apply pass (dispatch.rs:254-283)
  void encode_edge_collision() {
    EdgeColArgs a{ne, uint32_t(cedges_h.size()), edges.p, x4.p, p4.p, cedges.p, ce_cs.p, ce_srt.p, ce_cell,
                  kColEdgeTable, edge_mscale, edge_moff, acc.p};
    timed("edge_collision", [&] { k_edge_collision<<<grid(ne, 256), 256, 0, st>>>(a); });
    timed("edge_apply", [&] {
      k_apply<<<grid(n, 256), 256, 0, st>>>(n, x4.p, p4.p, local_len.p, acc.p, relief, enable_relief ? 1 : 0,
                                             max_disp_ratio);
    });
  }
  DBuf<Prim> prims;
  DBuf<MeshTri> tris;
  DBuf<float4> bounds, cl16, cl256, cl4096;
  // device-side upload of the mesh collider (collider_prep.cuh): input floats
  // through a pinned staging buffer, packed triangles, Morton keys, sort scratch
  uint32_t ntris = 0;         // triangles in `tris`
  bool tris_h_valid = true;   // tris_h mirrors `tris` (refreshed when a host step needs it)
  DBuf<float> col_in, col_box;
  DBuf<MeshTri> col_raw;
  DBuf<uint32_t> col_code, col_code2, col_idx, col_idx2;
  DBuf<unsigned char> col_tmp;
  float* h_col = nullptr;
  size_t h_col_cap = 0;       // floats the staging buffer holds
  cudaEvent_t col_ev = nullptr;
  bool col_ev_used = false;   // col_ev marks the last copy out of h_col
  // batched instances (empty for a single cloth)
  std::vector<uint32_t> inst_vert_off;  // n_instances + 1
  // cluster solver: bins of whole instances, one thread-block cluster each
  static constexpr uint32_t kClusterCtas = 8;
  bool cluster_mode = false, cl_stale = true;
  int cl_max_active = 0;
  uint32_t cl_bins = 0;
  DBuf<uint2> cl_vrange, cl_pins, cl_dist, cl_bend;
  DBuf<uint32_t> cl_dperm, cl_bperm;
  // staged cluster solver: the same bins with each bin's vertex records in
  // the shared memory of its cluster (k_solver_staged); st_cap vertices per
  // CTA slice, kStageCtas slices per bin
  static constexpr uint32_t kStageCtas = 8;
  static constexpr uint32_t kStageThreads = 512;
  bool stage_mode = false, st_stale = true;
  int st_max_active = 0;
  uint32_t st_cap = 0, st_bins = 0;
  size_t st_smem = 0;
  DBuf<uint2> st_vrange, st_pins;
  DBuf<uint32_t> st_dist, st_bend, st_dperm, st_bperm;
  DBuf<uint2> st_dids;
  DBuf<uint4> st_bids;
  DBuf<float4> st_dpar, st_bpar;
  DBuf<float> st_dlam, st_blam;
  std::vector<uint2> inst_prims_h;
  DBuf<uint32_t> vinst;
  DBuf<uint2> inst_prims;
  // pins
  std::map<uint32_t, PinH> pins;
  DBuf<uint32_t> pin_v;
  DBuf<float4> pin_t;
  // persistent solver (one cooperative launch per substep / frame)
  bool persistent = true;
  unsigned int persist_blocks = 0, persist_max_per_sm = 0, num_sms = 0, persist_bone_per_sm = 0;
  unsigned int spin_limit = 1u << 22;  // ~0.5 s of polling per barrier
  DBuf<GridBar> bar;
  DBuf<uint32_t> dist_offc, dist_cntc, bend_offc, bend_cntc;
  // sewing (mesh.rs:904-936; settings dispatch.rs:29-35, simulation/mod.rs:1211-1420)
  uint32_t nsw = 0;
  std::vector<SewC> sew_h;              // colour-sorted, as uploaded
  DBuf<uint2> sew_ids;
  DBuf<float2> sew_rest;                // (current, target)
  DBuf<float> slam;
  DBuf<uint32_t> sew_offc, sew_cntc;
  float sew_stiffness = 10000.f, sew_speed = 1.f, sew_lock_dist = 0.02f;
  bool sew_lock = true;
  // sewing priority: gravity held at 0 until the seams close, then ramped
  // back over ramp_frames frames (simulation/mod.rs:1257-1420)
  struct SewPriority {
    bool enabled = false;
    float threshold = 0.9f, merge = 0.005f;
    uint32_t ramp_frames = 3, max_frames = 600;
    bool latched = false;
    uint32_t frame = 0;
    float ramp_t = 0.f, ratio = 0.f;
  } pri;
  float priority_scale() const {  // sewing_priority_scale (mod.rs:1359-1371)
    if (!pri.enabled || nsw == 0) return 1.f;
    if (!pri.latched) return 0.f;
    if (pri.ramp_frames == 0) return 1.f;
    const float x = std::fmin(std::fmax(pri.ramp_t, 0.f), 1.f);
    return x * x * (3.0f - 2.0f * x);
  }
  SewParams sew_params() const {
    return SewParams{sew_stiffness >= 5000.f ? 0.f : 1.f / std::fmax(sew_stiffness, 1.f), sew_lock ? 1.f : 0.f,
                     sew_lock_dist};
  }
  // substep parameters of a frame: gravity scaled by the sewing priority
  SubstepParams make_sp(float dts) const {
    const float k = priority_scale();
    return SubstepParams{dts, g[0] * k, g[1] * k, g[2] * k, damping, td, cd, sd, bd};
  }
  void upload_sew() {
    std::vector<uint2> ids(nsw);
    std::vector<float2> rest(nsw);
    for (uint32_t i = 0; i < nsw; ++i) {
      ids[i] = make_uint2(sew_h[i].v0, sew_h[i].v1);
      rest[i] = make_float2(sew_h[i].cur_rest, sew_h[i].target_rest);
    }
    sew_ids.upload(ids, st);
    sew_rest.upload(rest, st);
    slam.alloc(nsw);
    sew_offc.upload(m.sew_off, st);
    sew_cntc.upload(m.sew_cnt, st);
  }
  // per-colour sewing projection (the iteration's pass, or the final one)
  void launch_sewing(float dts, const unsigned int* gate = nullptr) {
    const SewParams sw = sew_params();
    for (size_t c = 0; c < m.sew_cnt.size(); ++c)
      if (m.sew_cnt[c])
        launch_k(k_sewing, grid(m.sew_cnt[c], 256), 256, m.sew_off[c], m.sew_cnt[c], (const uint2*)sew_ids.p,
                 sew_rest.p, (const float4*)x4.p, p4.p, slam.p, dts, sw, gate);
  }
  // at the start of a substep: sewing lambdas cleared, rest lengths shrunk
  void launch_sew_start(float dts) {
    if (!nsw) return;
    TC_CK(cudaMemsetAsync(slam.p, 0, nsw * sizeof(float), st));
    launch_k(k_sew_shrink, grid(nsw, 256), 256, nsw, sew_rest.p, sew_speed, dts);
  }
  int* h_err = nullptr;  // pinned
  WarmStart ws;
  BoneSdfState bone;
  // adaptive substeps / iterations with their GPU feedback (max displacement,
  // strided strain sample), read after each frame
  AdaptiveCtl ad;
  DBuf<float4> fb_prev;
  DBuf<float> fb_out, rest0;
  float* h_fb = nullptr;  // pinned: [0] = max displacement, [1 .. ] strain sample
  uint32_t fb_nsamp = 0, fb_stride = 1;
  uint32_t run_iters() const { return ad.enabled ? std::max(ad.effective_iterations, 1u) : iters; }
  // residual instrumentation
  bool track_residual = false;
  DBuf<float> res_sum, res_max;  // [ndc + nbc] each
  // parameters (simulation/mod.rs:607-690 defaults)
  float g[3] = {0.f, 0.f, -9.81f};
  float damping = 1.0f, td = 0.f, cd = 0.f, sd = 0.f, bd = 0.f;
  uint32_t iters = 2;
  bool self_collision = true;
  float relief = 0.2f, max_disp_ratio = 0.2f;
  bool enable_relief = true, exclude_neighbors = true, untangle_opt = true;
  uint32_t max_search = 256;
  // self-collision / E-E substep intervals (dispatch.rs:105-114, defaults mod.rs:624-625)
  uint32_t sc_interval = 1, ee_interval = 1;
  bool sc_due(uint32_t s, uint32_t substeps) const {
    return self_collision && (sc_interval <= 1 || s % sc_interval == 0 || s + 1 == substeps);
  }
  bool ee_due(uint32_t s, uint32_t substeps) const {
    return ee_interval == 0 ? false : (ee_interval == 1 ? true : (s % ee_interval == 0 || s + 1 == substeps));
  }
  bool coupled = false, auto_coupled = true, recovery = true;
  // settings the CUDA path stores for the config record only: the shader
  // workgroup size (pipeline_cache.rs:25-31), the post-collision relaxation
  // count of the coupled modes (mod.rs:1055-1058), the areal density
  // (mod.rs:1241-1245)
  uint32_t wg_size = 32, relax_iters = 1;
  float areal_density = 0.15f;
  float cloth_thickness = 0.005f;
  float last_max_disp = 0.f, last_eff_disp = 0.f;
  std::vector<float> prev_frame_pos;
  // graph cache
  cudaGraphExec_t gexec = nullptr;
  bool graph_dirty = true;
  float g_dt = -1.f;
  uint32_t g_sub = 0;
  bool g_coupled = false;
  uint32_t g_iters = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  bool async_pending = false;
  // per-pass profiling (GpuProfiler / take_profile, simulation/profile.rs:38-252):
  // when on, frames run eagerly with an event pair around every launch group
  bool profiling = false;
  struct Mark { const char* name; cudaEvent_t a, b; };
  std::vector<Mark> marks;
  std::vector<cudaEvent_t> ev_pool;
  size_t ev_used = 0;
  std::vector<std::string> prof_names;
  std::vector<double> prof_ms;
  std::vector<uint32_t> prof_cnt;

  cudaEvent_t ev_get() {
    if (ev_used == ev_pool.size()) {
      cudaEvent_t e;
      TC_CK(cudaEventCreate(&e));
      ev_pool.push_back(e);
    }
    return ev_pool[ev_used++];
  }
  template <class F>
  void timed(const char* name, F&& f) {
    if (!profiling) { f(); return; }
    cudaEvent_t a = ev_get(), b = ev_get();
    TC_CK(cudaEventRecord(a, st));
    f();
    TC_CK(cudaEventRecord(b, st));
    marks.push_back({name, a, b});
  }
  void collect_marks() {
    for (const auto& mk : marks) {
      float ms = 0.f;
      TC_CK(cudaEventElapsedTime(&ms, mk.a, mk.b));
      size_t k = 0;
      while (k < prof_names.size() && prof_names[k] != mk.name) ++k;
      if (k == prof_names.size()) { prof_names.push_back(mk.name); prof_ms.push_back(0.0); prof_cnt.push_back(0); }
      prof_ms[k] += ms;
      prof_cnt[k] += 1;
    }
    marks.clear();
    ev_used = 0;
  }

  ~Sim() {
    if (gexec) cudaGraphExecDestroy(gexec);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    for (auto e : ev_pool) cudaEventDestroy(e);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    if (st2) cudaStreamDestroy(st2);
    if (st) cudaStreamDestroy(st);
    if (h_err) cudaFreeHost(h_err);
    if (h_fb) cudaFreeHost(h_fb);
    if (h_pos3) cudaFreeHost(h_pos3);
    if (col_ev) {
      if (col_ev_used) cudaEventSynchronize(col_ev);
      cudaEventDestroy(col_ev);
    }
    if (h_col) cudaFreeHost(h_col);
  }

  void mark() { graph_dirty = true; }

  // the settings as the reference's SimConfig record (config_impl.rs:16-92)
  tcloth::SimSettings settings() const {
    tcloth::SimSettings c;
    for (int k = 0; k < 3; ++k) c.gravity[k] = g[k];
    c.damping = damping;
    c.tension_damping = td; c.compression_damping = cd; c.shear_damping = sd; c.bending_damping = bd;
    c.tension_stiffness = tcloth::compliance_to_stiffness(base_tc);
    c.compression_stiffness = tcloth::compliance_to_stiffness(base_cc);
    c.shear_stiffness = tcloth::compliance_to_stiffness(base_shc);
    c.bending_stiffness = base_bk;
    for (const auto& q : bend_h)
      if (q.pad0 <= 1.5f) { c.bending_stiffness = tcloth::compliance_to_stiffness(q.comp); break; }
    c.solver_iterations = iters;
    c.solver_mode = 0;
    c.workgroup_size = wg_size;
    c.enable_self_collision = self_collision;
    c.relief_factor = relief; c.max_displacement_ratio = max_disp_ratio;
    c.exclude_neighbors = exclude_neighbors; c.enable_normal_untangling = untangle_opt;
    c.self_collision_max_iterations = max_search;
    c.coupled_mode = 0; c.coupled_collider = coupled; c.post_relaxation_iters = relax_iters;
    c.substep_interval = sc_interval; c.ee_substep_interval = ee_interval;
    c.self_collision_algorithm = sc_algorithm; c.enable_pair_cache = pair_cache;
    c.pair_margin_mode = pair_margin_mode; c.pair_safety_margin = pair_safety;
    c.pair_horizon_scale = pair_hscale; c.pair_max_horizon = pair_max_h;
    c.pair_max_pairs = std::max(pair_max_vt, pair_max_ee);
    c.enable_pair_final_fallback = pair_final_fallback;
    c.enable_edge_collision = edge_collision; c.edge_margin_scale = edge_mscale; c.edge_margin_offset = edge_moff;
    c.sewing_stiffness = sew_stiffness; c.sewing_shrink_speed = sew_speed;
    c.enable_sewing_lock = sew_lock; c.sewing_lock_distance = sew_lock_dist;
    c.areal_density = areal_density;
    c.sewing_priority_enabled = pri.enabled; c.sewing_priority_threshold = pri.threshold;
    c.sewing_priority_merge_dist = pri.merge; c.sewing_priority_ramp_frames = pri.ramp_frames;
    c.sewing_priority_max_frames = pri.max_frames;
    c.enable_adaptive_substep = ad.enabled; c.min_substeps = ad.min_substeps; c.max_substeps = ad.max_substeps;
    c.auto_coupled_on_low_substeps = auto_coupled; c.auto_compensate_iterations = ad.auto_compensate;
    c.enable_strain_adaptive = ad.strain_adaptive; c.strain_tolerance = ad.strain_tolerance;
    return c;
  }

  // ---- upload of the vertex state from host arrays
  void upload_vertices(const float* pos, const float* vel, const float* w) {
    std::vector<float4> hx(n), hp(n), hv(n);
    for (uint32_t i = 0; i < n; ++i) {
      hx[i] = make_float4(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], w[i]);
      hp[i] = make_float4(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], m.thickness[i]);
      float vx = vel ? vel[3 * i] : 0.f, vy = vel ? vel[3 * i + 1] : 0.f, vz = vel ? vel[3 * i + 2] : 0.f;
      uint32_t layer = m.layer[i];
      float lf;
      std::memcpy(&lf, &layer, 4);
      hv[i] = make_float4(vx, vy, vz, lf);
    }
    x4.upload(hx, st);
    p4.upload(hp, st);
    v4.upload(hv, st);
    if (ws.ready) TC_CK(cudaMemsetAsync(ws.dprev.p, 0, size_t(n) * sizeof(float4), st));
    TC_CK(cudaStreamSynchronize(st));
  }

  void upload_dist() {
    std::vector<uint2> ids(nd);
    std::vector<float4> par(nd);
    for (uint32_t i = 0; i < nd; ++i) {
      ids[i] = make_uint2(dist_h[i].v0, dist_h[i].v1);
      par[i] = make_float4(dist_h[i].rest, dist_h[i].tc, dist_h[i].cc, dist_h[i].type == 1 ? 1.f : 0.f);
    }
    dist_ids.upload(ids, st);
    dist_par.upload(par, st);
    st_stale = true;  // the staged solver's copies follow on its next frame
    TC_CK(cudaStreamSynchronize(st));
  }
  void upload_bend() {
    std::vector<uint4> ids(nb);
    std::vector<float4> par(nb);
    for (uint32_t i = 0; i < nb; ++i) {
      const BendC& c = bend_h[i];
      ids[i] = make_uint4(c.v0, c.v1, c.v2, c.v3);
      par[i] = make_float4(c.rest, c.comp, c.pad0, c.pad1);
    }
    bend_ids.upload(ids, st);
    st_stale = true;
    bend_par.upload(par, st);
    TC_CK(cudaStreamSynchronize(st));
  }

  void init(const MeshInput& in, int dev) {
    device = dev;
    TC_CK(cudaSetDevice(device));
    TC_CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    TC_CK(cudaEventCreate(&ev0));
    TC_CK(cudaEventCreate(&ev1));
    m = build_mesh(in);
    cell_ref = m.cell;
    n = m.n;
    {  // vertices of one warp close in space for the collider pass (any order is exact)
      float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
      for (uint32_t i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) {
          lo[k] = std::fmin(lo[k], m.pos[3 * size_t(i) + k]);
          hi[k] = std::fmax(hi[k], m.pos[3 * size_t(i) + k]);
        }
      float inv[3];
      for (int k = 0; k < 3; ++k) inv[k] = hi[k] > lo[k] ? 1.f / (hi[k] - lo[k]) : 0.f;
      std::vector<std::pair<uint32_t, uint32_t>> code(n);
      for (uint32_t i = 0; i < n; ++i)
        code[i] = {tcloth::morton3(m.pos[3 * size_t(i)], m.pos[3 * size_t(i) + 1], m.pos[3 * size_t(i) + 2], lo, inv),
                   i};
      std::sort(code.begin(), code.end());
      std::vector<uint32_t> ord(n);
      for (uint32_t i = 0; i < n; ++i) ord[i] = code[i].second;
      col_order.upload(ord, st);
    }
    nd = uint32_t(m.dist.size());
    nb = uint32_t(m.bend.size());
    ne = uint32_t(m.edges.size() / 2);
    dist_h = m.dist;
    bend_h = m.bend;
    orig_edge_to_dist = m.orig_edge_to_dist;
    mult.assign(nd, 1.f);
    base_rest.resize(nd);
    for (uint32_t i = 0; i < nd; ++i) base_rest[i] = dist_h[i].rest;
    // base compliances (simulation/mod.rs:419-434)
    base_tc = base_cc = 1.f / 500.f;
    base_shc = 1.f / 250.f;
    bool got_t = false, got_s = false;
    for (const auto& c : dist_h) {
      if (c.type == 1) { if (!got_s) { base_shc = c.tc; got_s = true; } }
      else if (!got_t) { base_tc = c.tc; base_cc = c.cc; got_t = true; }
    }
    base_bk = in.bending_k > 0.f ? in.bending_k : 0.f;
    orig_w = m.inv_mass;
    init_w = m.inv_mass;
    init_pos = m.pos;
    prev_frame_pos = m.pos;
    {  // CFL characteristic length, mean rest length, diameter in hops (mod.rs:380-420)
      float min_d2 = 3.4028235e38f;
      for (const auto& c : dist_h) {
        const float* a = &m.pos[3 * size_t(c.v0)];
        const float* b = &m.pos[3 * size_t(c.v1)];
        const float dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
        const float d2 = (dx * dx + dy * dy) + dz * dz;
        if (d2 > 1e-8f && d2 < min_d2) min_d2 = d2;
      }
      const float min_edge = min_d2 < 3.4028235e38f ? std::sqrt(min_d2) : 0.02f;
      ad.mesh_char_len = std::fmax(std::fmin(0.005f * 2.0f, min_edge), 0.001f);
      float lo[3] = {3.4028235e38f, 3.4028235e38f, 3.4028235e38f}, hi[3] = {-3.4028235e38f, -3.4028235e38f, -3.4028235e38f};
      for (uint32_t i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) { lo[k] = std::fmin(lo[k], m.pos[3 * i + k]); hi[k] = std::fmax(hi[k], m.pos[3 * i + k]); }
      const float ex = hi[0] - lo[0], ey = hi[1] - lo[1], ez = hi[2] - lo[2];
      const float diag = n ? std::sqrt((ex * ex + ey * ey) + ez * ez) : 0.f;
      float tot = 0.f;
      for (const auto& c : dist_h) tot += c.rest;
      ad.mesh_avg_edge_len = nd ? std::fmax(tot / float(nd), 1e-4f) : 0.02f;
      ad.mesh_diameter_hops = std::min(std::max(uint32_t(std::ceil(diag / ad.mesh_avg_edge_len)), 10u), 60u);
    }
    upload_vertices(m.pos.data(), nullptr, m.inv_mass.data());
    local_len.upload(m.local_len, st);
    upload_dist();
    upload_bend();
    dlam.alloc(nd);
    blam.alloc(nb);
    adj_off.upload(m.adj_off, st);
    adj_idx.upload(m.adj_idx, st);
    th_off.upload(m.th_off, st);
    th_idx.upload(m.th_idx, st);
    th_rest.upload(m.th_rest, st);
    star_off.upload(m.star_off, st);
    star_idx.upload(reinterpret_cast<const uint2*>(m.star_idx.data()), m.star_idx.size() / 2, st);
    edges.upload(reinterpret_cast<const uint2*>(m.edges.data()), ne, st);
    edge_bits.upload(m.edge_bits, st);
    const size_t T = m.table;
    keys.alloc(n); counts.alloc(T + 1); cursor.alloc(T + 1); cs.alloc(T + 1); srt.alloc(n);
    ekeys.alloc(ne); ecs.alloc(T + 1); esrt.alloc(ne);
    ecounts.alloc(T + 1); ecursor.alloc(T + 1); etile_sum.alloc(64);
    TC_CK(cudaStreamCreateWithFlags(&st2, cudaStreamNonBlocking));
    TC_CK(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
    TC_CK(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
    nrm.alloc(n);
    acc.alloc(size_t(n) * A_N);
    vcell.alloc(n); mlen.alloc(n); sbox.alloc(3 * size_t(n)); ecell.alloc(ne); eamin.alloc(ne); eamax.alloc(ne);
    ccd_q.alloc(size_t(ne) * 8 + 1024); ccd_n.alloc(1 + tcloth::kEeSeg);
    ee_q.alloc(size_t(ne) * 24 + 1024);
    vs_p.alloc(n); vs_q.alloc(n); vs_c.alloc(n); tile_sum.alloc(64); es_c.alloc(ne); es_v.alloc(ne); es_lo.alloc(ne); es_hi.alloc(ne);
    TC_CK(cudaMemsetAsync(acc.p, 0, size_t(n) * A_N * sizeof(int32_t), st));
    TC_CK(cudaMemsetAsync(nrm.p, 0, size_t(n) * sizeof(float4), st));
    res_sum.alloc(m.dist_cnt.size() + m.bend_cnt.size() + 1);
    res_max.alloc(m.dist_cnt.size() + m.bend_cnt.size() + 1);
    prims.alloc(1); tris.alloc(1); bounds.alloc(1); cl16.alloc(1); cl256.alloc(1); cl4096.alloc(1);
    dist_offc.upload(m.dist_off, st); dist_cntc.upload(m.dist_cnt, st);
    bend_offc.upload(m.bend_off, st); bend_cntc.upload(m.bend_cnt, st);
    sew_h = m.sew;
    nsw = uint32_t(sew_h.size());
    sew_speed = std::fmax(in.sew_shrink_speed, 0.f);
    upload_sew();
    pair_defaults();
    bar.alloc(2);
    TC_CK(cudaMemsetAsync(bar.p, 0, 2 * sizeof(GridBar), st));
    TC_CK(cudaHostAlloc(&h_err, sizeof(int), cudaHostAllocDefault));
    *h_err = 0;
    {
      int coop = 0, nsm = 0, per_sm = 0;
      TC_CK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device));
      TC_CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
      TC_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_solver_persistent<false>, 256, 0));
      persist_blocks = coop && per_sm > 0 ? unsigned(nsm * std::min(per_sm, 4)) : 0u;
      persist_max_per_sm = unsigned(per_sm);
      int per_sm_bone = 0;
      TC_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_bone, k_solver_persistent<true>, 256, 0));
      persist_bone_per_sm = coop ? unsigned(per_sm_bone) : 0u;
      {  // co-resident clusters of the cluster solver (0 when clusters cannot launch)
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(kClusterCtas * 64);
        cfg.blockDim = dim3(256);
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = kClusterCtas;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int ncl = 0;
        if (cudaOccupancyMaxActiveClusters(&ncl, k_solver_cluster<false>, &cfg) != cudaSuccess) {
          cudaGetLastError();
          ncl = 0;
        }
        cl_max_active = ncl;
      }
      {  // staged cluster solver: slice capacity from the opt-in shared memory, co-resident clusters
        int optin = 0;
        TC_CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
        st_cap = std::min<uint32_t>(uint32_t(optin) / uint32_t(3u * sizeof(float4)), 65535u);  // slots fit 16 bits
        st_smem = size_t(st_cap) * 3u * sizeof(float4);
        int ncl = 0;
        if (st_cap > 0 &&
            cudaFuncSetAttribute(k_solver_staged<kStageCtas, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(st_smem)) == cudaSuccess &&
            cudaFuncSetAttribute(k_solver_staged<kStageCtas, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(st_smem)) == cudaSuccess) {
          cudaLaunchConfig_t cfg = {};
          cfg.gridDim = dim3(kStageCtas * 16);
          cfg.blockDim = dim3(kStageThreads);
          cfg.dynamicSmemBytes = st_smem;
          cudaLaunchAttribute attr[1];
          attr[0].id = cudaLaunchAttributeClusterDimension;
          attr[0].val.clusterDim.x = kStageCtas;
          attr[0].val.clusterDim.y = 1;
          attr[0].val.clusterDim.z = 1;
          cfg.attrs = attr;
          cfg.numAttrs = 1;
          if (cudaOccupancyMaxActiveClusters(&ncl, k_solver_staged<kStageCtas, false>, &cfg) != cudaSuccess) ncl = 0;
        }
        cudaGetLastError();
        st_max_active = ncl;
      }
      num_sms = unsigned(nsm);
      if (!persist_blocks) persistent = false;
    }
    pin_v.alloc(1); pin_t.alloc(1);
    TC_CK(cudaStreamSynchronize(st));
  }

  // ---- colliders
  void upload_prims() {
    prims.upload(prims_h, st);
    TC_CK(cudaStreamSynchronize(st));
    mark();
  }
  uint32_t graph_ntris = UINT32_MAX;
  // The triangles go to the device as floats and are packed, Morton-sorted and
  // bounded there (collider_prep.cuh, simulation/mod.rs:2613-2670), in the
  // stream ahead of the next frame; the host only copies them into pinned
  // memory, after the previous upload's copy out of it has finished.
  void set_mesh(const float* t9, uint32_t T, float fric, float thick, float rest, bool single, const float* attr) {
    tris_h.clear();
    tris_h_valid = T == 0;
    ntris = T;
    if (T == 0) { mark(); graph_ntris = 0; ce_stale = true; return; }
    if (T > 0x7FFFFFFFu) throw TcError(TC_ERR_INVALID, "too many collider triangles");  // the device sort counts in int
    const size_t nf = size_t(T) * (attr ? 13 : 9);
    if (!col_ev) TC_CK(cudaEventCreateWithFlags(&col_ev, cudaEventDisableTiming));
    if (col_ev_used) TC_CK(cudaEventSynchronize(col_ev));
    if (h_col_cap < nf) {
      if (h_col) TC_CK(cudaFreeHost(h_col));
      h_col = nullptr;
      h_col_cap = 0;
      TC_CK(cudaMallocHost(&h_col, nf * sizeof(float)));
      h_col_cap = nf;
    }
    std::memcpy(h_col, t9, size_t(T) * 9 * sizeof(float));
    if (attr) std::memcpy(h_col + size_t(T) * 9, attr, size_t(T) * 4 * sizeof(float));
    col_in.alloc(nf);
    TC_CK(cudaMemcpyAsync(col_in.p, h_col, nf * sizeof(float), cudaMemcpyHostToDevice, st));
    TC_CK(cudaEventRecord(col_ev, st));
    col_ev_used = true;
    const uint32_t n16 = (T + 15) / 16, n256 = (T + 255) / 256, n4096 = (T + 4095) / 4096;
    const void* before[5] = {tris.p, bounds.p, cl16.p, cl256.p, cl4096.p};
    col_raw.alloc(T);
    col_box.alloc(6);
    col_code.alloc(T); col_code2.alloc(T); col_idx.alloc(T); col_idx2.alloc(T);
    tris.alloc(T); bounds.alloc(T); cl16.alloc(n16); cl256.alloc(n256); cl4096.alloc(n4096);
    k_col_pack<<<grid(T, 256), 256, 0, st>>>(T, col_in.p, attr ? col_in.p + size_t(T) * 9 : nullptr, fric, thick,
                                             rest, single ? 1u : 0u, col_raw.p);
    k_col_bounds<<<1, 1024, 0, st>>>(T, col_raw.p, col_box.p);
    k_col_codes<<<grid(T, 256), 256, 0, st>>>(T, col_raw.p, col_box.p, col_code.p, col_idx.p);
    // stable LSD radix sort of the 30-bit codes: equal codes keep index order
    size_t tmp_bytes = 0;
    TC_CK(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, col_code.p, col_code2.p, col_idx.p, col_idx2.p, int(T),
                                          0, 30, st));
    col_tmp.alloc(std::max<size_t>(tmp_bytes, 1));
    TC_CK(cub::DeviceRadixSort::SortPairs(col_tmp.p, tmp_bytes, col_code.p, col_code2.p, col_idx.p, col_idx2.p,
                                          int(T), 0, 30, st));
    k_col_gather<<<grid(T, 256), 256, 0, st>>>(T, col_raw.p, col_idx2.p, tris.p, bounds.p);
    k_col_groups<<<n16, 256, 0, st>>>(T, 16, bounds.p, cl16.p);
    k_col_groups<<<n256, 256, 0, st>>>(T, 256, bounds.p, cl256.p);
    k_col_groups<<<n4096, 256, 0, st>>>(T, 4096, bounds.p, cl4096.p);
    TC_CK(cudaGetLastError());
    // the recorded frame only holds pointers and the triangle count: new
    // contents of the same size replay without re-recording
    const void* after[5] = {tris.p, bounds.p, cl16.p, cl256.p, cl4096.p};
    if (T != graph_ntris || std::memcmp(before, after, sizeof before) != 0) mark();
    graph_ntris = T;
    ce_stale = true;
  }
  // the sorted triangles on the host, for the host-side collider-edge build
  const std::vector<MeshTri>& host_tris() {
    if (!tris_h_valid) {
      tris_h.resize(ntris);
      if (ntris) TC_CK(cudaMemcpyAsync(tris_h.data(), tris.p, size_t(ntris) * sizeof(MeshTri), cudaMemcpyDeviceToHost, st));
      TC_CK(cudaStreamSynchronize(st));
      tris_h_valid = true;
    }
    return tris_h;
  }

  // ---- pins
  void upload_pins() {
    cl_stale = true;
    st_stale = true;
    std::vector<uint32_t> v;
    std::vector<float4> t;
    for (const auto& kv : pins) {
      v.push_back(kv.first);
      t.push_back(make_float4(kv.second.target[0], kv.second.target[1], kv.second.target[2], kv.second.weight));
    }
    pin_v.upload(v, st);
    pin_t.upload(t, st);
    TC_CK(cudaStreamSynchronize(st));
    mark();
  }
  void write_inv_mass(uint32_t v, float w) {
    TC_CK(cudaMemcpyAsync(reinterpret_cast<char*>(x4.p) + size_t(v) * sizeof(float4) + 12, &w, 4,
                          cudaMemcpyHostToDevice, st));
    TC_CK(cudaStreamSynchronize(st));
  }
  static float clamp_w(float w) { return std::isfinite(w) ? std::fmin(std::fmax(w, 0.f), 1.f) : 0.f; }

  // ---- compliance
  static float scale_compliance(float base, float mlt) {
    if (base >= 1e9f) return base;
    if (base <= 0.f) return 0.f;
    return base / mlt;
  }
  void apply_distance_compliances() {
    for (uint32_t i = 0; i < nd; ++i) {
      float ml = std::fmax(mult[i], 1e-3f);
      if (dist_h[i].type == 1) dist_h[i].tc = dist_h[i].cc = scale_compliance(base_shc, ml);
      else { dist_h[i].tc = scale_compliance(base_tc, ml); dist_h[i].cc = scale_compliance(base_cc, ml); }
    }
    upload_dist();
    mark();
  }

  SCArgs sc_args() {
    SCArgs a;
    a.n = n; a.ne = ne; a.table = m.table; a.cell = m.cell;
    a.relief = relief; a.enable_relief = enable_relief; a.max_disp_ratio = max_disp_ratio;
    a.exclude_neighbors = exclude_neighbors; a.untangle = (untangle_opt && m.multi_layer) ? 1 : 0;
    a.max_search = max_search;
    a.x4 = x4.p; a.p4 = p4.p; a.v4 = v4.p; a.local_len = local_len.p;
    a.adj_off = adj_off.p; a.adj_idx = adj_idx.p; a.th_off = th_off.p; a.th_idx = th_idx.p; a.th_rest = th_rest.p;
    a.star_off = star_off.p; a.star_idx = star_idx.p; a.edges = edges.p; a.edge_bits = edge_bits.p;
    a.cs = cs.p; a.srt = srt.p; a.ecs = ecs.p; a.esrt = esrt.p; a.nrm = nrm.p; a.acc = acc.p;
    a.sbox = sbox.p;
    a.vcell = vcell.p; a.mlen = mlen.p; a.ecell = ecell.p; a.eamin = eamin.p; a.eamax = eamax.p;
    a.ccd_q = ccd_q.p; a.ccd_n = ccd_n.p; a.ccd_cap = uint32_t(ccd_q.n);
    a.ee_q = ee_q.p; a.ee_n = ccd_n.p ? ccd_n.p + 1 : nullptr;
    const size_t ee_entries = ee_list_entries ? std::min(ee_list_entries, ee_q.n) : ee_q.n;
    a.ee_cap = ee_list ? uint32_t(std::min<size_t>(ee_entries, 0xffffffffu)) : 0u;
    a.vs_p = vs_p.p; a.vs_q = vs_q.p; a.vs_c = vs_c.p; a.es_c = es_c.p; a.es_v = es_v.p; a.es_lo = es_lo.p; a.es_hi = es_hi.p;
    a.rec_vt = rec_pairs ? rec_vt.p : nullptr;
    a.rec_ee = rec_pairs ? rec_ee.p : nullptr;
    a.rec_n = rec_pairs ? rec_n.p : nullptr;
    a.rec_vt_cap = rec_pairs ? rec_vt_cap : 0u;
    a.rec_ee_cap = rec_pairs ? rec_ee_cap : 0u;
    return a;
  }
  // threads per block of the per-colour constraint launches (autotuned;
  // results do not depend on it)
  uint32_t col_block = 256;
  // the collider pass's vertex order: Morton order of the initial positions
  DBuf<uint32_t> col_order;
  float cell_ref = 0.f;  // the reference formula's hash cell (tc_set_hash_cell_size can override m.cell)
  // E-E kernel: false = one warp per edge (k_ee), true = one lane per edge
  // with per-cell candidate lists in shared memory (k_ee_grouped); same pairs
  // and results
  bool ee_grouped = false;
  // k_ee lists its counted pairs for k_ee_pairs (one lane per pair) instead
  // of working them in the edge's warp; same pairs and results.  The list
  // holds ee_list_entries pairs (0: all of ee_q, 24 per edge + 1024).
  bool ee_list = true;
  size_t ee_list_entries = 0;
  // narrow-phase pair record of the latest self-collision pass (off by default)
  bool rec_pairs = false;
  DBuf<uint4> rec_vt;
  DBuf<uint2> rec_ee;
  DBuf<uint32_t> rec_n;
  uint32_t rec_vt_cap = 0, rec_ee_cap = 0;

  static unsigned grid(uint32_t cnt, unsigned b) { return (cnt + b - 1) / b; }

  // Spatial hash of the vertices (which = 0) or edge midpoints (which = 1) on
  // stream `ss`; the edge build has its own counting scratch so that it can
  // run beside the vertex side.
  void encode_hash(int which, cudaStream_t ss) {
    const uint32_t cnt = which == 0 ? n : ne;
    const uint32_t T = m.table;
    uint32_t* k = which == 0 ? keys.p : ekeys.p;
    uint32_t* start = which == 0 ? cs.p : ecs.p;
    uint32_t* sorted = which == 0 ? srt.p : esrt.p;
    uint32_t* cnts = which == 0 ? counts.p : ecounts.p;
    uint32_t* curs = which == 0 ? cursor.p : ecursor.p;
    uint32_t* tsum = which == 0 ? tile_sum.p : etile_sum.p;
    TC_CK(cudaMemsetAsync(cnts, 0, (T + 1) * sizeof(uint32_t), ss));
    TC_CK(cudaMemsetAsync(curs, 0, (T + 1) * sizeof(uint32_t), ss));
    timed(which == 0 ? "hash_vertices" : "hash_edges", [&] {
      if (cnt)
        k_hash_count<<<grid(cnt, 256), 256, 0, ss>>>(cnt, which, x4.p, p4.p, edges.p, m.cell, T, k, cnts,
                                                      which == 0 ? vcell.p : ecell.p, mlen.p, eamin.p, eamax.p);
      const uint32_t ntiles = (T + 1023) / 1024;
      k_scan_blocks<<<ntiles, 1024, 0, ss>>>(T, cnts, start, tsum);
      k_scan_finish<<<ntiles, 1024, 0, ss>>>(T, ntiles, tsum, start);
      if (cnt) k_hash_scatter<<<grid(cnt, 256), 256, 0, ss>>>(cnt, k, start, curs, sorted);
      k_hash_sort_buckets_warp<<<grid(T, 8), 256, 0, ss>>>(T, start, sorted);
      if (cnt && which == 0)
        k_gather_vertices<<<grid(cnt, 256), 256, 0, ss>>>(cnt, sorted, x4.p, p4.p, v4.p, local_len.p, mlen.p, vcell.p,
                                                           vs_p.p, vs_c.p, vs_q.p);
      if (cnt && which == 1)
        k_gather_edges<<<grid(cnt, 256), 256, 0, ss>>>(cnt, sorted, edges.p, ecell.p, eamin.p, eamax.p, es_c.p, es_v.p,
                                                        es_lo.p, es_hi.p);
    });
  }
  void encode_hash(int which) { encode_hash(which, st); }
  void encode_ee(const SCArgs& a, cudaStream_t ss) {
    timed("sc_solve_ee", [&] {
      TC_CK(cudaMemsetAsync(ccd_n.p, 0, (1 + tcloth::kEeSeg) * sizeof(uint32_t), ss));
      if (ee_grouped) {
        k_ee_grouped<<<grid(ne, 32 * tcloth::kEeWarps), 32 * tcloth::kEeWarps, 0, ss>>>(a);
      } else {
        if (a.ee_cap) k_ee<true><<<grid(ne, 8), 256, 0, ss>>>(a);
        else k_ee<false><<<grid(ne, 8), 256, 0, ss>>>(a);
        if (a.ee_cap) k_ee_pairs<<<tcloth::kEeSeg * tcloth::kEePairBlocks, 256, 0, ss>>>(a);
      }
    });
    timed("sc_solve_ee_ccd", [&] { k_ee_ccd<<<148 * 8, 256, 0, ss>>>(a); });
  }

  // The edge side (edge hash, E-E, deferred CCD) reads positions, normals
  // and its own hash, and writes the contact accumulators only through
  // atomic add / max / min, which commute with the vertex side's; so outside
  // profiling it runs on a second stream concurrently with the vertex side
  // (vertex hash, V-V / V-T, untangle), joined before apply.
  PairArgs pair_args(float dt) {
    PairArgs p;
    p.safety = pair_safety; p.dt_frame = dt; p.hscale = pair_hscale; p.max_h = pair_max_h;
    p.margin_mode = pair_margin_mode; p.quota_vt = pair_qvt; p.quota_ee = pair_qee;
    p.island = island_d.p; p.hz = pair_hz.p; p.vt = pair_vt.p; p.ee = pair_ee.p; p.counters = pair_cnt.p;
    return p;
  }
  // Pair-cache pass (dispatch.rs:1556-1645): the vertex hash and the broad
  // phase only at the first substep of the frame, the narrow phase over the
  // cached slots at every substep.  With the final fallback on (default) the
  // last substep runs the direct pass on a fresh hash instead.
  void encode_pair_self_collision(bool run_ee, bool rebuild, float dt) {
    SCArgs a = sc_args();
    const PairArgs p = pair_args(dt);
    if (a.untangle) timed("sc_normals", [&] { k_normals<<<grid(n, 256), 256, 0, st>>>(n, x4.p, star_off.p, star_idx.p, nrm.p); });
    if (rebuild) {
      encode_hash(0);
      TC_CK(cudaMemsetAsync(pair_cnt.p, 0, 4 * sizeof(uint32_t), st));
      timed("pair_collect", [&] {
        k_pair_horizon<<<grid(n, 256), 256, 0, st>>>(n, v4.p, p);
        if (profiling) {
          k_pair_collect<0><<<grid(n, 128), 128, 0, st>>>(a, p);
          k_pair_collect<1><<<grid(n, 128), 128, 0, st>>>(a, p);
        } else {  // the two lists are independent: the edge-edge scan runs beside
          TC_CK(cudaEventRecord(ev_fork, st));
          TC_CK(cudaStreamWaitEvent(st2, ev_fork, 0));
          k_pair_collect<1><<<grid(n, 128), 128, 0, st2>>>(a, p);
          TC_CK(cudaEventRecord(ev_join, st2));
          k_pair_collect<0><<<grid(n, 128), 128, 0, st>>>(a, p);
          TC_CK(cudaStreamWaitEvent(st, ev_join, 0));
        }
      });
    }
    const uint32_t vts = n * pair_qvt, ees = n * pair_qee;
    timed("pair_vt", [&] { k_pair_vt<<<grid(vts, 128), 128, 0, st>>>(a, p, vts); });
    if (run_ee) timed("pair_ee", [&] { k_pair_ee<<<grid(ees, 128), 128, 0, st>>>(a, p, ees); });
    if (a.untangle) timed("sc_untangle", [&] { k_untangle<<<grid(n, 128), 128, 0, st>>>(a); });
    timed("sc_apply", [&] {
      k_apply<<<grid(n, 256), 256, 0, st>>>(n, x4.p, p4.p, local_len.p, acc.p, relief, enable_relief ? 1 : 0,
                                             max_disp_ratio);
    });
  }

  void encode_self_collision(bool run_ee, uint32_t s, uint32_t substeps, float dt) {
    if (rec_pairs) TC_CK(cudaMemsetAsync(rec_n.p, 0, 2 * sizeof(uint32_t), st));
    const bool force_direct = pair_cache && pair_final_fallback && s + 1 == substeps;
    if (pair_cache && !force_direct) {
      encode_pair_self_collision(run_ee, s == 0, dt);
      return;
    }
    SCArgs a = sc_args();
    if (a.untangle) timed("sc_normals", [&] { k_normals<<<grid(n, 256), 256, 0, st>>>(n, x4.p, star_off.p, star_idx.p, nrm.p); });
    const bool edges_on = run_ee && ne > 0;
    const bool fork = edges_on && !profiling;
    if (fork) {
      TC_CK(cudaEventRecord(ev_fork, st));
      TC_CK(cudaStreamWaitEvent(st2, ev_fork, 0));
      encode_hash(1, st2);
      encode_ee(a, st2);
      TC_CK(cudaEventRecord(ev_join, st2));
    }
    encode_hash(0);
    timed("sc_star_box", [&] { k_star_box<<<grid(n, 256), 256, 0, st>>>(n, star_off.p, star_idx.p, x4.p, p4.p, sbox.p); });
    if (edges_on && !fork) encode_hash(1);
    timed("sc_solve", [&] { k_sc_solve<<<grid(n, 8), 256, 0, st>>>(a); });
    if (a.untangle) timed("sc_untangle", [&] { k_untangle<<<grid(n, 128), 128, 0, st>>>(a); });
    if (fork) TC_CK(cudaStreamWaitEvent(st, ev_join, 0));
    if (edges_on && !fork) encode_ee(a, st);
    timed("sc_apply", [&] {
      k_apply<<<grid(n, 256), 256, 0, st>>>(n, x4.p, p4.p, local_len.p, acc.p, relief, enable_relief ? 1 : 0,
                                             max_disp_ratio);
    });
  }

  ColliderArgs collider_args() {
    ColliderArgs c;
    c.prims = prims.p; c.nprims = uint32_t(prims_h.size());
    c.tris = tris.p; c.bounds = bounds.p; c.cl16 = cl16.p; c.cl256 = cl256.p; c.cl4096 = cl4096.p; c.ntris = ntris;
    c.recovery = recovery;
    c.vinst = inst_prims_h.empty() ? nullptr : vinst.p;
    c.inst_prims = inst_prims_h.empty() ? nullptr : inst_prims.p;
    c.bone = BoneSdfArgs{bone.info.p, bone.xf.p, bone.atlas.p,
                         bone.enabled ? uint32_t(std::min(bone.info_h.size(), bone.xf_h.size())) : 0u,
                         bone.w, bone.h, bone.d};
    return c;
  }
  bool has_colliders() const { return !prims_h.empty() || ntris != 0 || bone.enabled; }

  // ---- bone SDF
  // update_bone_transforms (simulation/mod.rs:1865-1935): store the
  // transforms and the world bounding sphere of each bone in the infos' .w
  void set_bone_transforms(const float* world, const float* inv, uint32_t nbt) {
    bone.xf_h.resize(nbt);
    for (uint32_t b = 0; b < nbt; ++b) {
      std::memcpy(bone.xf_h[b].m, world + 16 * size_t(b), 64);
      std::memcpy(bone.xf_h[b].inv, inv + 16 * size_t(b), 64);
    }
    const uint32_t nn = uint32_t(std::min(bone.info_h.size(), bone.xf_h.size()));
    for (uint32_t b = 0; b < nn; ++b) {
      BoneInfo& I = bone.info_h[b];
      const float* m = bone.xf_h[b].m;
      const float c[3] = {(I.aabb_min.x + I.aabb_max.x) * 0.5f, (I.aabb_min.y + I.aabb_max.y) * 0.5f,
                          (I.aabb_min.z + I.aabb_max.z) * 0.5f};
      const float ex = I.aabb_max.x - I.aabb_min.x, ey = I.aabb_max.y - I.aabb_min.y, ez = I.aabb_max.z - I.aabb_min.z;
      const float rl = 0.5f * std::sqrt((ex * ex + ey * ey) + ez * ez);
      float cw[3];
      for (int j = 0; j < 3; ++j) cw[j] = ((m[0 + j] * c[0] + m[4 + j] * c[1]) + m[8 + j] * c[2]) + m[12 + j];
      const float sx = std::sqrt((m[0] * m[0] + m[1] * m[1]) + m[2] * m[2]);
      const float sy = std::sqrt((m[4] * m[4] + m[5] * m[5]) + m[6] * m[6]);
      const float sz = std::sqrt((m[8] * m[8] + m[9] * m[9]) + m[10] * m[10]);
      const float rw = rl * std::fmax(std::fmax(sx, sy), sz) + 0.1f;
      I.aabb_min.w = cw[0];
      I.aabb_max.w = cw[1];
      I.uvw_scale.w = cw[2];
      I.uvw_offset.w = rw;
    }
    const void* before[2] = {bone.info.p, bone.xf.p};
    if (!bone.info_h.empty()) bone.info.upload(bone.info_h, st);
    if (!bone.xf_h.empty()) bone.xf.upload(bone.xf_h, st);
    TC_CK(cudaStreamSynchronize(st));
    const void* after[2] = {bone.info.p, bone.xf.p};
    if (std::memcmp(before, after, sizeof before) != 0) mark();
  }
  void set_identity_transforms(uint32_t nbt) {
    std::vector<float> id(16 * size_t(nbt), 0.f);
    for (uint32_t b = 0; b < nbt; ++b)
      for (int k = 0; k < 4; ++k) id[16 * size_t(b) + 5 * k] = 1.f;
    set_bone_transforms(id.data(), id.data(), nbt);
  }
  void clear_bone() {
    bone.info_h.clear();
    bone.xf_h.clear();
    bone.enabled = false;
    bone.dyn = bone.dyn_on = false;
    mark();
  }
  // dispatch_dynamic_bone_sdf_update (simulation/mod.rs:2320-2464), before a frame
  void dynamic_bone_update() {
    BoneSdfState& B = bone;
    if (!B.dyn || !B.dyn_on) return;
    B.counter += 1;
    if ((B.counter - 1) % B.interval != 0) return;
    if (B.xf_h.size() < B.nb) return;
    std::vector<uint32_t> list;
    if (!B.baked || !B.dirty_set) {
      list.resize(B.nb);
      for (uint32_t b = 0; b < B.nb; ++b) list[b] = b;
    } else {
      if (B.dirty.empty()) return;  // no pose change: nothing to do
      for (uint32_t b : B.dirty)
        if (b < B.nb) list.push_back(b);
    }
    std::vector<float> skin(16 * size_t(B.nb)), inv(16 * size_t(B.nb));
    for (uint32_t b = 0; b < B.nb; ++b) {
      float wr[4][4], bb[4][4], sr[4][4];
      for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) { wr[i][j] = B.xf_h[b].m[j * 4 + i]; bb[i][j] = B.bind_inv[16 * size_t(b) + i * 4 + j]; }
      for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j)
          sr[i][j] = ((wr[i][0] * bb[0][j] + wr[i][1] * bb[1][j]) + wr[i][2] * bb[2][j]) + wr[i][3] * bb[3][j];
      for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) skin[16 * size_t(b) + i * 4 + j] = sr[j][i];
      std::memcpy(&inv[16 * size_t(b)], B.xf_h[b].inv, 64);
    }
    B.skin_m.upload(skin, st);
    B.inv_m.upload(inv, st);
    timed("bone_skin", [&] {
      k_bone_skin<<<(B.nv + 127) / 128, 128, 0, st>>>(B.nv, B.rest.p, B.bidx.p, B.bw.p, B.skin_m.p, B.skinned.p);
    });
    timed("bone_prep", [&] {
      if (B.bake.nt)
        k_bone_prep<<<(B.bake.nt + 127) / 128, 128, 0, st>>>(B.bake.nt, B.skinned.p, B.inv_m.p, B.tsrc.p, B.tsrcw.p,
                                                              B.bake.tris.p);
    });
    std::vector<BakeParams> ps;
    for (uint32_t b : list) ps.push_back(B.params_h[b]);
    timed("bone_bake", [&] { B.bake.bake(ps, list, B.atlas.p, st); });
    TC_CK(cudaGetLastError());
    B.baked = true;
  }

  void encode_residual(const SubstepParams& sp);

  SolverArgs solver_args(const SubstepParams& sp, uint32_t nsub, bool use_coupled, bool with_update) {
    SolverArgs a;
    a.n = n; a.nsub = nsub; a.iters = run_iters(); a.npins = uint32_t(pins.size());
    a.ndc = uint32_t(m.dist_cnt.size()); a.nbc = uint32_t(m.bend_cnt.size());
    a.hascol = has_colliders();
    a.coupled = use_coupled;
    a.ddamp = td != 0.f || cd != 0.f || sd != 0.f;
    a.bdamp = bd != 0.f;
    a.with_update = with_update;
    a.sp = sp;
    a.x4 = x4.p; a.p4 = p4.p; a.v4 = v4.p;
    a.dist_ids = dist_ids.p; a.dist_par = dist_par.p; a.dlam = dlam.p; a.nd = nd;
    a.bend_ids = bend_ids.p; a.bend_par = bend_par.p; a.blam = blam.p; a.nb = nb;
    a.dist_off = dist_offc.p; a.dist_cnt = dist_cntc.p; a.bend_off = bend_offc.p; a.bend_cnt = bend_cntc.p;
    a.pin_v = pin_v.p; a.pin_t = pin_t.p;
    a.ca = collider_args();
    a.bar = bar.p;
    a.expected = 0;  // the launch fills in its grid size
    a.spin_limit = spin_limit;
    a.skip_predict = false;
    a.ppred = nullptr;
    a.dprev = nullptr;
    a.iters_extra = 0;
    a.res_thresh = 0.f;
    a.res_ratio = 0.f;
    a.res_floor = 0.f;
    a.res_pred = nullptr;
    a.nsw = nsw;
    a.nsc = uint32_t(m.sew_cnt.size());
    a.sew_ids = sew_ids.p; a.sew_rest = sew_rest.p; a.slam = slam.p;
    a.sew_off = sew_offc.p; a.sew_cnt = sew_cntc.p;
    a.sew_speed = sew_speed;
    a.sw = sew_params();
    a.res_part = nullptr;
    a.res_out = nullptr;
    a.fallbacks = nullptr;
    return a;
  }
  bool can_cluster() const {
    return !inst_vert_off.empty() && cl_max_active > 0 && !self_collision && nsw == 0 && !edge_collision;
  }
  // bins: contiguous runs of instances, balanced by vertex count; the
  // constraint permutations are sorted by (bin, colour, original index)
  void build_cluster_tables() {
    const uint32_t ninst = uint32_t(inst_vert_off.size() - 1);
    const uint32_t B = std::max(1u, std::min(ninst, uint32_t(cl_max_active)));
    const uint64_t target = (uint64_t(n) + B - 1) / B;
    std::vector<uint32_t> bin_of_inst(ninst);
    for (uint32_t k = 0; k < ninst; ++k) {
      const uint64_t mid = uint64_t(inst_vert_off[k]) + (inst_vert_off[k + 1] - inst_vert_off[k]) / 2;
      bin_of_inst[k] = uint32_t(std::min<uint64_t>(B - 1, mid / std::max<uint64_t>(target, 1)));
    }
    std::vector<uint2> vr(B, make_uint2(0, 0));
    std::vector<char> seen(B, 0);
    for (uint32_t k = 0; k < ninst; ++k) {
      const uint32_t b = bin_of_inst[k];
      if (!seen[b]) { vr[b] = make_uint2(inst_vert_off[k], inst_vert_off[k + 1]); seen[b] = 1; }
      else vr[b].y = inst_vert_off[k + 1];
    }
    for (uint32_t b = 0; b < B; ++b)  // empty bins: an empty range
      if (!seen[b]) vr[b] = make_uint2(b ? vr[b - 1].y : 0u, b ? vr[b - 1].y : 0u);
    std::vector<uint32_t> bin_of_v(n);
    for (uint32_t k = 0; k < ninst; ++k)
      for (uint32_t v = inst_vert_off[k]; v < inst_vert_off[k + 1]; ++v) bin_of_v[v] = bin_of_inst[k];
    std::vector<uint32_t> pv;
    for (const auto& kv : pins) pv.push_back(kv.first);
    std::vector<uint2> pr(B);
    for (uint32_t b = 0; b < B; ++b) {
      const uint32_t lo = uint32_t(std::lower_bound(pv.begin(), pv.end(), vr[b].x) - pv.begin());
      const uint32_t hi = uint32_t(std::lower_bound(pv.begin(), pv.end(), vr[b].y) - pv.begin());
      pr[b] = make_uint2(lo, hi - lo);
    }
    auto perm_of = [&](const std::vector<uint32_t>& off, const std::vector<uint32_t>& cnt, auto vert_of,
                       std::vector<uint32_t>& perm, std::vector<uint2>& tab) {
      const uint32_t nc = uint32_t(off.size());
      std::vector<std::vector<uint32_t>> bucket(size_t(B) * std::max(nc, 1u));
      for (uint32_t c = 0; c < nc; ++c)
        for (uint32_t k = off[c]; k < off[c] + cnt[c]; ++k) bucket[size_t(bin_of_v[vert_of(k)]) * nc + c].push_back(k);
      perm.clear();
      tab.assign(size_t(B) * nc, make_uint2(0, 0));
      for (size_t q = 0; q < size_t(B) * nc; ++q) {
        tab[q] = make_uint2(uint32_t(perm.size()), uint32_t(bucket[q].size()));
        perm.insert(perm.end(), bucket[q].begin(), bucket[q].end());
      }
    };
    std::vector<uint32_t> dperm, bperm;
    std::vector<uint2> dtab, btab;
    perm_of(m.dist_off, m.dist_cnt, [&](uint32_t k) { return dist_h[k].v0; }, dperm, dtab);
    perm_of(m.bend_off, m.bend_cnt, [&](uint32_t k) { return bend_h[k].v0; }, bperm, btab);
    cl_vrange.upload(vr, st);
    cl_pins.upload(pr, st);
    cl_dist.upload(dtab, st);
    cl_bend.upload(btab, st);
    cl_dperm.upload(dperm, st);
    cl_bperm.upload(bperm, st);
    TC_CK(cudaStreamSynchronize(st));
    cl_bins = B;
    cl_stale = false;
  }
  void launch_cluster(const SolverArgs& a) {
    const ClusterTables t{cl_vrange.p, cl_pins.p, cl_dist.p, cl_bend.p, cl_dperm.p, cl_bperm.p};
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cl_bins * kClusterCtas);
    cfg.blockDim = dim3(256);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = kClusterCtas;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (a.ca.bone.nbones > 0) TC_CK(cudaLaunchKernelEx(&cfg, k_solver_cluster<true>, a, t));
    else TC_CK(cudaLaunchKernelEx(&cfg, k_solver_cluster<false>, a, t));
  }
  // the staged solver applies where the cluster solver does and every
  // instance fits the shared memory of one cluster
  bool can_stage() const {
    if (!can_cluster() || st_max_active <= 0 || st_cap == 0) return false;
    for (size_t k = 0; k + 1 < inst_vert_off.size(); ++k)
      if (inst_vert_off[k + 1] - inst_vert_off[k] > kStageCtas * st_cap) return false;
    return true;
  }
  // bins: contiguous runs of instances balanced by vertex count (at least
  // as many as fit on the device at once, more while a bin is over a
  // cluster's capacity); each bin's range is cut into kStageCtas slices and
  // each (bin, colour) constraint range is ordered by the slice that owns
  // the constraint's first vertex
  void build_stage_tables() {
    const uint32_t K = kStageCtas;
    const uint32_t ninst = uint32_t(inst_vert_off.size() - 1);
    const uint64_t bin_cap = uint64_t(K) * st_cap;
    std::vector<uint32_t> bin_of_inst(ninst);
    uint32_t B = std::max(1u, std::min(ninst, uint32_t(st_max_active)));
    for (;; ++B) {
      const uint64_t target = (uint64_t(n) + B - 1) / B;
      std::vector<uint64_t> size(B, 0);
      for (uint32_t k = 0; k < ninst; ++k) {
        const uint64_t mid = uint64_t(inst_vert_off[k]) + (inst_vert_off[k + 1] - inst_vert_off[k]) / 2;
        bin_of_inst[k] = uint32_t(std::min<uint64_t>(B - 1, mid / std::max<uint64_t>(target, 1)));
        size[bin_of_inst[k]] += inst_vert_off[k + 1] - inst_vert_off[k];
      }
      if (*std::max_element(size.begin(), size.end()) <= bin_cap || B >= ninst) break;
    }
    std::vector<uint2> vr(B, make_uint2(0, 0));
    std::vector<char> seen(B, 0);
    for (uint32_t k = 0; k < ninst; ++k) {
      const uint32_t b = bin_of_inst[k];
      if (!seen[b]) { vr[b] = make_uint2(inst_vert_off[k], inst_vert_off[k + 1]); seen[b] = 1; }
      else vr[b].y = inst_vert_off[k + 1];
    }
    for (uint32_t b = 0; b < B; ++b)
      if (!seen[b]) vr[b] = make_uint2(b ? vr[b - 1].y : 0u, b ? vr[b - 1].y : 0u);
    std::vector<uint32_t> bin_of_v(n), owner(n);
    for (uint32_t b = 0; b < B; ++b) {
      const uint32_t nv = vr[b].y - vr[b].x, chunk = nv ? (nv + K - 1) / K : 1u;
      for (uint32_t v = vr[b].x; v < vr[b].y; ++v) {
        bin_of_v[v] = b;
        owner[v] = (v - vr[b].x) / chunk;
      }
    }
    std::vector<uint32_t> pv;
    std::vector<uint2> pr(size_t(B) * K, make_uint2(0, 0));
    for (const auto& kv : pins) pv.push_back(kv.first);  // pin_v order: ascending vertex
    for (uint32_t q = 0; q < uint32_t(pv.size());) {
      const uint32_t slot = bin_of_v[pv[q]] * K + owner[pv[q]];
      uint32_t e = q;
      while (e < pv.size() && bin_of_v[pv[e]] * K + owner[pv[e]] == slot) ++e;
      pr[slot] = make_uint2(q, e - q);
      q = e;
    }
    auto perm_of = [&](const std::vector<uint32_t>& off, const std::vector<uint32_t>& cnt, auto vert_of,
                       std::vector<uint32_t>& perm, std::vector<uint32_t>& tab) {
      const uint32_t nc = uint32_t(off.size());
      std::vector<std::vector<uint32_t>> bucket(size_t(B) * nc * K);
      for (uint32_t c = 0; c < nc; ++c)
        for (uint32_t k = off[c]; k < off[c] + cnt[c]; ++k) {
          const uint32_t v = vert_of(k);
          bucket[(size_t(bin_of_v[v]) * nc + c) * K + owner[v]].push_back(k);
        }
      perm.clear();
      tab.assign(size_t(B) * nc * (K + 1), 0u);
      for (size_t bc = 0; bc < size_t(B) * nc; ++bc) {
        for (uint32_t r = 0; r < K; ++r) {
          tab[bc * (K + 1) + r] = uint32_t(perm.size());
          perm.insert(perm.end(), bucket[bc * K + r].begin(), bucket[bc * K + r].end());
        }
        tab[bc * (K + 1) + K] = uint32_t(perm.size());
      }
    };
    std::vector<uint32_t> dperm, bperm, dtab, btab;
    perm_of(m.dist_off, m.dist_cnt, [&](uint32_t k) { return dist_h[k].v0; }, dperm, dtab);
    perm_of(m.bend_off, m.bend_cnt, [&](uint32_t k) { return bend_h[k].v0; }, bperm, btab);
    st_vrange.upload(vr, st);
    st_pins.upload(pr, st);
    st_dist.upload(dtab, st);
    st_bend.upload(btab, st);
    st_dperm.upload(dperm, st);
    st_bperm.upload(bperm, st);
    // the records in staged order
    const uint32_t ndp = uint32_t(dperm.size()), nbp = uint32_t(bperm.size());
    st_dids.alloc(ndp); st_dpar.alloc(ndp); st_dlam.alloc(ndp);
    st_bids.alloc(nbp); st_bpar.alloc(nbp); st_blam.alloc(nbp);
    // vertex ids as staged ids: owning slice << 16 | slot in that slice
    std::vector<uint32_t> sid(n);
    for (uint32_t b = 0; b < B; ++b) {
      const uint32_t nv = vr[b].y - vr[b].x, chunk = nv ? (nv + K - 1) / K : 1u;
      for (uint32_t v = vr[b].x; v < vr[b].y; ++v) {
        const uint32_t o = v - vr[b].x;
        sid[v] = ((o / chunk) << 16) | (o % chunk);
      }
    }
    std::vector<uint2> dids(ndp);
    for (uint32_t k = 0; k < ndp; ++k) dids[k] = make_uint2(sid[dist_h[dperm[k]].v0], sid[dist_h[dperm[k]].v1]);
    std::vector<uint4> bids(nbp);
    for (uint32_t k = 0; k < nbp; ++k) {
      const BendC& c = bend_h[bperm[k]];
      bids[k] = make_uint4(sid[c.v0], sid[c.v1], sid[c.v2], sid[c.v3]);
    }
    st_dids.upload(dids, st);
    st_bids.upload(bids, st);
    if (ndp) k_stage_gather<<<grid(ndp, 256), 256, 0, st>>>(ndp, st_dperm.p, dist_par.p, st_dpar.p);
    if (nbp) k_stage_gather<<<grid(nbp, 256), 256, 0, st>>>(nbp, st_bperm.p, bend_par.p, st_bpar.p);
    TC_CK(cudaGetLastError());
    TC_CK(cudaStreamSynchronize(st));
    st_bins = B;
    st_stale = false;
    mark();  // a captured frame holds the old tables
  }
  void launch_staged(const SolverArgs& a) {
    const StageTables t{st_vrange.p, st_pins.p, st_dist.p, st_bend.p, st_dids.p, st_dpar.p, st_dlam.p,
                        st_bids.p,   st_bpar.p, st_blam.p, st_cap};
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(st_bins * kStageCtas);
    cfg.blockDim = dim3(kStageThreads);
    cfg.dynamicSmemBytes = st_smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = kStageCtas;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (a.ca.bone.nbones > 0) TC_CK(cudaLaunchKernelEx(&cfg, k_solver_staged<kStageCtas, true>, a, t));
    else TC_CK(cudaLaunchKernelEx(&cfg, k_solver_staged<kStageCtas, false>, a, t));
  }
  // the persistent path is available: cooperative launch, and with bone
  // colliders the bone instantiation fits on an SM
  bool can_persist() const { return persist_blocks > 0 && (!bone.enabled || persist_bone_per_sm > 0); }
  unsigned persist_grid(bool with_bone) const {
    if (!with_bone) return persist_blocks;
    return num_sms * std::min(persist_blocks / std::max(num_sms, 1u), persist_bone_per_sm);
  }
  void launch_persistent(const SolverArgs& args) {
    SolverArgs a = args;
    const bool with_bone = a.ca.bone.nbones > 0;
    const unsigned blocks = persist_grid(with_bone);
    if (a.expected == 0) a.expected = blocks;
    TC_CK(cudaMemsetAsync(a.bar, 0, sizeof(GridBar), st));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(blocks);
    cfg.blockDim = dim3(256);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (with_bone) TC_CK(cudaLaunchKernelEx(&cfg, k_solver_persistent<true>, a));
    else TC_CK(cudaLaunchKernelEx(&cfg, k_solver_persistent<false>, a));
  }

  // ---- learned warm start
  void ws_setup() {
    if (ws.ready) return;
    ws.net.setup(st, n, adj_off.p, adj_idx.p);
    ws.net.err = &bar.p->err;  // read back with the frame's barrier status
    ws.net.set_ell(m.adj_off.data(), m.adj_idx.data());
    const std::vector<float> blob = Mlp::init_blob(1);
    ws.net.set_params(blob.data());
    ws.ppred.alloc(n);
    ws.dprev.alloc(n);
    std::vector<float> rest(m.adj_idx.size());
    for (uint32_t i = 0; i < n; ++i)
      for (uint32_t q = m.adj_off[i]; q < m.adj_off[i + 1]; ++q) {
        const uint32_t j = m.adj_idx[q];
        const float dx = init_pos[3 * i] - init_pos[3 * j], dy = init_pos[3 * i + 1] - init_pos[3 * j + 1],
                    dz = init_pos[3 * i + 2] - init_pos[3 * j + 2];
        rest[q] = std::sqrt(dx * dx + dy * dy + dz * dz);
      }
    ws.adj_rest.upload(rest, st);
    ws.res_max.alloc(1);
    ws.res_part.alloc(size_t(num_sms) * std::max(persist_max_per_sm, 4u));
    ws.fallbacks.alloc(1);
    ws.gate.alloc(1);
    ws.res_pred.alloc(1);
    TC_CK(cudaMemsetAsync(ws.dprev.p, 0, size_t(n) * sizeof(float4), st));
    TC_CK(cudaMemsetAsync(ws.res_max.p, 0, sizeof(float), st));
    TC_CK(cudaMemsetAsync(ws.fallbacks.p, 0, sizeof(unsigned int), st));
    TC_CK(cudaStreamSynchronize(st));
    ws.ready = true;
  }
  WsFeatArgs ws_feat_args(const SubstepParams& sp, __nv_bfloat16* feat) {
    WsFeatArgs f;
    f.n = n; f.x4 = x4.p; f.p4 = p4.p; f.v4 = v4.p; f.dprev = ws.dprev.p; f.local_len = local_len.p;
    f.adj_off = adj_off.p; f.adj_idx = adj_idx.p; f.adj_rest = ws.adj_rest.p;
    f.prims = prims.p; f.nprims = uint32_t(prims_h.size());
    f.vinst = inst_prims_h.empty() ? nullptr : vinst.p;
    f.inst_prims = inst_prims_h.empty() ? nullptr : inst_prims.p;
    f.dt = sp.dt;
    f.g_dt2 = std::sqrt(sp.gx * sp.gx + sp.gy * sp.gy + sp.gz * sp.gz) * sp.dt * sp.dt;
    f.feat = feat;
    return f;
  }
  bool ws_recording() const { return ws.ready && ws.rec_count < ws.rec_cap; }
  // One frame with the warm start: per substep predict, features, MLP, move
  // p by the predicted correction, then iters - k iterations, the RMS
  // residual judged against the plain solver's, and k more iterations when
  // it misses.  The solver part is one persistent launch per substep, or, in
  // the per-colour launch mode, the per-colour kernels with the residual
  // check on the device and the fallback iterations gated by its flag.
  void encode_frame_ws(float dt, uint32_t substeps, bool use_coupled) {
    const SubstepParams sp = make_sp(dt / float(substeps));
    const uint32_t itn = run_iters();
    const uint32_t kk = std::min(ws.k, itn > 1 ? itn - 1 : 0u);
    const WsFeatArgs fa = ws_feat_args(sp, nullptr);
    const bool colors = !persistent || cluster_mode;
    for (uint32_t s = 0; s < substeps; ++s) {
      if (colors) {
        encode_substep_ws_colors(sp, use_coupled, itn, kk, fa);
      } else {
        timed("predict", [&] { k_predict<<<grid(n, 256), 256, 0, st>>>(n, x4.p, p4.p, v4.p, sp); });
        SolverArgs a = solver_args(sp, 1, use_coupled, !(self_collision || edge_active()));
        timed("ws_check", [&] { encode_ws_res_pred(sp.dt, a.ca.bone.nbones > 0); });
        timed("ws_mlp", [&] { ws.net.infer(nullptr, &fa, ws.ppred.p, nullptr, x4.p, p4.p, local_len.p); });
        a.skip_predict = true;
        a.iters = itn - kk;
        a.iters_extra = kk;
        a.ppred = ws.ppred.p;
        a.dprev = ws.dprev.p;
        a.res_thresh = ws.res_thresh;
        a.res_ratio = ws.res_ratio;
        a.res_floor = ws_res_floor();
        a.res_pred = ws.res_pred.p;
        a.res_part = ws.res_part.p;
        a.res_out = ws.res_max.p;
        a.fallbacks = ws.fallbacks.p;
        timed("solver", [&] { launch_persistent(a); });
      }
      if (self_collision || edge_active()) {
        if (edge_active()) encode_edge_collision();
        if (sc_due(s, substeps)) encode_self_collision(ee_due(s, substeps), s, substeps, dt);
        if (nsw) timed("final_sewing", [&] { launch_sewing(sp.dt); });
        timed("update_vel", [&] { launch_k(k_update_vel, grid(n, 256), 256, n, x4.p, p4.p, v4.p, sp.dt); });
      } else if (colors) {
        if (nsw) timed("final_sewing", [&] { launch_sewing(sp.dt); });
        timed("update_vel", [&] { launch_k(k_update_vel, grid(n, 256), 256, n, x4.p, p4.p, v4.p, sp.dt); });
      }
    }
    TC_CK(cudaMemcpyAsync(h_err, &bar.p->err, sizeof(int), cudaMemcpyDeviceToHost, st));
    TC_CK(cudaGetLastError());
  }
  WsCheckArgs ws_check_args(float dts) {
    return WsCheckArgs{nd, nb, dist_ids.p, dist_par.p, bend_ids.p, bend_par.p, p4.p, dlam.p, blam.p, dts,
                       ws.res_thresh, ws.res_ratio, ws_res_floor(), ws.res_pred.p, ws.res_part.p, ws.res_max.p,
                       ws.fallbacks.p, ws.gate.p};
  }
  // floor of a relative threshold: a strain of 1e-6 of the mean edge length
  // (a rigidly moving cloth has a zero predicted residual)
  float ws_res_floor() const { return 1e-6f * ad.mesh_avg_edge_len;
  }
  // with a relative threshold: the residual of the predicted positions
  // (before the network moves them), lambdas read as zero
  void encode_ws_res_pred(float dts, bool bone_col) {
    if (ws.res_ratio <= 0.f) return;
    WsCheckArgs c = ws_check_args(dts);
    c.dlam = nullptr;
    c.blam = nullptr;
    const unsigned parts = persist_grid(bone_col);
    launch_k(k_ws_res_part, parts, 256, c);
    launch_k(k_ws_res_pred, 1, 32, c, uint32_t(parts));
  }
  // The constraint phase of one warm-started substep with per-colour
  // launches (the order of k_solver_persistent: clear lambdas, predict, the
  // network, iterations, check, gated iterations, the correction for the
  // next substep's features, decoupled collision, final pins).
  void encode_substep_ws_colors(const SubstepParams& sp, bool use_coupled, uint32_t itn, uint32_t kk,
                                const WsFeatArgs& fa) {
    const float dts = sp.dt;
    const bool ddamp = td != 0.f || cd != 0.f || sd != 0.f;
    const bool bdamp = bd != 0.f;
    const bool hascol = has_colliders();
    const uint32_t npins = uint32_t(pins.size());
    const ColliderArgs ca = collider_args();
    const bool bone_col = ca.bone.nbones > 0;
    if (nd) TC_CK(cudaMemsetAsync(dlam.p, 0, nd * sizeof(float), st));
    if (nb) TC_CK(cudaMemsetAsync(blam.p, 0, nb * sizeof(float), st));
    if (nsw) timed("sew_shrink", [&] { launch_sew_start(dts); });
    timed("predict", [&] { launch_k(k_predict, grid(n, 256), 256, n, x4.p, p4.p, v4.p, sp); });
    timed("ws_check", [&] { encode_ws_res_pred(dts, bone_col); });
    timed("ws_mlp", [&] { ws.net.infer(nullptr, &fa, ws.ppred.p, nullptr, x4.p, p4.p, local_len.p); });
    auto iteration = [&](const unsigned int* gate) {
      if (npins) {
        if (gate) launch_k(k_pin_gated, grid(npins, 128), 128, gate, npins, pin_v.p, pin_t.p, x4.p, p4.p, dts);
        else launch_k(k_pin, grid(npins, 128), 128, npins, pin_v.p, pin_t.p, x4.p, p4.p, dts);
      }
      for (size_t c = 0; c < m.dist_cnt.size(); ++c)
        if (m.dist_cnt[c]) {
          if (gate)
            launch_k(k_distance_gated, grid(m.dist_cnt[c], col_block), col_block, gate, m.dist_off[c], m.dist_cnt[c], dist_ids.p,
                     dist_par.p, x4.p, p4.p, dlam.p, sp, ddamp);
          else
            launch_k(k_distance, grid(m.dist_cnt[c], col_block), col_block, m.dist_off[c], m.dist_cnt[c], dist_ids.p,
                     dist_par.p, x4.p, p4.p, dlam.p, sp, ddamp);
        }
      if (nsw) launch_sewing(dts, gate);
      for (size_t c = 0; c < m.bend_cnt.size(); ++c)
        if (m.bend_cnt[c]) {
          if (gate)
            launch_k(k_bending_gated, grid(m.bend_cnt[c], col_block), col_block, gate, m.bend_off[c], m.bend_cnt[c], bend_ids.p,
                     bend_par.p, x4.p, p4.p, blam.p, sp, bdamp);
          else
            launch_k(k_bending, grid(m.bend_cnt[c], col_block), col_block, m.bend_off[c], m.bend_cnt[c], bend_ids.p,
                     bend_par.p, x4.p, p4.p, blam.p, sp, bdamp);
        }
      if (hascol && use_coupled) {
        if (!gate) launch_collision(ca, dts);
        else if (bone_col) launch_k(k_collision_gated<true>, grid(n, 128), 128, gate, n, x4.p, p4.p, ca, dts, col_order.p);
        else launch_k(k_collision_gated<false>, grid(n, 128), 128, gate, n, x4.p, p4.p, ca, dts, col_order.p);
      }
    };
    timed("solver", [&] {
      for (uint32_t it = 0; it < itn - kk; ++it) iteration(nullptr);
      if (kk) {
        const WsCheckArgs c = ws_check_args(dts);
        const unsigned parts = persist_grid(bone_col);
        launch_k(k_ws_res_part, parts, 256, c);
        launch_k(k_ws_res_decide, 1, 32, c, uint32_t(parts));
        for (uint32_t it = 0; it < kk; ++it) iteration(ws.gate.p);
      }
      k_ws_correction<<<grid(n, 256), 256, 0, st>>>(n, p4.p, ws.ppred.p, x4.p, local_len.p, ws.dprev.p, nullptr,
                                                    nullptr);
      if (hascol && !use_coupled) launch_collision(ca, dts);
      if (npins) launch_k(k_pin, grid(npins, 128), 128, npins, pin_v.p, pin_t.p, x4.p, p4.p, dts);
    });
  }
  // train on the recorded snapshots: epochs x snapshots Adam steps in a
  // seeded shuffled order; returns the mean loss of the first and last epoch
  void ws_train(uint32_t epochs, float lr, uint64_t seed, float* first, float* last) {
    if (!ws.ready || ws.rec_count == 0) throw TcError(TC_ERR_INVALID, "no recorded snapshots to train on");
    if (epochs == 0) throw TcError(TC_ERR_INVALID, "epochs must be positive");
    const uint32_t cnt = ws.rec_count;
    ws.net.alloc_train();
    if (!ws.normalized) {
      ws.net.fit_normalizer(ws.rec_feat.p, ws.rec_target.p, ws.rec_mask.p, size_t(cnt) * n);
      ws.normalized = true;
    }
    ws.losses.alloc(size_t(epochs) * cnt);
    TC_CK(cudaMemsetAsync(ws.losses.p, 0, size_t(epochs) * cnt * sizeof(float), st));
    std::vector<uint32_t> order(cnt);
    for (uint32_t i = 0; i < cnt; ++i) order[i] = i;
    uint64_t x = seed * 2862933555777941757ull + 3037000493ull;
    for (uint32_t ep = 0; ep < epochs; ++ep) {
      for (uint32_t i = cnt; i > 1; --i) {
        x = x * 6364136223846793005ull + 1442695040888963407ull;
        std::swap(order[i - 1], order[uint32_t((x >> 33) % i)]);
      }
      for (uint32_t j = 0; j < cnt; ++j) {
        const uint32_t sidx = order[j];
        const __nv_bfloat16* f = ws.rec_feat.p + size_t(sidx) * n * kWsF;
        ws.net.forward(f, true, ws.rec_target.p + size_t(sidx) * n * 3, ws.rec_mask.p + size_t(sidx) * n,
                       ws.losses.p + size_t(ep) * cnt + j);
        ws.net.backward();
        ws.net.adam(lr);
      }
    }
    std::vector<float> h(size_t(epochs) * cnt);
    TC_CK(cudaMemcpyAsync(h.data(), ws.losses.p, h.size() * sizeof(float), cudaMemcpyDeviceToHost, st));
    TC_CK(cudaMemcpyAsync(h_err, &bar.p->err, sizeof(int), cudaMemcpyDeviceToHost, st));
    TC_CK(cudaStreamSynchronize(st));
    TC_CK(cudaGetLastError());
    check_barrier_status();
    double a = 0, b = 0;
    for (uint32_t j = 0; j < cnt; ++j) { a += h[j]; b += h[size_t(epochs - 1) * cnt + j]; }
    if (first) *first = float(a / cnt);
    if (last) *last = float(b / cnt);
  }

  // Launch of a per-colour-path kernel; with pdl (not while profiling) the
  // launch carries programmatic stream serialization, so the kernel's launch
  // overlaps the tail of the previous one (the kernel waits for its data).
  bool pdl = true;
  template <typename... KArgs, typename... Args>
  void launch_k(void (*kern)(KArgs...), unsigned gx, unsigned block, Args... args) {
    if (!pdl || profiling) {
      kern<<<gx, block, 0, st>>>(args...);
      return;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(gx);
    cfg.blockDim = dim3(block);
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    TC_CK(cudaLaunchKernelEx(&cfg, kern, args...));
  }
  void launch_collision(const ColliderArgs& ca, float dts) {
    if (ca.bone.nbones > 0) launch_k(k_collision<true>, grid(n, 128), 128, n, x4.p, p4.p, ca, dts, col_order.p);
    else launch_k(k_collision<false>, grid(n, 128), 128, n, x4.p, p4.p, ca, dts, col_order.p);
  }

  // encode_simulation_steps (dispatch.rs:7-354) for one frame
  void encode_frame(float dt, uint32_t substeps, bool use_coupled) {
    if (ws.on && !ws_recording()) {
      encode_frame_ws(dt, substeps, use_coupled);
      return;
    }
    if (stage_mode && can_stage() && !st_stale && !profiling && !track_residual && !ws_recording()) {
      const SubstepParams sp = make_sp(dt / float(substeps));
      launch_staged(solver_args(sp, substeps, use_coupled, true));
      TC_CK(cudaGetLastError());
      return;
    }
    if (cluster_mode && can_cluster() && !cl_stale && !profiling && !track_residual && !ws_recording()) {
      const SubstepParams sp = make_sp(dt / float(substeps));
      launch_cluster(solver_args(sp, substeps, use_coupled, true));
      TC_CK(cudaGetLastError());
      return;
    }
    if (persistent && can_persist() && !profiling && !track_residual && !ws_recording()) {
      const SubstepParams sp = make_sp(dt / float(substeps));
      if (!self_collision && !edge_active()) {
        launch_persistent(solver_args(sp, substeps, use_coupled, true));
      } else {
        for (uint32_t s = 0; s < substeps; ++s) {
          launch_persistent(solver_args(sp, 1, use_coupled, false));
          if (edge_active()) encode_edge_collision();
          if (sc_due(s, substeps)) encode_self_collision(ee_due(s, substeps), s, substeps, dt);
          launch_sewing(sp.dt);  // final sewing (dispatch.rs:323-337)
          k_update_vel<<<grid(n, 256), 256, 0, st>>>(n, x4.p, p4.p, v4.p, sp.dt);
        }
      }
      TC_CK(cudaMemcpyAsync(h_err, &bar.p->err, sizeof(int), cudaMemcpyDeviceToHost, st));
      TC_CK(cudaGetLastError());
      return;
    }
    const float dts = dt / float(substeps);
    SubstepParams sp = make_sp(dts);
    const bool ddamp = td != 0.f || cd != 0.f || sd != 0.f;
    const bool bdamp = bd != 0.f;
    const bool hascol = has_colliders();
    const uint32_t npins = uint32_t(pins.size());
    ColliderArgs ca = collider_args();
    for (uint32_t s = 0; s < substeps; ++s) {
      if (nd) TC_CK(cudaMemsetAsync(dlam.p, 0, nd * sizeof(float), st));
      if (nb) TC_CK(cudaMemsetAsync(blam.p, 0, nb * sizeof(float), st));
      if (nsw) timed("sew_shrink", [&] { launch_sew_start(dts); });
      timed("predict", [&] { launch_k(k_predict, grid(n, 256), 256, n, x4.p, p4.p, v4.p, sp); });
      if (track_residual && s + 1 == substeps && nd + nb)
        k_residual_pred<<<grid(nd + nb, 256), 256, 0, st>>>(nd, nb, dist_ids.p, dist_par.p, bend_ids.p, bend_par.p,
                                                           p4.p, fmaxf(dts, 1e-8f),
                                                           res_sum.p + m.dist_cnt.size() + m.bend_cnt.size());
      // recording for the warm start: features after predict, the
      // iterations' correction as the target
      const bool rec = ws_recording();
      const bool rec_this = rec && (ws.rec_phase++ % ws.rec_every) == 0;
      const uint32_t slot = ws.rec_count;
      if (rec) {
        k_copy4<<<grid(n, 256), 256, 0, st>>>(n, p4.p, ws.ppred.p);
        if (rec_this)
          k_ws_features<<<grid(n, 128), 128, 0, st>>>(ws_feat_args(sp, ws.rec_feat.p + size_t(slot) * n * kWsF));
      }
      for (uint32_t it = 0, itn = run_iters(); it < itn; ++it) {
        if (npins) timed("pin", [&] { launch_k(k_pin, grid(npins, 128), 128, npins, pin_v.p, pin_t.p, x4.p, p4.p, dts); });
        timed("distance", [&] {
          for (size_t c = 0; c < m.dist_cnt.size(); ++c)
            if (m.dist_cnt[c])
              launch_k(k_distance, grid(m.dist_cnt[c], col_block), col_block, m.dist_off[c], m.dist_cnt[c], dist_ids.p,
                       dist_par.p, x4.p, p4.p, dlam.p, sp, ddamp);
        });
        if (nsw) timed("sewing", [&] { launch_sewing(dts); });
        timed("bending", [&] {
          for (size_t c = 0; c < m.bend_cnt.size(); ++c)
            if (m.bend_cnt[c])
              launch_k(k_bending, grid(m.bend_cnt[c], col_block), col_block, m.bend_off[c], m.bend_cnt[c], bend_ids.p,
                       bend_par.p, x4.p, p4.p, blam.p, sp, bdamp);
        });
        if (hascol && use_coupled) timed("collision", [&] { launch_collision(ca, dts); });
      }
      if (track_residual && s + 1 == substeps) encode_residual(sp);
      if (rec) {
        k_ws_correction<<<grid(n, 256), 256, 0, st>>>(n, p4.p, ws.ppred.p, x4.p, local_len.p, ws.dprev.p,
                                                      rec_this ? ws.rec_target.p + size_t(slot) * n * 3 : nullptr,
                                                      rec_this ? ws.rec_mask.p + size_t(slot) * n : nullptr);
        if (rec_this) ++ws.rec_count;
      }
      if (hascol && !use_coupled) timed("collision", [&] { launch_collision(ca, dts); });
      if (npins) timed("pin", [&] { launch_k(k_pin, grid(npins, 128), 128, npins, pin_v.p, pin_t.p, x4.p, p4.p, dts); });
      if (edge_active()) encode_edge_collision();
      if (sc_due(s, substeps)) encode_self_collision(ee_due(s, substeps), s, substeps, dt);
      if (nsw) timed("final_sewing", [&] { launch_sewing(dts); });
      timed("update_vel", [&] { launch_k(k_update_vel, grid(n, 256), 256, n, x4.p, p4.p, v4.p, dts); });
    }
    TC_CK(cudaGetLastError());
  }

  // auto-coupled decision (dispatch.rs:93-102)
  bool coupled_for(float dt, uint32_t substeps) const {
    const float dts = dt / float(substeps);
    const float ga = std::sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
    const float ff = 0.5f * ga * dts * dts;
    const float emd = std::fmax(last_eff_disp, last_max_disp);
    const float sdp = std::fmax(ff, emd / std::fmax(float(substeps), 1.f));
    const float sm = std::fmax(cloth_thickness * 0.8f, 0.002f);
    return coupled || (auto_coupled && sdp > sm * 0.25f);
  }

  void launch_frame(float dt, uint32_t substeps) {
    if (n == 0) return;
    if (cluster_mode && can_cluster() && cl_stale) build_cluster_tables();  // before any capture
    if (stage_mode && can_stage() && st_stale) build_stage_tables();        // before any capture
    if (edge_active()) ensure_collider_edges();                             // before any capture
    // the frame's device time (last_frame_ms) includes the dynamic bone SDF rebake
    TC_CK(cudaEventRecord(ev0, st));
    dynamic_bone_update();
    const bool use_coupled = coupled_for(dt, substeps);
    if (ws.on && !ws_recording()) ws.substeps_run += substeps;
    if (profiling || ws_recording()) {
      encode_frame(dt, substeps, use_coupled);
      TC_CK(cudaEventRecord(ev1, st));
      TC_CK(cudaStreamSynchronize(st));
      if (profiling) collect_marks();
      return;
    }
    if (graph_dirty || !gexec || g_dt != dt || g_sub != substeps || g_coupled != use_coupled ||
        g_iters != run_iters()) {
      if (gexec) { cudaGraphExecDestroy(gexec); gexec = nullptr; }
      cudaGraph_t graph = nullptr;
      TC_CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      try {
        encode_frame(dt, substeps, use_coupled);
      } catch (...) {
        cudaStreamEndCapture(st, &graph);
        if (graph) cudaGraphDestroy(graph);
        throw;
      }
      TC_CK(cudaStreamEndCapture(st, &graph));
      size_t nn = 0;
      TC_CK(cudaGraphGetNodes(graph, nullptr, &nn));
      std::vector<cudaGraphNode_t> nodes(nn);
      if (nn) TC_CK(cudaGraphGetNodes(graph, nodes.data(), &nn));
      graph_kernels = 0;
      for (auto nd_ : nodes) {
        cudaGraphNodeType t;
        TC_CK(cudaGraphNodeGetType(nd_, &t));
        if (t == cudaGraphNodeTypeKernel) ++graph_kernels;
      }
      cudaError_t e = cudaGraphInstantiate(&gexec, graph, 0);
      cudaGraphDestroy(graph);
      TC_CK(e);
      graph_dirty = false;
      g_dt = dt;
      g_sub = substeps;
      g_coupled = use_coupled;
      g_iters = run_iters();
    }
    if (track_residual) {
      const size_t k = m.dist_cnt.size() + m.bend_cnt.size();
      TC_CK(cudaMemsetAsync(res_sum.p, 0, (k + 1) * sizeof(float), st));
      TC_CK(cudaMemsetAsync(res_max.p, 0, (k + 1) * sizeof(float), st));
    }
    TC_CK(cudaGraphLaunch(gexec, st));
    TC_CK(cudaEventRecord(ev1, st));
  }

  uint32_t graph_kernels = 0;
  void check_barrier_status() {
    if (*h_err != 0) {
      const int e = *h_err;
      *h_err = 0;
      TC_CK(cudaMemsetAsync(bar.p, 0, sizeof(GridBar), st));
      TC_CK(cudaStreamSynchronize(st));
      throw TcError(TC_ERR_TIMEOUT, e == 2 ? "a tensor-core completion wait of the warm-start network timed out; "
                                             "the frame is incomplete"
                                           : "a grid barrier of the persistent solver timed out; the frame is incomplete");
    }
  }
  // ---- adaptive substeps: plan before a frame, GPU feedback after it
  void adaptive_enable_buffers() {
    if (h_fb) return;
    const uint32_t total = nd;
    fb_stride = std::max(total / 2048u, 1u);
    fb_nsamp = total ? (total + fb_stride - 1) / fb_stride : 0u;
    fb_prev.alloc(n);
    fb_out.alloc(1 + std::max(fb_nsamp, 1u));
    rest0.upload(base_rest, st);
    TC_CK(cudaMemcpyAsync(fb_prev.p, x4.p, size_t(n) * sizeof(float4), cudaMemcpyDeviceToDevice, st));
    TC_CK(cudaHostAlloc(&h_fb, (2 + size_t(fb_nsamp)) * sizeof(float), cudaHostAllocDefault));
    TC_CK(cudaStreamSynchronize(st));
  }
  uint32_t plan_frame(float dt, uint32_t requested) {
    const uint32_t sub = ad.substeps(dt, requested, g, n);
    ad.iterations(iters, sub);
    return sub;
  }
  void encode_feedback() {
    if (!ad.enabled || !h_fb) return;
    TC_CK(cudaMemsetAsync(fb_out.p, 0, sizeof(float), st));
    k_fb_disp<<<grid(n, 256), 256, 0, st>>>(n, x4.p, fb_prev.p, fb_out.p);
    const float min_ref = std::fmax(0.5f * ad.mesh_avg_edge_len, 0.002f);
    if (fb_nsamp)
      k_fb_strain<<<grid(fb_nsamp, 256), 256, 0, st>>>(fb_nsamp, fb_stride, dist_ids.p, rest0.p, x4.p, min_ref,
                                                       fb_out.p + 1);
    TC_CK(cudaMemcpyAsync(h_fb, fb_out.p, (1 + size_t(fb_nsamp)) * sizeof(float), cudaMemcpyDeviceToHost, st));
  }
  void consume_feedback() {  // after the stream is synchronised
    if (!ad.enabled || !h_fb) return;
    ad.last_max_disp = h_fb[0];
    last_max_disp = h_fb[0];
    std::vector<float> pos;
    for (uint32_t k = 0; k < fb_nsamp; ++k)
      if (h_fb[1 + k] > 0.f) pos.push_back(h_fb[1 + k]);
    ad.last_strain = AdaptiveCtl::p95(std::move(pos));
  }
  void step(float dt, uint32_t substeps) {
    launch_frame(dt, substeps);
    encode_feedback();
    TC_CK(cudaStreamSynchronize(st));
    TC_CK(cudaGetLastError());
    check_barrier_status();
    consume_feedback();
  }

  // buffered frames (dispatch.rs:1293-1408): positions of up to 8 frames
  // kept on the device, fetched in one copy
  static constexpr uint32_t kMaxBuffered = 8;
  DBuf<float> ring;
  uint32_t buffered = 0;
  uint32_t step_buffered(float dt, uint32_t substeps) {
    if (n == 0) return 0;
    ring.alloc(size_t(kMaxBuffered) * n * 3);
    const uint32_t slot = std::min(buffered, kMaxBuffered - 1);
    launch_frame(dt, substeps);
    encode_feedback();
    k_extract_positions<<<grid(n, 256), 256, 0, st>>>(n, x4.p, ring.p + size_t(slot) * n * 3);
    TC_CK(cudaGetLastError());
    if (buffered < kMaxBuffered) ++buffered;
    return buffered;
  }
  // positions packed xyz on the device, one copy into a pinned staging
  // buffer, then into the caller's array
  DBuf<float> pos3;
  float* h_pos3 = nullptr;
  uint32_t pos3_cap = 0;  // vertices the two staging buffers hold
  void get_positions(float* out) {
    if (n == 0) return;
    if (pos3_cap < n) {
      if (h_pos3) TC_CK(cudaFreeHost(h_pos3));
      h_pos3 = nullptr;
      pos3.alloc(size_t(n) * 3);
      TC_CK(cudaHostAlloc(&h_pos3, size_t(n) * 3 * sizeof(float), cudaHostAllocDefault));
      pos3_cap = n;
    }
    k_extract_positions<<<grid(n, 256), 256, 0, st>>>(n, x4.p, pos3.p);
    TC_CK(cudaGetLastError());
    TC_CK(cudaMemcpyAsync(h_pos3, pos3.p, size_t(n) * 3 * sizeof(float), cudaMemcpyDeviceToHost, st));
    TC_CK(cudaStreamSynchronize(st));
    std::memcpy(out, h_pos3, size_t(n) * 3 * sizeof(float));
  }
};

// Residual |C(x) + alpha~ lambda| per constraint after the last iteration,
// reduced per colour into (sum of squares, max).
__global__ void k_residual_dist(uint32_t off, uint32_t cnt, const uint2* ids, const float4* par, const float4* p4,
                                const float* lam, float dt, float* sum, float* mx) {
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  float r = 0.f;
  if (k < cnt) {
    const uint32_t ci = off + k;
    const uint2 e = ids[ci];
    const float4 c = par[ci];
    const float dist = length(mk(p4[e.x]) - mk(p4[e.y]));
    const float cv = dist - c.x;
    const float comp = cv >= 0.f ? c.y : c.z;
    if (comp < 1e9f) r = fabsf(cv + comp / (dt * dt) * lam[ci]);
  }
  float s = r * r, m2 = r;
  for (int o = 16; o > 0; o >>= 1) {
    s += __shfl_down_sync(0xffffffffu, s, o);
    m2 = fmaxf(m2, __shfl_down_sync(0xffffffffu, m2, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(sum, s);
    atomicMax(reinterpret_cast<int*>(mx), __float_as_int(m2));
  }
}
__global__ void k_residual_bend(uint32_t off, uint32_t cnt, const uint4* ids, const float4* par, const float4* p4,
                                const float* lam, float dt, float* sum, float* mx) {
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  float r = 0.f;
  if (k < cnt) {
    const uint32_t ci = off + k;
    const uint4 e = ids[ci];
    const float4 c = par[ci];
    if (c.y < 1e9f) {
      const float cv = length(mk(p4[e.z]) - mk(p4[e.w])) - c.x;
      r = fabsf(cv + c.y / (dt * dt) * lam[ci]);
    }
  }
  float s = r * r, m2 = r;
  for (int o = 16; o > 0; o >>= 1) {
    s += __shfl_down_sync(0xffffffffu, s, o);
    m2 = fmaxf(m2, __shfl_down_sync(0xffffffffu, m2, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(sum, s);
    atomicMax(reinterpret_cast<int*>(mx), __float_as_int(m2));
  }
}

void Sim::encode_residual(const SubstepParams& sp) {
  const float dt = fmaxf(sp.dt, 1e-8f);
  const size_t kd = m.dist_cnt.size();
  for (size_t c = 0; c < kd; ++c)
    if (m.dist_cnt[c])
      k_residual_dist<<<grid(m.dist_cnt[c], col_block), col_block, 0, st>>>(m.dist_off[c], m.dist_cnt[c], dist_ids.p, dist_par.p,
                                                                 p4.p, dlam.p, dt, res_sum.p + c, res_max.p + c);
  for (size_t c = 0; c < m.bend_cnt.size(); ++c)
    if (m.bend_cnt[c])
      k_residual_bend<<<grid(m.bend_cnt[c], col_block), col_block, 0, st>>>(m.bend_off[c], m.bend_cnt[c], bend_ids.p, bend_par.p,
                                                                 p4.p, blam.p, dt, res_sum.p + kd + c,
                                                                 res_max.p + kd + c);
}

}  // namespace tcloth

// ===================================================================
// C ABI
// ===================================================================
using tcloth::GridBar;
using tcloth::Sim;
using tcloth::SolverArgs;
using tcloth::SubstepParams;
using tcloth::TcError;

struct tc_sim {
  Sim s;
};
static tcloth::Prim make_prim(uint32_t type, const float* a, const float* b, float r, float f, float rest) {
  float tf;
  std::memcpy(&tf, &type, 4);
  return tcloth::Prim{make_float4(f, rest, r, tf), make_float4(a[0], a[1], a[2], 0.f),
                      make_float4(b ? b[0] : 0.f, b ? b[1] : 0.f, b ? b[2] : 0.f, 0.f)};
}


static thread_local std::string g_err;

template <class F>
static tc_status guard(F&& f) {
  try {
    f();
    g_err.clear();
    return TC_OK;
  } catch (const TcError& e) {
    g_err = e.what();
    return e.code;
  } catch (const std::bad_alloc&) {
    g_err = "host allocation failed";
    return TC_ERR_NOMEM;
  } catch (const std::exception& e) {
    g_err = e.what();
    return TC_ERR_CUDA;
  }
}
static void need(bool ok, const char* msg) {
  if (!ok) throw TcError(TC_ERR_INVALID, msg);
}
// ---- device health (crates/cloth_core/src/context.rs:101-140): a per-device
// "lost" flag and context epoch.  A device marked lost is re-initialised by
// the next simulator creation on it (epoch + 1); simulators of an older epoch
// refuse every call with TC_ERR_CUDA and must be re-created.  Marking is
// host-side (tc_mark_device_lost) and never touches the GPU; re-initialising
// synchronises the device and gives up when it does not answer, since a real
// sticky fault needs a fresh process.
namespace {
struct DeviceHealth {
  std::atomic<bool> lost{false};
  std::atomic<uint64_t> epoch{1};
};
DeviceHealth g_health[64];
std::mutex g_health_mu;
DeviceHealth& health(int dev) {
  if (dev < 0 || dev >= 64) throw TcError(TC_ERR_CUDA, "device index out of range");
  return g_health[dev];
}
uint64_t acquire_device(int dev) {
  DeviceHealth& h = health(dev);
  if (!h.lost.load()) return h.epoch.load();
  std::lock_guard<std::mutex> lk(g_health_mu);
  if (h.lost.load()) {
    TC_CK(cudaSetDevice(dev));
    cudaGetLastError();
    const cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess)
      throw TcError(TC_ERR_CUDA, std::string("device lost and not recoverable in this process: ") +
                                     cudaGetErrorString(e));
    h.epoch.fetch_add(1);
    h.lost.store(false);
  }
  return h.epoch.load();
}
}  // namespace

static Sim& S(tc_sim* s) {
  need(s != nullptr, "null simulator handle");
  DeviceHealth& h = health(s->s.device);
  if (h.lost.load() || h.epoch.load() != s->s.epoch)
    throw TcError(TC_ERR_CUDA, "the device of this simulator was lost (context epoch " + std::to_string(s->s.epoch) +
                                   ", now " + std::to_string(h.epoch.load()) + (h.lost.load() ? ", lost" : "") +
                                   "); create a new simulator");
  TC_CK(cudaSetDevice(s->s.device));
  return s->s;
}
// read-back guard: with the check on, non-finite positions are an error
static void check_finite(const Sim& m, const float* out, size_t count) {
  if (!m.nonfinite_check) return;
  for (size_t i = 0; i < count; ++i)
    if (!std::isfinite(out[i]))
      throw TcError(TC_ERR_NONFINITE, "non-finite position at vertex " + std::to_string(i / 3));
}

extern "C" {

const char* tc_last_error(void) { return g_err.c_str(); }

int tc_gpu_available(void) {
  int cnt = 0;
  if (cudaGetDeviceCount(&cnt) != cudaSuccess || cnt == 0) {
    cudaGetLastError();
    return 0;
  }
  for (int d = 0; d < cnt; ++d) {
    cudaDeviceProp p;
    if (cudaGetDeviceProperties(&p, d) == cudaSuccess && p.major == 10) return 1;
  }
  return 0;
}

tc_status tc_device_name(int device, char* buf, size_t len) {
  return guard([&] {
    need(buf && len > 0, "buffer required");
    cudaDeviceProp p;
    TC_CK(cudaGetDeviceProperties(&p, device));
    std::snprintf(buf, len, "%s", p.name);
  });
}

tc_status tc_create(tc_sim** out, const float* positions, uint32_t n, const uint32_t* edges, uint32_t ne,
                    const uint32_t* faces, uint32_t nf, const float* inv_masses, const uint32_t* layer_ids,
                    const float* thicknesses, uint32_t layer_id, float thickness, float tension_stiffness,
                    float compression_stiffness, float shear_stiffness, float bending_stiffness, int device) {
  return tc_create_sewn(out, positions, n, edges, ne, faces, nf, inv_masses, layer_ids, thicknesses, layer_id,
                        thickness, tension_stiffness, compression_stiffness, shear_stiffness, bending_stiffness,
                        nullptr, 0, 1.0f, 10000.0f, 1, 0.02f, device);
}
static void need_sewing(const uint32_t* sewing, uint32_t nsew, uint32_t n) {
  need(sewing != nullptr || nsew == 0, "sewing springs required");
  for (uint32_t k = 0; k < 2 * nsew; ++k) need(sewing[k] < n, "sewing springs contain an index >= number of vertices");
}
tc_status tc_create_sewn(tc_sim** out, const float* positions, uint32_t n, const uint32_t* edges, uint32_t ne,
                         const uint32_t* faces, uint32_t nf, const float* inv_masses, const uint32_t* layer_ids,
                         const float* thicknesses, uint32_t layer_id, float thickness, float tension_stiffness,
                         float compression_stiffness, float shear_stiffness, float bending_stiffness,
                         const uint32_t* sewing, uint32_t nsew, float sewing_shrink_speed, float sewing_stiffness,
                         int enable_sewing_lock, float sewing_lock_distance, int device) {
  return guard([&] {
    need(out != nullptr, "out handle required");
    *out = nullptr;
    need(positions != nullptr || n == 0, "positions required");
    need(edges != nullptr || ne == 0, "edges required");
    for (uint32_t e = 0; e < ne; ++e)
      need(edges[2 * size_t(e)] < n && edges[2 * size_t(e) + 1] < n, "edges contain an index >= number of vertices");
    for (uint32_t f = 0; f < nf; ++f)
      for (int k = 0; k < 3; ++k) need(faces[3 * size_t(f) + k] < n, "faces contain an index >= number of vertices");
    int cnt = 0;
    if (cudaGetDeviceCount(&cnt) != cudaSuccess || device < 0 || device >= cnt) {
      cudaGetLastError();
      throw TcError(TC_ERR_CUDA, "GPU initialisation failed: no CUDA device " + std::to_string(device));
    }
    tcloth::MeshInput in;
    in.pos = positions; in.n = n; in.edges = edges; in.ne = ne;
    in.faces = nf ? faces : nullptr; in.nf = nf;
    in.inv_masses = inv_masses; in.layer_ids = layer_ids; in.thicknesses = thicknesses;
    in.layer_id = layer_id; in.thickness = thickness;
    in.tension_k = tension_stiffness; in.compression_k = compression_stiffness;
    in.shear_k = shear_stiffness; in.bending_k = bending_stiffness;
    need_sewing(sewing, nsew, n);
    in.sew = sewing; in.nsew = nsew; in.sew_shrink_speed = sewing_shrink_speed;
    in.sew_stiffness = std::isnan(sewing_stiffness) ? 10000.0f : sewing_stiffness;
    in.sew_lock = enable_sewing_lock != 0;
    const uint64_t epoch = acquire_device(device);
    std::unique_ptr<tc_sim> h(new tc_sim);
    h->s.init(in, device);
    h->s.epoch = epoch;
    if (!std::isnan(sewing_lock_distance)) h->s.sew_lock_dist = std::fmax(sewing_lock_distance, 0.f);
    *out = h.release();
  });
}

// Batched instances: one simulator over the disjoint union of the instance
// meshes.  Each constraint keeps its standalone colour (Welsh-Powell order
// restricted to one instance is that instance's own order), so a batch
// colour is the union of the instances' colours and every instance evolves
// exactly as it would alone.  Each instance has its own compliances and
// primitive colliders.
tc_status tc_batch_create(tc_sim** out, uint32_t ninst, const uint32_t* vcount, const uint32_t* ecount,
                          const uint32_t* fcount, const float* positions, const uint32_t* edges, const uint32_t* faces,
                          const float* inv_masses, float thickness, const float* compliance,
                          const uint32_t* prim_count, const float* prims, int device) {
  return guard([&] {
    need(out != nullptr && ninst > 0, "at least one instance");
    need(vcount && ecount && fcount && positions && edges && compliance && prim_count, "instance arrays required");
    *out = nullptr;
    std::vector<uint32_t> voff(ninst + 1, 0);
    uint64_t NE = 0, NF = 0, NP = 0;
    for (uint32_t k = 0; k < ninst; ++k) {
      voff[k + 1] = voff[k] + vcount[k];
      NE += ecount[k]; NF += fcount[k]; NP += prim_count[k];
    }
    const uint32_t N = voff[ninst];
    std::vector<uint32_t> ge(2 * NE), gf(3 * NF);
    uint64_t eo = 0, fo = 0;
    for (uint32_t k = 0; k < ninst; ++k) {
      for (uint32_t e = 0; e < 2 * ecount[k]; ++e, ++eo) {
        need(edges[eo] < vcount[k], "edge index >= instance vertex count");
        ge[eo] = edges[eo] + voff[k];
      }
      for (uint32_t f = 0; f < 3 * fcount[k]; ++f, ++fo) {
        need(faces[fo] < vcount[k], "face index >= instance vertex count");
        gf[fo] = faces[fo] + voff[k];
      }
    }
    std::vector<uint32_t> layers(N, 0u);
    tcloth::MeshInput in;
    in.pos = positions; in.n = N; in.edges = ge.data(); in.ne = uint32_t(NE);
    in.faces = NF ? gf.data() : nullptr; in.nf = uint32_t(NF);
    in.inv_masses = inv_masses; in.layer_ids = layers.data(); in.thickness = thickness;
    in.tension_k = in.compression_k = in.shear_k = in.bending_k = 1000.f;
    const uint64_t epoch = acquire_device(device);
    std::unique_ptr<tc_sim> h(new tc_sim);
    Sim& m = h->s;
    m.init(in, device);
    m.epoch = epoch;
    m.self_collision = false;
    // per-instance compliances (tension, compression, shear, bending)
    std::vector<uint32_t> vi(N);
    for (uint32_t k = 0; k < ninst; ++k)
      for (uint32_t v = voff[k]; v < voff[k + 1]; ++v) vi[v] = k;
    for (auto& c : m.dist_h) {
      const float* cp = compliance + 4 * size_t(vi[c.v0]);
      if (c.type == 1) c.tc = c.cc = cp[2];
      else { c.tc = cp[0]; c.cc = cp[1]; }
    }
    for (auto& c : m.bend_h) {
      const float b = compliance[4 * size_t(vi[c.v2]) + 3];
      c.comp = c.pad0 > 1.5f ? std::fmax(b * 10.f, 0.5f) : b;
    }
    m.upload_dist();
    m.upload_bend();
    // per-instance primitives: 10 floats each (type, friction, restitution,
    // radius, a.xyz, b.xyz); type 0 sphere, 1 capsule, 2 plane
    m.inst_vert_off = voff;
    m.inst_prims_h.resize(ninst);
    uint32_t po = 0;
    for (uint32_t k = 0; k < ninst; ++k) {
      m.inst_prims_h[k] = make_uint2(po, prim_count[k]);
      for (uint32_t q = 0; q < prim_count[k]; ++q, ++po) {
        const float* f = prims + 10 * size_t(po);
        const uint32_t type = uint32_t(f[0]);
        need(type <= 2, "primitive type must be 0 (sphere), 1 (capsule) or 2 (plane)");
        m.prims_h.push_back(make_prim(type, f + 4, f + 7, f[3], f[1], f[2]));
      }
    }
    m.vinst.upload(vi, m.st);
    m.inst_prims.upload(m.inst_prims_h, m.st);
    m.upload_prims();
    *out = h.release();
  });
}

tc_status tc_batch_instance_offsets(tc_sim* s, uint32_t* offsets, uint32_t max_entries, uint32_t* n_instances) {
  return guard([&] {
    Sim& m = S(s);
    need(n_instances != nullptr, "n_instances required");
    const uint32_t k = m.inst_vert_off.empty() ? 1u : uint32_t(m.inst_vert_off.size() - 1);
    *n_instances = k;
    if (offsets) {
      for (uint32_t i = 0; i <= k && i < max_entries; ++i)
        offsets[i] = m.inst_vert_off.empty() ? (i == 0 ? 0u : m.n) : m.inst_vert_off[i];
    }
  });
}

tc_status tc_destroy(tc_sim* s) {
  return guard([&] {
    if (!s) return;
    cudaSetDevice(s->s.device);
    cudaStreamSynchronize(s->s.st);
    delete s;
  });
}

tc_status tc_step(tc_sim* s, float dt, uint32_t substeps, uint32_t* eff) {
  return guard([&] {
    Sim& m = S(s);
    const uint32_t sub = m.plan_frame(dt, substeps);
    m.step(dt, sub);
    if (eff) *eff = sub;
  });
}

// step_single_substep (dispatch.rs:674-688): one substep of dt_sub, no
// adaptive planning and no displacement feedback
tc_status tc_step_single_substep(tc_sim* s, float dt_sub) {
  return guard([&] {
    Sim& m = S(s);
    m.launch_frame(dt_sub, 1);
    TC_CK(cudaStreamSynchronize(m.st));
    TC_CK(cudaGetLastError());
    m.check_barrier_status();
  });
}

tc_status tc_step_async(tc_sim* s, float dt, uint32_t substeps) {
  return guard([&] {
    Sim& m = S(s);
    m.launch_frame(dt, m.plan_frame(dt, substeps));
    m.encode_feedback();
    m.async_pending = true;
  });
}

// fetch_positions (dispatch.rs:808-863): waits for the pending frame, copies
// positions and updates the displacement feedback used by auto-coupling.
tc_status tc_fetch_positions(tc_sim* s, float* out, size_t out_len, int* ok) {
  return guard([&] {
    Sim& m = S(s);
    if (ok) *ok = 0;
    if (!m.async_pending) return;
    need(out != nullptr && out_len >= size_t(m.n) * 3, "out_array too small");
    m.get_positions(out);
    m.async_pending = false;
    check_finite(m, out, size_t(m.n) * 3);
    m.check_barrier_status();
    m.consume_feedback();
    float md = 0.f;
    for (size_t i = 0; i < size_t(m.n) * 3; ++i) md = std::fmax(md, std::fabs(out[i] - m.prev_frame_pos[i]));
    std::memcpy(m.prev_frame_pos.data(), out, size_t(m.n) * 3 * sizeof(float));
    m.last_max_disp = md;
    if (ok) *ok = 1;
  });
}

// step_buffered (dispatch.rs:1293-1340): one frame, its positions into the
// next slot of the device ring (the last slot once 8 are held); no wait
tc_status tc_step_buffered(tc_sim* s, float dt, uint32_t substeps, uint32_t* count) {
  return guard([&] {
    Sim& m = S(s);
    const uint32_t c = m.step_buffered(dt, m.plan_frame(dt, substeps));
    if (count) *count = c;
  });
}
tc_status tc_get_buffered_frame_count(tc_sim* s, uint32_t* count) {
  return guard([&] { need(count != nullptr, "count required"); *count = S(s).buffered; });
}
tc_status tc_clear_frame_buffer(tc_sim* s) {
  return guard([&] { S(s).buffered = 0; });
}
// fetch_buffered_positions (dispatch.rs:1349-1403): every buffered frame
// (frames x n x 3 floats, as much as fits in out), then the feedback of the
// last frame and an empty ring.
tc_status tc_fetch_buffered_positions(tc_sim* s, float* out, size_t out_len, uint32_t* count) {
  return guard([&] {
    Sim& m = S(s);
    need(count != nullptr, "count required");
    *count = 0;
    const uint32_t c = m.buffered;
    if (c == 0 || m.n == 0) return;
    need(out != nullptr || out_len == 0, "output required");
    const size_t nv3 = size_t(m.n) * 3, total = size_t(c) * nv3, len = std::min(out_len, total);
    if (len) TC_CK(cudaMemcpyAsync(out, m.ring.p, len * sizeof(float), cudaMemcpyDeviceToHost, m.st));
    TC_CK(cudaStreamSynchronize(m.st));
    TC_CK(cudaGetLastError());
    m.check_barrier_status();
    m.consume_feedback();
    if (len == total) {
      const float* last = out + (size_t(c) - 1) * nv3;
      float md = 0.f;
      for (size_t i = 0; i < nv3; ++i) md = std::fmax(md, std::fabs(last[i] - m.prev_frame_pos[i]));
      std::memcpy(m.prev_frame_pos.data(), last, nv3 * sizeof(float));
      m.last_max_disp = md;
    }
    m.buffered = 0;
    *count = c;
    check_finite(m, out, len);
  });
}

tc_status tc_get_positions(tc_sim* s, float* out, size_t out_len) {
  return guard([&] {
    Sim& m = S(s);
    need(out != nullptr && out_len >= size_t(m.n) * 3, "output array too small");
    m.get_positions(out);
    check_finite(m, out, size_t(m.n) * 3);
  });
}

tc_status tc_mark_device_lost(int device) {
  return guard([&] { health(device).lost.store(true); });
}
tc_status tc_device_status(int device, int* lost, uint64_t* epoch) {
  return guard([&] {
    DeviceHealth& h = health(device);
    if (lost) *lost = h.lost.load() ? 1 : 0;
    if (epoch) *epoch = h.epoch.load();
  });
}
tc_status tc_set_nonfinite_check(tc_sim* s, int enable) {
  return guard([&] { S(s).nonfinite_check = enable != 0; });
}

tc_status tc_set_positions_and_velocities(tc_sim* s, const float* pos, const float* vel, uint32_t n) {
  return guard([&] {
    Sim& m = S(s);
    if (m.n == 0 || n != m.n || !pos) return;  // the reference ignores a length mismatch
    std::vector<float> w(m.n);
    for (uint32_t i = 0; i < m.n; ++i) {
      auto it = m.pins.find(i);
      w[i] = it != m.pins.end() ? m.orig_w[i] * (1.f - Sim::clamp_w(it->second.weight)) : m.orig_w[i];
    }
    m.upload_vertices(pos, vel, w.data());
  });
}

tc_status tc_reset(tc_sim* s) {
  return guard([&] {
    Sim& m = S(s);
    m.pins.clear();
    m.upload_pins();
    m.upload_vertices(m.init_pos.data(), nullptr, m.init_w.data());
    for (uint32_t i = 0; i < m.nd; ++i) m.dist_h[i].rest = m.base_rest[i];
    std::fill(m.mult.begin(), m.mult.end(), 1.f);
    m.apply_distance_compliances();
    TC_CK(cudaMemsetAsync(m.acc.p, 0, size_t(m.n) * tcloth::A_N * sizeof(int32_t), m.st));
    m.buffered = 0;         // dispatch.rs:1425
    m.pri.latched = false;  // sewing priority restarts (dispatch.rs:1414-1417)
    m.pri.frame = 0;
    m.pri.ramp_t = 0.f;
    m.pri.ratio = 0.f;
    m.mark();
    TC_CK(cudaStreamSynchronize(m.st));
  });
}

// ---- edge colliders (simulation/mod.rs:1007-1025, lib.rs:2736-2749)
tc_status tc_set_enable_edge_collision(tc_sim* s, int enable) {
  return guard([&] { Sim& m = S(s); m.edge_collision = enable != 0; m.mark(); });
}
tc_status tc_set_edge_margin_scale(tc_sim* s, float scale) {
  return guard([&] { Sim& m = S(s); m.edge_mscale = std::fmax(scale, 1.f); m.mark(); });
}
tc_status tc_set_edge_margin_offset(tc_sim* s, float offset) {
  return guard([&] { Sim& m = S(s); m.edge_moff = std::fmax(offset, 0.f); m.mark(); });
}
tc_status tc_get_num_collider_edges(tc_sim* s, uint32_t* count) {
  return guard([&] {
    need(count != nullptr, "count required");
    Sim& m = S(s);
    m.ensure_collider_edges();
    *count = uint32_t(m.cedges_h.size());
  });
}

// ---- sewing settings (simulation/mod.rs:1211-1420, lib.rs:2798-2925)
tc_status tc_get_num_sewing_constraints(tc_sim* s, uint32_t* count) {
  return guard([&] { need(count != nullptr, "count required"); *count = S(s).nsw; });
}
tc_status tc_set_sewing_stiffness(tc_sim* s, float stiffness) {
  return guard([&] { Sim& m = S(s); m.sew_stiffness = std::fmax(stiffness, 1.f); m.mark(); });
}
tc_status tc_set_sewing_shrink_speed(tc_sim* s, float speed) {
  return guard([&] {
    Sim& m = S(s);
    m.sew_speed = std::isfinite(speed) ? std::fmax(speed, 0.f) : 1.f;
    m.mark();
  });
}
tc_status tc_get_sewing_shrink_speed(tc_sim* s, float* speed) {
  return guard([&] { need(speed != nullptr, "speed required"); *speed = S(s).sew_speed; });
}
tc_status tc_set_enable_sewing_lock(tc_sim* s, int enabled) {
  return guard([&] { Sim& m = S(s); m.sew_lock = enabled != 0; m.mark(); });
}
tc_status tc_set_sewing_lock_distance(tc_sim* s, float distance) {
  return guard([&] { Sim& m = S(s); m.sew_lock_dist = std::fmax(distance, 0.f); m.mark(); });
}
tc_status tc_get_sewing_lock_distance(tc_sim* s, float* distance) {
  return guard([&] { need(distance != nullptr, "distance required"); *distance = S(s).sew_lock_dist; });
}
tc_status tc_get_sewing_current_rest_lengths(tc_sim* s, float* out, size_t len) {
  return guard([&] {
    Sim& m = S(s);
    need(out != nullptr || m.nsw == 0, "output required");
    need(len >= m.nsw, "output array too small");
    std::vector<float2> r(m.nsw);
    if (m.nsw) TC_CK(cudaMemcpyAsync(r.data(), m.sew_rest.p, m.nsw * sizeof(float2), cudaMemcpyDeviceToHost, m.st));
    TC_CK(cudaStreamSynchronize(m.st));
    for (uint32_t i = 0; i < m.nsw; ++i) out[i] = r[i].x;
  });
}
tc_status tc_set_sewing_current_rest_lengths(tc_sim* s, const float* values, size_t len) {
  return guard([&] {
    Sim& m = S(s);
    if (values == nullptr || len != m.nsw || len == 0) return;  // ignored, as the reference does (dispatch.rs:928-932)
    std::vector<float2> r(m.nsw);
    TC_CK(cudaMemcpyAsync(r.data(), m.sew_rest.p, m.nsw * sizeof(float2), cudaMemcpyDeviceToHost, m.st));
    TC_CK(cudaStreamSynchronize(m.st));
    for (uint32_t i = 0; i < m.nsw; ++i) r[i].x = values[i];
    TC_CK(cudaMemcpyAsync(m.sew_rest.p, r.data(), m.nsw * sizeof(float2), cudaMemcpyHostToDevice, m.st));
    TC_CK(cudaStreamSynchronize(m.st));
  });
}
tc_status tc_set_sewing_priority_options(tc_sim* s, int enabled, float threshold, float merge_dist,
                                         uint32_t ramp_frames, uint32_t max_frames) {
  return guard([&] {
    Sim& m = S(s);
    auto& p = m.pri;
    const float th = std::fmin(std::fmax(threshold, 0.f), 1.f), md = std::fmin(std::fmax(merge_dist, 0.0005f), 0.1f);
    const uint32_t rf = std::min(ramp_frames, 120u), mf = std::min(max_frames, 100000u);
    if (p.enabled == (enabled != 0) && p.threshold == th && p.merge == md && p.ramp_frames == rf && p.max_frames == mf)
      return;  // unchanged: the latch is kept
    p.enabled = enabled != 0; p.threshold = th; p.merge = md; p.ramp_frames = rf; p.max_frames = mf;
    p.latched = false; p.frame = 0; p.ramp_t = 0.f; p.ratio = 0.f;
    m.mark();
  });
}
tc_status tc_set_sewing_priority_state(tc_sim* s, int latched, uint32_t frame, float ramp_t, float ratio) {
  return guard([&] {
    Sim& m = S(s);
    m.pri.latched = latched != 0;
    m.pri.frame = frame;
    m.pri.ramp_t = std::fmin(std::fmax(ramp_t, 0.f), 1.f);
    m.pri.ratio = std::fmin(std::fmax(ratio, 0.f), 1.f);
    m.mark();
  });
}
// update_sewing_priority_from_positions (mod.rs:1323-1356): the share of
// sewing pairs within merge_dist in `positions` (host data, no readback),
// then the one-way latch and the ramp.  out = (ratio, gravity scale, latched).
tc_status tc_update_sewing_priority(tc_sim* s, const float* positions, uint32_t n, float out[3]) {
  return guard([&] {
    Sim& m = S(s);
    need(out != nullptr, "out required");
    auto& p = m.pri;
    if (!p.enabled || m.nsw == 0) { out[0] = 1.f; out[1] = 1.f; out[2] = 1.f; return; }
    need(positions != nullptr || n == 0, "positions required");
    const float msq = p.merge * p.merge;
    size_t closed = 0, total = 0;
    for (const auto& c : m.sew_h) {
      if (c.v0 >= n || c.v1 >= n) continue;
      ++total;
      const float* a = positions + 3 * size_t(c.v0);
      const float* b = positions + 3 * size_t(c.v1);
      const float dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
      if (dx * dx + dy * dy + dz * dz <= msq) ++closed;
    }
    const float ratio = total ? float(closed) / float(total) : 1.f;
    p.ratio = ratio;
    p.frame = p.frame == UINT32_MAX ? p.frame : p.frame + 1;
    if (!p.latched && (ratio >= p.threshold || (p.max_frames > 0 && p.frame >= p.max_frames))) p.latched = true;
    if (p.latched && p.ramp_frames > 0) p.ramp_t = std::fmin(p.ramp_t + 1.0f / float(p.ramp_frames), 1.0f);
    else if (p.latched) p.ramp_t = 1.f;
    else p.ramp_t = 0.f;
    m.mark();
    out[0] = ratio; out[1] = m.priority_scale(); out[2] = p.latched ? 1.f : 0.f;
  });
}
// (gravity scale, last closure ratio, priority active = gravity held, latched)
tc_status tc_get_sewing_priority(tc_sim* s, float out[4]) {
  return guard([&] {
    Sim& m = S(s);
    need(out != nullptr, "out required");
    const bool on = m.pri.enabled && m.nsw > 0;
    out[0] = m.priority_scale();
    out[1] = on ? m.pri.ratio : 1.f;
    out[2] = on && !m.pri.latched ? 1.f : 0.f;
    out[3] = m.pri.latched ? 1.f : 0.f;
  });
}

tc_status tc_set_gravity(tc_sim* s, float gx, float gy, float gz) {
  return guard([&] { Sim& m = S(s); m.g[0] = gx; m.g[1] = gy; m.g[2] = gz; m.mark(); });
}
tc_status tc_set_damping(tc_sim* s, float d) {
  return guard([&] { Sim& m = S(s); m.damping = std::fmax(d, 0.f); m.mark(); });
}
tc_status tc_set_damping_all(tc_sim* s, float t, float c, float sh, float b) {
  return guard([&] {
    Sim& m = S(s);
    m.td = std::fmax(t, 0.f); m.cd = std::fmax(c, 0.f); m.sd = std::fmax(sh, 0.f); m.bd = std::fmax(b, 0.f);
    m.mark();
  });
}
tc_status tc_set_solver_iterations(tc_sim* s, uint32_t it) {
  return guard([&] { Sim& m = S(s); m.iters = std::max(it, 1u); m.mark(); });
}
// set_stiffness_all (simulation/mod.rs:1106-1170)
tc_status tc_set_stiffness_all(tc_sim* s, float t, float c, float sh, float b) {
  return guard([&] {
    Sim& m = S(s);
    m.base_tc = tcloth::stiffness_to_compliance(t);
    m.base_cc = tcloth::stiffness_to_compliance(c);
    m.base_shc = tcloth::stiffness_to_compliance(sh);
    m.base_bk = b > 0.f ? b : 0.f;
    m.apply_distance_compliances();
    const float bc = b > 0.f ? 1.f / b : 1e10f;
    for (auto& q : m.bend_h) q.comp = q.pad0 > 1.5f ? std::fmax(bc * 10.f, 0.5f) : bc;
    m.upload_bend();
    m.mark();
  });
}
tc_status tc_set_compliance_all(tc_sim* s, float t, float c, float sh, float b) {
  return guard([&] {
    Sim& m = S(s);
    m.base_tc = t; m.base_cc = c; m.base_shc = sh;
    for (auto& q : m.dist_h) {
      if (q.type == 1) q.tc = q.cc = sh;
      else { q.tc = t; q.cc = c; }
    }
    m.upload_dist();
    for (auto& q : m.bend_h) q.comp = q.pad0 > 1.5f ? std::fmax(b * 10.f, 0.5f) : b;
    m.upload_bend();
    m.mark();
  });
}
// set_edge_stiffness_multipliers (simulation/mod.rs:1494-1525)
tc_status tc_set_edge_stiffness_multipliers(tc_sim* s, const uint32_t* idx, const float* ml, uint32_t count) {
  return guard([&] {
    Sim& m = S(s);
    bool changed = false;
    for (uint32_t i = 0; i < count; ++i) {
      const uint32_t e = idx[i];
      if (e >= m.orig_edge_to_dist.size()) continue;
      const int64_t ci = m.orig_edge_to_dist[e];
      if (ci < 0) continue;
      const float v = std::isfinite(ml[i]) ? std::fmax(ml[i], 1e-3f) : 1.f;
      if (std::fabs(m.mult[size_t(ci)] - v) > 1e-6f) { m.mult[size_t(ci)] = v; changed = true; }
    }
    if (changed) m.apply_distance_compliances();
  });
}
// reset_edge_stiffness_multipliers (simulation/mod.rs:1526-1532)
tc_status tc_reset_edge_stiffness_multipliers(tc_sim* s) {
  return guard([&] {
    Sim& m = S(s);
    bool all_one = true;
    for (float v : m.mult) all_one = all_one && std::fabs(v - 1.f) <= 1e-6f;
    if (all_one) return;
    std::fill(m.mult.begin(), m.mult.end(), 1.f);
    m.apply_distance_compliances();
  });
}
// set_edge_rest_length_scales / reset_edge_rest_lengths (simulation/mod.rs:1450-1491):
// rest = initial rest x max(scale, 0.01) for each listed input edge
tc_status tc_set_edge_rest_length_scales(tc_sim* s, const uint32_t* idx, const float* scales, uint32_t count) {
  return guard([&] {
    need(count == 0 || (idx != nullptr && scales != nullptr), "indices and scales required");
    Sim& m = S(s);
    bool changed = false;
    for (uint32_t i = 0; i < count; ++i) {
      const uint32_t e = idx[i];
      if (e >= m.orig_edge_to_dist.size()) continue;
      const int64_t ci = m.orig_edge_to_dist[e];
      if (ci < 0 || size_t(ci) >= m.dist_h.size()) continue;
      m.dist_h[size_t(ci)].rest = m.base_rest[size_t(ci)] * std::fmax(scales[i], 0.01f);
      changed = true;
    }
    if (changed && m.nd) { m.upload_dist(); m.mark(); }
  });
}
tc_status tc_reset_edge_rest_lengths(tc_sim* s) {
  return guard([&] {
    Sim& m = S(s);
    for (uint32_t i = 0; i < m.nd; ++i) m.dist_h[i].rest = m.base_rest[i];
    if (m.nd) { m.upload_dist(); m.mark(); }
  });
}
// get_edge_rest_length / get_edge_initial_rest_length / get_edge_tension_compliance
// (simulation/mod.rs:1535-1568): the distance constraint of an input edge,
// 0 for an edge without one; out = (rest, initial rest, tension compliance)
tc_status tc_get_edge_constraint(tc_sim* s, uint32_t edge_idx, float out[3]) {
  return guard([&] {
    need(out != nullptr, "out required");
    Sim& m = S(s);
    out[0] = out[1] = out[2] = 0.f;
    if (edge_idx >= m.orig_edge_to_dist.size()) return;
    const int64_t ci = m.orig_edge_to_dist[edge_idx];
    if (ci < 0 || size_t(ci) >= m.dist_h.size()) return;
    out[0] = m.dist_h[size_t(ci)].rest;
    out[1] = m.base_rest[size_t(ci)];
    out[2] = m.dist_h[size_t(ci)].tc;
  });
}
tc_status tc_set_enable_self_collision(tc_sim* s, int on) {
  return guard([&] { Sim& m = S(s); m.self_collision = on != 0; m.mark(); });
}
tc_status tc_set_self_collision_options(tc_sim* s, float relief, float ratio, int excl, int untangle, uint32_t maxit) {
  return guard([&] {
    Sim& m = S(s);
    m.relief = relief; m.max_disp_ratio = ratio; m.enable_relief = relief < 0.999f;
    m.exclude_neighbors = excl != 0; m.untangle_opt = untangle != 0; m.max_search = maxit;
    m.mark();
  });
}
tc_status tc_set_enable_pair_cache(tc_sim* s, int enable) {
  return guard([&] { S(s).set_pair_cache(enable != 0); });
}
tc_status tc_get_enable_pair_cache(tc_sim* s, int* enabled) {
  return guard([&] { need(enabled != nullptr, "enabled required"); *enabled = S(s).pair_cache ? 1 : 0; });
}
tc_status tc_set_self_collision_algorithm(tc_sim* s, uint32_t algo) {
  return guard([&] {
    need(algo <= 1u, "self-collision algorithm 2 (virtual-particle vertex-vertex) is not built");
    Sim& m = S(s);
    m.set_pair_cache(algo == 1u);
    m.sc_algorithm = algo;
  });
}
tc_status tc_get_self_collision_algorithm(tc_sim* s, uint32_t* algo) {
  return guard([&] { need(algo != nullptr, "algo required"); *algo = S(s).sc_algorithm; });
}
tc_status tc_set_pair_cache_options(tc_sim* s, uint32_t max_vt_pairs, uint32_t max_ee_pairs, uint32_t margin_mode,
                                    float safety_margin, float horizon_scale, float max_horizon) {
  return guard([&] {
    Sim& m = S(s);
    m.pair_max_vt = std::min(std::max(max_vt_pairs, 64u), 262144u);
    m.pair_max_ee = std::min(std::max(max_ee_pairs, 64u), 262144u);
    m.pair_qvt = Sim::quota_for_budget(m.pair_max_vt, m.n);
    m.pair_qee = Sim::quota_for_budget(m.pair_max_ee, m.n);
    m.pair_margin_mode = margin_mode == 0 ? 0u : 1u;
    m.pair_safety = std::min(std::max(safety_margin, 0.f), 0.05f);
    m.pair_hscale = std::min(std::max(horizon_scale, 0.f), 4.f);
    m.pair_max_h = std::min(std::max(max_horizon, 0.f), 0.1f);
    m.mark();
  });
}
tc_status tc_set_enable_pair_cache_final_fallback(tc_sim* s, int enable) {
  return guard([&] { Sim& m = S(s); m.pair_final_fallback = enable != 0; m.mark(); });
}
tc_status tc_get_enable_pair_cache_final_fallback(tc_sim* s, int* enabled) {
  return guard([&] { need(enabled != nullptr, "enabled required"); *enabled = S(s).pair_final_fallback ? 1 : 0; });
}
tc_status tc_get_pair_cache_stats(tc_sim* s, uint32_t out[4]) {
  return guard([&] {
    need(out != nullptr, "out required");
    Sim& m = S(s);
    uint32_t c[4] = {0u, 0u, 0u, 0u};
    if (m.pair_cnt.p) {
      TC_CK(cudaMemcpyAsync(c, m.pair_cnt.p, sizeof c, cudaMemcpyDeviceToHost, m.st));
      TC_CK(cudaStreamSynchronize(m.st));
    }
    out[0] = c[0]; out[1] = c[1]; out[2] = m.pair_max_vt; out[3] = m.pair_max_ee;
  });
}
tc_status tc_get_active_pairs(tc_sim* s, uint32_t counts[4], uint32_t* vt_pairs, size_t vt_cap, uint32_t* ee_pairs,
                              size_t ee_cap) {
  return guard([&] {
    need(counts != nullptr, "counts required");
    Sim& m = S(s);
    counts[0] = counts[1] = counts[2] = counts[3] = 0u;
    if (!m.pair_cnt.p) return;
    uint32_t c[4];
    TC_CK(cudaMemcpyAsync(c, m.pair_cnt.p, sizeof c, cudaMemcpyDeviceToHost, m.st));
    const size_t nvt = size_t(m.n) * m.pair_qvt, nee = size_t(m.n) * m.pair_qee;
    std::vector<uint4> hv(nvt), he(nee);
    if (nvt) TC_CK(cudaMemcpyAsync(hv.data(), m.pair_vt.p, nvt * sizeof(uint4), cudaMemcpyDeviceToHost, m.st));
    if (nee) TC_CK(cudaMemcpyAsync(he.data(), m.pair_ee.p, nee * sizeof(uint4), cudaMemcpyDeviceToHost, m.st));
    TC_CK(cudaStreamSynchronize(m.st));
    counts[0] = c[0];
    counts[1] = c[1];
    auto take = [](const std::vector<uint4>& src, uint32_t* dst, size_t cap) {
      uint32_t k = 0;
      for (const uint4& q : src) {
        if (q.x == tcloth::kPairSentinel) continue;
        if (dst && k < cap) { dst[4 * size_t(k)] = q.x; dst[4 * size_t(k) + 1] = q.y; dst[4 * size_t(k) + 2] = q.z; dst[4 * size_t(k) + 3] = q.w; }
        ++k;
      }
      return k;
    };
    counts[2] = take(hv, vt_pairs, vt_cap);
    counts[3] = take(he, ee_pairs, ee_cap);
  });
}
tc_status tc_set_coupled_collider(tc_sim* s, int on) {
  return guard([&] { Sim& m = S(s); m.coupled = on != 0; m.mark(); });
}
tc_status tc_set_auto_coupled_on_low_substeps(tc_sim* s, int on) {
  return guard([&] { Sim& m = S(s); m.auto_coupled = on != 0; m.mark(); });
}
tc_status tc_set_collider_options(tc_sim* s, int cluster, int recovery, float sweep) {
  return guard([&] {
    Sim& m = S(s);
    (void)cluster;  // the exact broadphase makes cluster culling unnecessary
    (void)sweep;
    m.recovery = recovery != 0;
    m.mark();
  });
}

tc_status tc_add_sphere_collider(tc_sim* s, const float c[3], float r, float f, float rest) {
  return guard([&] { Sim& m = S(s); need(c, "center required"); m.prims_h.push_back(make_prim(0, c, nullptr, r, f, rest)); m.upload_prims(); });
}
tc_status tc_add_capsule_collider(tc_sim* s, const float a[3], const float b[3], float r, float f, float rest) {
  return guard([&] { Sim& m = S(s); need(a && b, "points required"); m.prims_h.push_back(make_prim(1, a, b, r, f, rest)); m.upload_prims(); });
}
tc_status tc_add_plane_collider(tc_sim* s, const float p[3], const float nrm[3], float f, float rest) {
  return guard([&] { Sim& m = S(s); need(p && nrm, "point and normal required"); m.prims_h.push_back(make_prim(2, p, nrm, 0.f, f, rest)); m.upload_prims(); });
}
tc_status tc_set_mesh_collider_triangles(tc_sim* s, const float* t, uint32_t T, float f, float th, float r, int single,
                                         const float* attr) {
  return guard([&] {
    Sim& m = S(s);
    need(t != nullptr || T == 0, "triangles required");
    m.set_mesh(t, T, f, th, r, single != 0, attr);
  });
}
tc_status tc_clear_colliders(tc_sim* s) {
  return guard([&] {
    Sim& m = S(s);
    m.prims_h.clear();
    m.tris_h.clear();
    m.tris_h_valid = true;
    m.ntris = 0;
    m.graph_ntris = 0;
    m.ce_stale = true;  // no triangles: no collider edges (mod.rs:2731-2736)
    m.mark();
  });
}

tc_status tc_set_pin(tc_sim* s, uint32_t v, const float target[3], float w) {
  return guard([&] {
    Sim& m = S(s);
    if (v >= m.n) return;  // the reference ignores out-of-range pins
    need(target != nullptr, "target required");
    m.pins[v] = tcloth::PinH{{target[0], target[1], target[2]}, w};
    m.upload_pins();
    m.write_inv_mass(v, m.orig_w[v] * (1.f - Sim::clamp_w(w)));
  });
}
tc_status tc_set_pins_batch(tc_sim* s, const uint32_t* idx, const float* targets, const float* weights, uint32_t count) {
  return guard([&] {
    Sim& m = S(s);
    for (uint32_t i = 0; i < count; ++i) {
      const uint32_t v = idx[i];
      if (v >= m.n) continue;
      m.pins[v] = tcloth::PinH{{targets[3 * i], targets[3 * i + 1], targets[3 * i + 2]}, weights[i]};
      m.write_inv_mass(v, m.orig_w[v] * (1.f - Sim::clamp_w(weights[i])));
    }
    m.upload_pins();
  });
}
tc_status tc_release_pin(tc_sim* s, uint32_t v) {
  return guard([&] {
    Sim& m = S(s);
    if (m.pins.erase(v)) {
      m.upload_pins();
      m.write_inv_mass(v, m.orig_w[v]);
    }
  });
}
tc_status tc_clear_pins(tc_sim* s) {
  return guard([&] {
    Sim& m = S(s);
    for (const auto& kv : m.pins) m.write_inv_mass(kv.first, m.orig_w[kv.first]);
    m.pins.clear();
    m.upload_pins();
  });
}
tc_status tc_set_vertex_inv_masses(tc_sim* s, const uint32_t* idx, const float* w, uint32_t count) {
  return guard([&] {
    Sim& m = S(s);
    for (uint32_t i = 0; i < count; ++i) {
      const uint32_t v = idx[i];
      if (v >= m.n) continue;
      m.orig_w[v] = w[i];
      auto it = m.pins.find(v);
      m.write_inv_mass(v, it != m.pins.end() ? w[i] * (1.f - Sim::clamp_w(it->second.weight)) : w[i]);
    }
    m.mark();
  });
}
tc_status tc_get_vertex_inv_masses(tc_sim* s, float* out, uint32_t n) {
  return guard([&] {
    Sim& m = S(s);
    need(out && n >= m.n, "output too small");
    std::copy(m.orig_w.begin(), m.orig_w.end(), out);
  });
}

tc_status tc_get_counts(tc_sim* s, uint32_t out[8]) {
  return guard([&] {
    Sim& m = S(s);
    out[0] = m.n; out[1] = m.nd; out[2] = m.nb; out[3] = m.ne;
    out[4] = uint32_t(m.m.dist_cnt.size()); out[5] = uint32_t(m.m.bend_cnt.size());
    out[6] = m.m.table; out[7] = m.m.multi_layer ? 1u : 0u;
  });
}
tc_status tc_get_num_virtual_vertices(tc_sim* s, uint32_t* count) {
  return guard([&] { need(count != nullptr, "count required"); *count = S(s).m.num_virtual; });
}
tc_status tc_get_cell_size(tc_sim* s, float* cell) {
  return guard([&] { Sim& m = S(s); *cell = m.m.cell; });
}

tc_status tc_get_state(tc_sim* s, float* x, float* p, float* v) {
  return guard([&] {
    Sim& m = S(s);
    std::vector<float4> hx(m.n), hp(m.n), hv(m.n);
    TC_CK(cudaMemcpyAsync(hx.data(), m.x4.p, m.n * sizeof(float4), cudaMemcpyDeviceToHost, m.st));
    TC_CK(cudaMemcpyAsync(hp.data(), m.p4.p, m.n * sizeof(float4), cudaMemcpyDeviceToHost, m.st));
    TC_CK(cudaMemcpyAsync(hv.data(), m.v4.p, m.n * sizeof(float4), cudaMemcpyDeviceToHost, m.st));
    TC_CK(cudaStreamSynchronize(m.st));
    for (uint32_t i = 0; i < m.n; ++i) {
      if (x) { x[3 * i] = hx[i].x; x[3 * i + 1] = hx[i].y; x[3 * i + 2] = hx[i].z; }
      if (p) { p[3 * i] = hp[i].x; p[3 * i + 1] = hp[i].y; p[3 * i + 2] = hp[i].z; }
      if (v) { v[3 * i] = hv[i].x; v[3 * i + 1] = hv[i].y; v[3 * i + 2] = hv[i].z; }
    }
  });
}
tc_status tc_get_distance_constraints(tc_sim* s, uint32_t* v01, float* par, uint32_t* off, uint32_t* cnt) {
  return guard([&] {
    Sim& m = S(s);
    for (uint32_t i = 0; i < m.nd; ++i) {
      const auto& c = m.dist_h[i];
      if (v01) { v01[2 * i] = c.v0; v01[2 * i + 1] = c.v1; }
      if (par) { par[4 * i] = c.rest; par[4 * i + 1] = c.tc; par[4 * i + 2] = c.cc; par[4 * i + 3] = float(c.type); }
    }
    if (off) std::copy(m.m.dist_off.begin(), m.m.dist_off.end(), off);
    if (cnt) std::copy(m.m.dist_cnt.begin(), m.m.dist_cnt.end(), cnt);
  });
}
tc_status tc_get_bending_constraints(tc_sim* s, uint32_t* v, float* par, uint32_t* off, uint32_t* cnt) {
  return guard([&] {
    Sim& m = S(s);
    for (uint32_t i = 0; i < m.nb; ++i) {
      const auto& c = m.bend_h[i];
      if (v) { v[4 * i] = c.v0; v[4 * i + 1] = c.v1; v[4 * i + 2] = c.v2; v[4 * i + 3] = c.v3; }
      if (par) { par[4 * i] = c.rest; par[4 * i + 1] = c.comp; par[4 * i + 2] = c.pad0; par[4 * i + 3] = c.pad1; }
    }
    if (off) std::copy(m.m.bend_off.begin(), m.m.bend_off.end(), off);
    if (cnt) std::copy(m.m.bend_cnt.begin(), m.m.bend_cnt.end(), cnt);
  });
}
tc_status tc_get_hash_state(tc_sim* s, int which, uint32_t* cell_starts, uint32_t* sorted) {
  return guard([&] {
    Sim& m = S(s);
    need(which == 0 || which == 1, "which must be 0 (vertices) or 1 (edges)");
    m.encode_hash(which);
    const uint32_t cnt = which == 0 ? m.n : m.ne;
    TC_CK(cudaMemcpyAsync(cell_starts, which == 0 ? m.cs.p : m.ecs.p, (m.m.table + 1) * sizeof(uint32_t),
                          cudaMemcpyDeviceToHost, m.st));
    if (cnt)
      TC_CK(cudaMemcpyAsync(sorted, which == 0 ? m.srt.p : m.esrt.p, cnt * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                            m.st));
    TC_CK(cudaStreamSynchronize(m.st));
    TC_CK(cudaGetLastError());
  });
}
tc_status tc_get_edges(tc_sim* s, uint32_t* e, uint32_t* bits) {
  return guard([&] {
    Sim& m = S(s);
    if (e) std::copy(m.m.edges.begin(), m.m.edges.end(), e);
    if (bits) std::copy(m.m.edge_bits.begin(), m.m.edge_bits.end(), bits);
  });
}
tc_status tc_set_residual_tracking(tc_sim* s, int on) {
  return guard([&] { Sim& m = S(s); m.track_residual = on != 0; m.mark(); });
}
tc_status tc_get_residuals(tc_sim* s, float* drms, float* dmax, float* brms, float* bmax, float totals[4]) {
  return guard([&] {
    Sim& m = S(s);
    const size_t kd = m.m.dist_cnt.size(), kb = m.m.bend_cnt.size();
    std::vector<float> sum(kd + kb + 1), mx(kd + kb + 1);
    TC_CK(cudaMemcpyAsync(sum.data(), m.res_sum.p, sum.size() * 4, cudaMemcpyDeviceToHost, m.st));
    TC_CK(cudaMemcpyAsync(mx.data(), m.res_max.p, mx.size() * 4, cudaMemcpyDeviceToHost, m.st));
    TC_CK(cudaStreamSynchronize(m.st));
    double ds = 0, bs = 0;
    float dm = 0, bm = 0;
    for (size_t c = 0; c < kd; ++c) {
      if (drms) drms[c] = m.m.dist_cnt[c] ? std::sqrt(sum[c] / float(m.m.dist_cnt[c])) : 0.f;
      if (dmax) dmax[c] = mx[c];
      ds += sum[c]; dm = std::fmax(dm, mx[c]);
    }
    for (size_t c = 0; c < kb; ++c) {
      if (brms) brms[c] = m.m.bend_cnt[c] ? std::sqrt(sum[kd + c] / float(m.m.bend_cnt[c])) : 0.f;
      if (bmax) bmax[c] = mx[kd + c];
      bs += sum[kd + c]; bm = std::fmax(bm, mx[kd + c]);
    }
    if (totals) {
      totals[0] = m.nd ? float(std::sqrt(ds / m.nd)) : 0.f;
      totals[1] = dm;
      totals[2] = m.nb ? float(std::sqrt(bs / m.nb)) : 0.f;
      totals[3] = bm;
    }
  });
}
tc_status tc_get_predicted_residual(tc_sim* s, float* rms) {
  return guard([&] {
    Sim& m = S(s);
    need(rms != nullptr, "rms required");
    float sum = 0.f;
    TC_CK(cudaMemcpyAsync(&sum, m.res_sum.p + m.m.dist_cnt.size() + m.m.bend_cnt.size(), sizeof(float),
                          cudaMemcpyDeviceToHost, m.st));
    TC_CK(cudaStreamSynchronize(m.st));
    *rms = m.nd + m.nb ? float(std::sqrt(double(sum) / double(m.nd + m.nb))) : 0.f;
  });
}
struct tc_mesh {
  tcloth::MeshData m;
};

tc_status tc_mesh_build(tc_mesh** out, const float* positions, uint32_t n, const uint32_t* edges, uint32_t ne,
                        const uint32_t* faces, uint32_t nf, const float* inv_masses, const uint32_t* layer_ids,
                        const float* thicknesses, uint32_t layer_id, float thickness, float tk, float ck, float sk,
                        float bk) {
  return tc_mesh_build_sewn(out, positions, n, edges, ne, faces, nf, inv_masses, layer_ids, thicknesses, layer_id,
                            thickness, tk, ck, sk, bk, nullptr, 0, 1.0f, 10000.0f, 1);
}
tc_status tc_mesh_build_sewn(tc_mesh** out, const float* positions, uint32_t n, const uint32_t* edges, uint32_t ne,
                             const uint32_t* faces, uint32_t nf, const float* inv_masses, const uint32_t* layer_ids,
                             const float* thicknesses, uint32_t layer_id, float thickness, float tk, float ck,
                             float sk, float bk, const uint32_t* sewing, uint32_t nsew, float sewing_shrink_speed,
                             float sewing_stiffness, int enable_sewing_lock) {
  return guard([&] {
    need(out != nullptr, "out handle required");
    *out = nullptr;
    for (uint32_t e = 0; e < ne; ++e)
      need(edges[2 * size_t(e)] < n && edges[2 * size_t(e) + 1] < n, "edges contain an index >= number of vertices");
    for (uint32_t f = 0; f < nf; ++f)
      for (int k = 0; k < 3; ++k) need(faces[3 * size_t(f) + k] < n, "faces contain an index >= number of vertices");
    tcloth::MeshInput in;
    in.pos = positions; in.n = n; in.edges = edges; in.ne = ne; in.faces = nf ? faces : nullptr; in.nf = nf;
    in.inv_masses = inv_masses; in.layer_ids = layer_ids; in.thicknesses = thicknesses;
    in.layer_id = layer_id; in.thickness = thickness;
    in.tension_k = tk; in.compression_k = ck; in.shear_k = sk; in.bending_k = bk;
    need_sewing(sewing, nsew, n);
    in.sew = sewing; in.nsew = nsew; in.sew_shrink_speed = sewing_shrink_speed;
    in.sew_stiffness = std::isnan(sewing_stiffness) ? 10000.0f : sewing_stiffness;
    in.sew_lock = enable_sewing_lock != 0;
    std::unique_ptr<tc_mesh> h(new tc_mesh);
    h->m = tcloth::build_mesh(in);
    *out = h.release();
  });
}
tc_status tc_mesh_destroy(tc_mesh* m) {
  return guard([&] { delete m; });
}
tc_status tc_mesh_counts(tc_mesh* h, uint32_t out[10], float* cell) {
  return guard([&] {
    need(h && out, "handle and output required");
    const auto& m = h->m;
    out[0] = m.n; out[1] = uint32_t(m.dist.size()); out[2] = uint32_t(m.bend.size()); out[3] = uint32_t(m.edges.size() / 2);
    out[4] = uint32_t(m.dist_cnt.size()); out[5] = uint32_t(m.bend_cnt.size()); out[6] = m.table;
    out[7] = m.multi_layer ? 1u : 0u; out[8] = m.num_virtual; out[9] = uint32_t(m.adj_idx.size());
    if (cell) *cell = m.cell;
  });
}
tc_status tc_mesh_constraints(tc_mesh* h, uint32_t* dv, float* dp, uint32_t* doff, uint32_t* dcnt, uint32_t* bv,
                              float* bp, uint32_t* boff, uint32_t* bcnt) {
  return guard([&] {
    need(h != nullptr, "handle required");
    const auto& m = h->m;
    for (size_t i = 0; i < m.dist.size(); ++i) {
      const auto& c = m.dist[i];
      if (dv) { dv[2 * i] = c.v0; dv[2 * i + 1] = c.v1; }
      if (dp) { dp[4 * i] = c.rest; dp[4 * i + 1] = c.tc; dp[4 * i + 2] = c.cc; dp[4 * i + 3] = float(c.type); }
    }
    for (size_t i = 0; i < m.bend.size(); ++i) {
      const auto& c = m.bend[i];
      if (bv) { bv[4 * i] = c.v0; bv[4 * i + 1] = c.v1; bv[4 * i + 2] = c.v2; bv[4 * i + 3] = c.v3; }
      if (bp) { bp[4 * i] = c.rest; bp[4 * i + 1] = c.comp; bp[4 * i + 2] = c.pad0; bp[4 * i + 3] = c.pad1; }
    }
    if (doff) std::copy(m.dist_off.begin(), m.dist_off.end(), doff);
    if (dcnt) std::copy(m.dist_cnt.begin(), m.dist_cnt.end(), dcnt);
    if (boff) std::copy(m.bend_off.begin(), m.bend_off.end(), boff);
    if (bcnt) std::copy(m.bend_cnt.begin(), m.bend_cnt.end(), bcnt);
  });
}
tc_status tc_mesh_sewing(tc_mesh* h, uint32_t* nsew, uint32_t* ncolors, uint32_t* v01, float* par, uint32_t* off,
                         uint32_t* cnt, uint32_t* rep) {
  return guard([&] {
    need(h != nullptr, "handle required");
    const auto& m = h->m;
    if (nsew) *nsew = uint32_t(m.sew.size());
    if (ncolors) *ncolors = uint32_t(m.sew_cnt.size());
    for (size_t i = 0; i < m.sew.size(); ++i) {
      const auto& c = m.sew[i];
      if (v01) { v01[2 * i] = c.v0; v01[2 * i + 1] = c.v1; }
      if (par) {
        par[5 * i] = c.cur_rest; par[5 * i + 1] = c.target_rest; par[5 * i + 2] = c.shrink_speed;
        par[5 * i + 3] = c.compliance; par[5 * i + 4] = c.lock;
      }
    }
    if (off) std::copy(m.sew_off.begin(), m.sew_off.end(), off);
    if (cnt) std::copy(m.sew_cnt.begin(), m.sew_cnt.end(), cnt);
    if (rep) std::copy(m.sew_rep.begin(), m.sew_rep.end(), rep);
  });
}
tc_status tc_mesh_topology_sizes(tc_mesh* h, uint32_t* a, uint32_t* t, uint32_t* s) {
  return guard([&] {
    need(h != nullptr, "handle required");
    *a = uint32_t(h->m.adj_idx.size()); *t = uint32_t(h->m.th_idx.size()); *s = uint32_t(h->m.star_idx.size() / 2);
  });
}
tc_status tc_mesh_topology(tc_mesh* h, uint32_t* adj_off, uint32_t* adj_idx, uint32_t* th_off, uint32_t* th_idx,
                           float* th_rest, float* local_len, uint32_t* star_off, uint32_t* star_idx, uint32_t* island,
                           uint32_t* layer, uint32_t* edges, uint32_t* edge_bits) {
  return guard([&] {
    need(h != nullptr, "handle required");
    const auto& m = h->m;
    auto cp = [](const auto& v, auto* dst) { if (dst) std::copy(v.begin(), v.end(), dst); };
    cp(m.adj_off, adj_off); cp(m.adj_idx, adj_idx); cp(m.th_off, th_off); cp(m.th_idx, th_idx);
    cp(m.th_rest, th_rest); cp(m.local_len, local_len); cp(m.star_off, star_off); cp(m.star_idx, star_idx);
    cp(m.island, island); cp(m.layer, layer); cp(m.edges, edges); cp(m.edge_bits, edge_bits);
  });
}

tc_status tc_set_profiling_enabled(tc_sim* s, int on) {
  return guard([&] {
    Sim& m = S(s);
    m.profiling = on != 0;
    m.prof_names.clear(); m.prof_ms.clear(); m.prof_cnt.clear();
  });
}
tc_status tc_take_profile(tc_sim* s, char* names, size_t names_len, float* ms, uint32_t* launches, uint32_t max_entries,
                          uint32_t* n_entries) {
  return guard([&] {
    Sim& m = S(s);
    need(n_entries != nullptr, "n_entries required");
    std::string joined;
    const uint32_t k = uint32_t(std::min<size_t>(m.prof_names.size(), max_entries));
    for (uint32_t i = 0; i < k; ++i) {
      joined += m.prof_names[i];
      joined += '\n';
      if (ms) ms[i] = float(m.prof_ms[i]);
      if (launches) launches[i] = m.prof_cnt[i];
    }
    if (names && names_len) std::snprintf(names, names_len, "%s", joined.c_str());
    *n_entries = k;
    m.prof_names.clear(); m.prof_ms.clear(); m.prof_cnt.clear();
  });
}

// Launch shape of the persistent solver: blocks per SM (1..occupancy limit).
// Results do not depend on it (grid-stride loops, same per-element work).
tc_status tc_set_launch_config(tc_sim* s, int persistent, uint32_t blocks_per_sm) {
  return guard([&] {
    Sim& m = S(s);
    if (persistent == 2) {  // cluster solver (batched instances without self-collision)
      need(m.can_cluster(), "the cluster solver needs batched instances, no self-collision and cluster launch");
      m.cluster_mode = true;
      m.cl_stale = true;
      m.stage_mode = false;
      m.mark();
      return;
    }
    if (persistent == 3) {  // staged cluster solver (the same, vertex records in shared memory)
      need(m.can_stage(), "the staged solver needs batched instances, no self-collision, cluster launch and "
                          "every instance within one cluster's shared memory");
      m.stage_mode = true;
      m.st_stale = true;
      m.cluster_mode = false;
      m.mark();
      return;
    }
    m.stage_mode = false;
    if (persistent) {
      need(m.persist_max_per_sm > 0, "cooperative launch is not available on this device");
      need(blocks_per_sm >= 1 && blocks_per_sm <= m.persist_max_per_sm, "blocks_per_sm out of the occupancy range");
      m.persist_blocks = m.num_sms * blocks_per_sm;
    }
    m.cluster_mode = false;
    m.persistent = persistent != 0;
    m.mark();
  });
}
tc_status tc_get_launch_limits(tc_sim* s, uint32_t* max_blocks_per_sm, uint32_t* num_sms) {
  return guard([&] {
    Sim& m = S(s);
    *max_blocks_per_sm = m.persist_max_per_sm;
    *num_sms = m.num_sms;
  });
}

tc_status tc_set_persistent_solver(tc_sim* s, int enable) {
  return guard([&] {
    Sim& m = S(s);
    if (enable && !m.persist_blocks) throw TcError(TC_ERR_CUDA, "cooperative launch is not available on this device");
    m.persistent = enable != 0;
    m.mark();
  });
}

// Runs the persistent solver's barrier once with one more expected arrival
// than there are blocks, so it can never be released, and with the given
// poll limit: every wait ends by the limit and the launch reports
// TC_ERR_TIMEOUT.  No vertex or constraint is touched (zero-size phases).
tc_status tc_check_barrier_timeout(tc_sim* s, uint32_t spin_limit) {
  return guard([&] {
    Sim& m = S(s);
    need(m.persist_blocks > 0, "cooperative launch is not available on this device");
    need(spin_limit > 0 && spin_limit <= (1u << 22), "spin_limit must be in [1, 4194304]");
    const SubstepParams sp{1e-3f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    SolverArgs a = m.solver_args(sp, 1, false, false);
    a.n = 0; a.nd = 0; a.nb = 0; a.npins = 0; a.ndc = 0; a.nbc = 0; a.hascol = false;
    a.ca.bone.nbones = 0;
    a.bar = m.bar.p + 1;
    a.expected = m.persist_blocks + 1;
    a.spin_limit = spin_limit;
    m.launch_persistent(a);
    int err = 0;
    TC_CK(cudaMemcpyAsync(&err, &a.bar->err, sizeof(int), cudaMemcpyDeviceToHost, m.st));
    TC_CK(cudaStreamSynchronize(m.st));
    TC_CK(cudaMemsetAsync(a.bar, 0, sizeof(GridBar), m.st));
    TC_CK(cudaStreamSynchronize(m.st));
    if (err) throw TcError(TC_ERR_TIMEOUT, "grid barrier wait reached its poll limit");
  });
}

tc_status tc_frame_kernel_count(tc_sim* s, uint32_t* count) {
  return guard([&] { Sim& m = S(s); need(count != nullptr, "count required"); *count = m.graph_kernels; });
}

tc_status tc_last_frame_ms(tc_sim* s, float* ms) {
  return guard([&] {
    Sim& m = S(s);
    TC_CK(cudaEventSynchronize(m.ev1));
    TC_CK(cudaEventElapsedTime(ms, m.ev0, m.ev1));
  });
}

// ---- bone SDF colliders
using tcloth::BakeParams;
using tcloth::BakeTri;
using tcloth::BoneInfo;
using tcloth::BoneSdfState;

static BoneInfo info_from_row(const float* r) {
  return BoneInfo{make_float4(r[0], r[1], r[2], r[3]), make_float4(r[4], r[5], r[6], r[7]),
                  make_float4(r[8], r[9], r[10], r[11]), make_float4(r[12], r[13], r[14], r[15]),
                  make_float4(r[16], r[17], r[18], r[19])};
}

tc_status tc_set_bone_sdf_colliders(tc_sim* s, uint32_t width, uint32_t height, uint32_t depth,
                                    const uint32_t* texels, size_t n_texels, const float* infos, uint32_t n_bones) {
  return guard([&] {
    Sim& m = S(s);
    const size_t nvox = size_t(width) * height * depth;
    need(n_texels == nvox && (nvox == 0 || texels != nullptr), "texture size must be width*height*depth texels");
    need(n_bones == 0 || infos != nullptr, "bone_infos required");
    m.bone.w = width; m.bone.h = height; m.bone.d = depth;
    if (nvox) m.bone.atlas.upload(texels, nvox, m.st);
    m.bone.info_h.resize(n_bones);
    for (uint32_t b = 0; b < n_bones; ++b) m.bone.info_h[b] = info_from_row(infos + 20 * size_t(b));
    m.bone.enabled = n_bones > 0 && nvox > 0;
    m.mark();
    if (n_bones) m.set_identity_transforms(n_bones);
    TC_CK(cudaStreamSynchronize(m.st));
  });
}

static void set_dirty(Sim& m, const uint32_t* dirty, int64_t ndirty) {
  if (ndirty < 0) { m.bone.dirty_set = false; m.bone.dirty.clear(); return; }
  m.bone.dirty_set = true;
  m.bone.dirty.assign(dirty, dirty + ndirty);
}

tc_status tc_update_bone_transforms(tc_sim* s, const float* world, const float* inv_world, uint32_t n_bones,
                                    const uint32_t* dirty, int64_t n_dirty) {
  return guard([&] {
    Sim& m = S(s);
    need(n_bones == 0 || (world && inv_world), "world and inverse matrices required");
    need(n_dirty <= 0 || dirty != nullptr, "dirty list required");
    if (n_bones) m.set_bone_transforms(world, inv_world, n_bones);
    set_dirty(m, dirty, n_dirty);
  });
}

tc_status tc_set_dynamic_bone_sdf_dirty_bones(tc_sim* s, const uint32_t* dirty, int64_t n_dirty) {
  return guard([&] {
    Sim& m = S(s);
    need(n_dirty <= 0 || dirty != nullptr, "dirty list required");
    set_dirty(m, dirty, n_dirty);
  });
}

tc_status tc_clear_bone_sdf_colliders(tc_sim* s) {
  return guard([&] { S(s).clear_bone(); });
}

tc_status tc_set_dynamic_bone_sdf_enabled(tc_sim* s, int enable) {
  return guard([&] { Sim& m = S(s); m.bone.dyn_on = enable != 0 && m.bone.dyn; });
}

tc_status tc_set_dynamic_bone_sdf_update_interval(tc_sim* s, uint32_t interval) {
  return guard([&] { S(s).bone.interval = std::max(interval, 1u); });
}

// open boundary edges: undirected edges used by exactly one valid triangle
// (sdf_baker.rs:203-240)
static std::vector<uint64_t> open_boundary_edges(const int32_t* tris, size_t nt, size_t nv) {
  std::vector<uint64_t> keys;
  keys.reserve(nt * 3);
  for (size_t t = 0; t < nt; ++t) {
    const int32_t i0 = tris[3 * t], i1 = tris[3 * t + 1], i2 = tris[3 * t + 2];
    if (i0 < 0 || i1 < 0 || i2 < 0 || size_t(i0) >= nv || size_t(i1) >= nv || size_t(i2) >= nv || i0 == i1 ||
        i1 == i2 || i2 == i0)
      continue;
    const int32_t e[3][2] = {{i0, i1}, {i1, i2}, {i2, i0}};
    for (auto& q : e)
      keys.push_back((uint64_t(uint32_t(std::min(q[0], q[1]))) << 32) | uint32_t(std::max(q[0], q[1])));
  }
  std::sort(keys.begin(), keys.end());
  std::vector<uint64_t> once;
  for (size_t i = 0; i < keys.size();) {
    size_t j = i;
    while (j < keys.size() && keys[j] == keys[i]) ++j;
    if (j - i == 1) once.push_back(keys[i]);
    i = j;
  }
  return once;
}
static bool has_edge(const std::vector<uint64_t>& sorted, int32_t a, int32_t b) {
  const uint64_t k = (uint64_t(uint32_t(std::min(a, b))) << 32) | uint32_t(std::max(a, b));
  return std::binary_search(sorted.begin(), sorted.end(), k);
}
static uint32_t bmask_of(const std::vector<uint64_t>& open, int32_t i0, int32_t i1, int32_t i2) {
  uint32_t m = 0;
  if (has_edge(open, i0, i1)) m |= 1u;
  if (has_edge(open, i1, i2)) m |= 2u;
  if (has_edge(open, i2, i0)) m |= 4u;
  return m;
}

tc_status tc_setup_dynamic_bone_sdf(tc_sim* s, uint32_t width, uint32_t height, uint32_t depth, uint32_t res,
                                    const float* infos, uint32_t n_bones, const float* rest_verts,
                                    uint32_t rest_cols, const uint32_t* bone_indices, const float* bone_weights,
                                    uint32_t nv, const uint32_t* tri_sources, const float* tri_weights, uint32_t nt,
                                    const float* bind_inv, uint32_t n_bind, uint32_t update_interval) {
  return guard([&] {
    Sim& m = S(s);
    need(res > 0 && width > 0 && height > 0 && depth > 0, "width, height, depth and res must be >= 1");
    need(rest_cols >= 3, "rest_verts needs at least 3 columns");
    need(n_bind >= n_bones, "bone_bind_inv_matrices must hold one matrix per bone");
    need((nv == 0 || (rest_verts && bone_indices && bone_weights)) && (nt == 0 || (tri_sources && tri_weights)) &&
             (n_bones == 0 || (infos && bind_inv)),
         "arrays required");
    // the reference's setup is a no-op without vertices, triangles or bones
    if (nv == 0 || nt == 0 || n_bones == 0) return;
    for (uint32_t i = 0; i < nv; ++i)
      for (int k = 0; k < 4; ++k)
        need(!(bone_weights[4 * size_t(i) + k] > 0.f) || bone_indices[4 * size_t(i) + k] < n_bones,
             "bone index out of range for a weighted vertex");
    for (uint32_t t = 0; t < nt; ++t) {
      const uint32_t* q = tri_sources + 4 * size_t(t);
      need(q[0] < nv && q[1] < nv && q[2] < nv && q[3] < n_bones, "triangle source index out of range");
    }
    BoneSdfState& B = m.bone;
    B.info_h.resize(n_bones);
    for (uint32_t b = 0; b < n_bones; ++b) B.info_h[b] = info_from_row(infos + 20 * size_t(b));
    // open-boundary mask from the first occurrence of each distinct triangle (lib.rs:2490-2540)
    std::vector<int32_t> uniq;
    {
      // (sorted triangle, index) pairs: the first index of each distinct key
      std::vector<std::pair<std::array<uint32_t, 3>, uint32_t>> seen(nt);
      for (uint32_t t = 0; t < nt; ++t) {
        const uint32_t* q = tri_sources + 4 * size_t(t);
        std::array<uint32_t, 3> k{q[0], q[1], q[2]};
        std::sort(k.begin(), k.end());
        seen[t] = std::make_pair(k, t);
      }
      std::sort(seen.begin(), seen.end());
      std::vector<char> first(nt, 0);
      for (uint32_t i = 0; i < nt; ++i)
        if (i == 0 || seen[i].first != seen[i - 1].first) first[seen[i].second] = 1;
      for (uint32_t t = 0; t < nt; ++t)
        if (first[t]) {
          const uint32_t* q = tri_sources + 4 * size_t(t);
          uniq.push_back(int32_t(q[0])); uniq.push_back(int32_t(q[1])); uniq.push_back(int32_t(q[2]));
        }
    }
    const std::vector<uint64_t> open = open_boundary_edges(uniq.data(), uniq.size() / 3, nv);
    std::vector<uint4> src(nt);
    std::vector<float4> srcw(nt);
    std::vector<uint32_t> start(n_bones, 0), count(n_bones, 0);
    for (uint32_t t = 0; t < nt; ++t) {
      const uint32_t* q = tri_sources + 4 * size_t(t);
      const float* w = tri_weights + 3 * size_t(t);
      float bm = 0.f;
      if (q[0] != q[1] && q[1] != q[2] && q[2] != q[0]) bm = float(bmask_of(open, int32_t(q[0]), int32_t(q[1]), int32_t(q[2])));
      src[t] = make_uint4(q[0], q[1], q[2], q[3]);
      srcw[t] = make_float4(w[0], w[1], w[2], bm);
      if (count[q[3]] == 0) start[q[3]] = t;
      count[q[3]] += 1;
    }
    const uint32_t ncols = std::max(width / res, 1u), nrows = std::max(height / res, 1u);
    B.params_h.resize(n_bones);
    for (uint32_t b = 0; b < n_bones; ++b) {
      const uint32_t l = b / (ncols * nrows), rem = b % (ncols * nrows);
      const BoneInfo& I = B.info_h[b];
      B.params_h[b] = BakeParams{{I.aabb_min.x, I.aabb_min.y, I.aabb_min.z}, start[b],
                                 {I.aabb_max.x, I.aabb_max.y, I.aabb_max.z}, count[b], rem % ncols, rem / ncols, l,
                                 res, width, height, depth, 0u};
      need(uint64_t(rem % ncols + 1) * res <= width && uint64_t(rem / ncols + 1) * res <= height &&
               uint64_t(l + 1) * res <= depth,
           "atlas too small for the bone tiles");
    }
    std::vector<float4> rp(nv), bwv(nv);
    std::vector<uint4> bi(nv);
    for (uint32_t i = 0; i < nv; ++i) {
      const float* r = rest_verts + size_t(rest_cols) * i;
      rp[i] = make_float4(r[0], r[1], r[2], 0.f);
      const uint32_t* x = bone_indices + 4 * size_t(i);
      const float* w = bone_weights + 4 * size_t(i);
      bi[i] = make_uint4(x[0], x[1], x[2], x[3]);
      bwv[i] = make_float4(w[0], w[1], w[2], w[3]);
    }
    B.rest.upload(rp, m.st); B.bidx.upload(bi, m.st); B.bw.upload(bwv, m.st); B.skinned.alloc(nv);
    B.tsrc.upload(src, m.st); B.tsrcw.upload(srcw, m.st);
    B.bake.nt = nt;
    B.bake.tris.alloc(nt);
    B.bake.setup_tiles(tcloth::make_bake_tiles(start, count), m.st);
    {
      // rest-pose centroids order the spatial tiles (culling only)
      std::vector<float> cent(3 * size_t(nt));
      for (uint32_t t = 0; t < nt; ++t) {
        const uint32_t* q = tri_sources + 4 * size_t(t);
        for (int a = 0; a < 3; ++a)
          cent[3 * size_t(t) + a] = (rest_verts[size_t(rest_cols) * q[0] + a] + rest_verts[size_t(rest_cols) * q[1] + a] +
                                     rest_verts[size_t(rest_cols) * q[2] + a]) / 3.0f;
      }
      B.bake.setup_spatial(tcloth::bake_spatial_perm(cent, start, count, nt), start, count, m.st);
    }
    B.bind_inv.assign(bind_inv, bind_inv + 16 * size_t(n_bones));
    B.nv = nv; B.nb = n_bones; B.res = res;
    B.w = width; B.h = height; B.d = depth;
    const size_t nvox = size_t(width) * height * depth;
    B.atlas.alloc(nvox);
    TC_CK(cudaMemsetAsync(B.atlas.p, 0, nvox * 4, m.st));
    // transforms: identity for bones without one yet (mod.rs:2055-2075); the
    // infos' world bounding spheres follow the current transforms
    {
      const size_t nx = std::max<size_t>(B.xf_h.size(), n_bones);
      std::vector<float> wm(16 * nx), im(16 * nx);
      for (size_t b = 0; b < nx; ++b) {
        if (b < B.xf_h.size()) {
          std::memcpy(&wm[16 * b], B.xf_h[b].m, 64);
          std::memcpy(&im[16 * b], B.xf_h[b].inv, 64);
        } else {
          for (int k = 0; k < 16; ++k) wm[16 * b + k] = im[16 * b + k] = (k % 5 == 0) ? 1.f : 0.f;
        }
      }
      m.set_bone_transforms(wm.data(), im.data(), uint32_t(nx));
    }
    B.enabled = true;
    B.dyn = true;
    B.dyn_on = true;
    B.baked = false;
    B.dirty_set = false;
    B.dirty.clear();
    B.counter = 0;
    B.interval = std::max(update_interval, 1u);
    m.mark();
    TC_CK(cudaStreamSynchronize(m.st));
  });
}

tc_status tc_get_bone_sdf_atlas(tc_sim* s, uint32_t* out, size_t len, uint32_t dims[3]) {
  return guard([&] {
    Sim& m = S(s);
    const size_t nvox = size_t(m.bone.w) * m.bone.h * m.bone.d;
    if (dims) { dims[0] = m.bone.w; dims[1] = m.bone.h; dims[2] = m.bone.d; }
    if (!out) return;
    need(len >= nvox, "output array too small");
    if (nvox) TC_CK(cudaMemcpyAsync(out, m.bone.atlas.p, nvox * 4, cudaMemcpyDeviceToHost, m.st));
    TC_CK(cudaStreamSynchronize(m.st));
  });
}

tc_status tc_get_bone_infos(tc_sim* s, float* out, size_t len, uint32_t* n_bones) {
  return guard([&] {
    Sim& m = S(s);
    if (n_bones) *n_bones = uint32_t(m.bone.info_h.size());
    if (!out) return;
    need(len >= m.bone.info_h.size() * 20, "output array too small");
    std::memcpy(out, m.bone.info_h.data(), m.bone.info_h.size() * sizeof(BoneInfo));
  });
}

// ---- bake_bone_sdf_gpu (sdf_baker.rs:465-940): host preparation, GPU bake
struct tc_bake {
  std::vector<uint32_t> texels;
  uint32_t w = 0, h = 0, d = 0;
  std::vector<float> infos;        // n_active x 20
  std::vector<uint32_t> active;    // source bone index per active bone
  std::vector<float> bind;         // n_active x 16 (row-major, as given)
  std::vector<uint32_t> nearest;   // coarse bake: 8 nearest triangles per voxel
  float coarse_voxel = 0.f;
};

namespace {
// row-major 4x4 point transform with the projective divide (sdf_baker.rs:167-177)
void tp_rowmajor(const float* m, const float* p, float* o) {
  const float x = ((m[0] * p[0] + m[1] * p[1]) + m[2] * p[2]) + m[3];
  const float y = ((m[4] * p[0] + m[5] * p[1]) + m[6] * p[2]) + m[7];
  const float z = ((m[8] * p[0] + m[9] * p[1]) + m[10] * p[2]) + m[11];
  const float w = ((m[12] * p[0] + m[13] * p[1]) + m[14] * p[2]) + m[15];
  if (std::fabs(w) > 1e-7f && std::fabs(w - 1.0f) > 1e-5f) {
    const float iw = 1.0f / w;
    o[0] = x * iw; o[1] = y * iw; o[2] = z * iw;
  } else {
    o[0] = x; o[1] = y; o[2] = z;
  }
}
void h_cross(const float* a, const float* b, float* o) {
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}
void h_normalize(const float* v, float* o) {
  const float l2 = (v[0] * v[0] + v[1] * v[1]) + v[2] * v[2];
  if (l2 > 1e-12f) {
    const float inv = 1.0f / std::sqrt(l2);
    o[0] = v[0] * inv; o[1] = v[1] * inv; o[2] = v[2] * inv;
  } else {
    o[0] = 0.f; o[1] = 1.f; o[2] = 0.f;
  }
}
bool valid_tri(const int32_t* t, size_t nv) {
  return !(t[0] < 0 || t[1] < 0 || t[2] < 0 || size_t(t[0]) >= nv || size_t(t[1]) >= nv || size_t(t[2]) >= nv ||
           t[0] == t[1] || t[1] == t[2] || t[2] == t[0]);
}
// close_open_boundary_loops (sdf_baker.rs:242-453): fan caps over closed
// boundary loops of solid meshes; the cap centre's bone weights are the loop
// average.  weights: n_bones rows of `nv` (grown by one per added centre).
void close_open_loops(std::vector<float>& verts, std::vector<int32_t>& tris, std::vector<std::vector<float>>& weights) {
  const size_t nv = verts.size() / 3, nt = tris.size() / 3;
  if (nt < 4 || nv < 4) return;
  std::map<std::pair<int32_t, int32_t>, uint32_t> ecount;
  std::vector<std::array<int32_t, 3>> existing;
  for (size_t t = 0; t < nt; ++t) {
    const int32_t* q = &tris[3 * t];
    if (!valid_tri(q, nv)) continue;
    std::array<int32_t, 3> k{q[0], q[1], q[2]};
    std::sort(k.begin(), k.end());
    existing.push_back(k);
    const int32_t e[3][2] = {{q[0], q[1]}, {q[1], q[2]}, {q[2], q[0]}};
    for (auto& x : e) ecount[{std::min(x[0], x[1]), std::max(x[0], x[1])}] += 1;
  }
  std::sort(existing.begin(), existing.end());
  std::vector<std::pair<int32_t, int32_t>> bedges;
  std::vector<std::array<float, 3>> bnormal;
  std::map<int32_t, std::vector<size_t>> next;
  for (size_t t = 0; t < nt; ++t) {
    const int32_t* q = &tris[3 * t];
    if (!valid_tri(q, nv)) continue;
    const float* p0 = &verts[3 * size_t(q[0])];
    const float* p1 = &verts[3 * size_t(q[1])];
    const float* p2 = &verts[3 * size_t(q[2])];
    const float e01[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]};
    const float e02[3] = {p2[0] - p0[0], p2[1] - p0[1], p2[2] - p0[2]};
    float cr[3], tn[3];
    h_cross(e01, e02, cr);
    h_normalize(cr, tn);
    const int32_t e[3][2] = {{q[0], q[1]}, {q[1], q[2]}, {q[2], q[0]}};
    for (auto& x : e) {
      if (ecount[{std::min(x[0], x[1]), std::max(x[0], x[1])}] == 1) {
        next[x[0]].push_back(bedges.size());
        bedges.push_back({x[0], x[1]});
        bnormal.push_back({tn[0], tn[1], tn[2]});
      }
    }
  }
  if (bedges.empty()) return;
  std::vector<char> used(bedges.size(), 0);
  for (size_t s0 = 0; s0 < bedges.size(); ++s0) {
    if (used[s0]) continue;
    used[s0] = 1;
    const int32_t su = bedges[s0].first, sv = bedges[s0].second;
    std::vector<int32_t> lv{su, sv};
    std::vector<size_t> le{s0};
    int32_t cur = sv;
    bool closed = false;
    while (lv.size() <= nv) {
      if (cur == su) { lv.pop_back(); closed = true; break; }
      bool found = false;
      auto it = next.find(cur);
      if (it != next.end())
        for (size_t ei : it->second)
          if (!used[ei]) {
            used[ei] = 1;
            le.push_back(ei);
            cur = bedges[ei].second;
            lv.push_back(cur);
            found = true;
            break;
          }
      if (!found) break;
    }
    const size_t k = lv.size();
    if (!closed || k < 3 || k >= nv) continue;
    const float invk = 1.0f / float(k);
    float c[3] = {0.f, 0.f, 0.f};
    for (int32_t v : lv)
      for (int j = 0; j < 3; ++j) c[j] += verts[3 * size_t(v) + j];
    for (int j = 0; j < 3; ++j) c[j] *= invk;
    float cs[3] = {0.f, 0.f, 0.f};
    for (size_t i = 0; i < k; ++i) {
      const float* pu = &verts[3 * size_t(lv[i])];
      const float* pv = &verts[3 * size_t(lv[(i + 1) % k])];
      const float d1[3] = {pu[0] - pv[0], pu[1] - pv[1], pu[2] - pv[2]};
      const float d2[3] = {c[0] - pv[0], c[1] - pv[1], c[2] - pv[2]};
      float cn[3];
      h_cross(d1, d2, cn);
      for (int j = 0; j < 3; ++j) cs[j] += cn[j];
    }
    float capn[3];
    h_normalize(cs, capn);
    float ds = 0.f;
    for (size_t ei : le) ds += (bnormal[ei][0] * capn[0] + bnormal[ei][1] * capn[1]) + bnormal[ei][2] * capn[2];
    if (ds / float(std::max<size_t>(le.size(), 1)) <= -0.85f) continue;
    if (k == 3) {
      std::array<int32_t, 3> key{lv[0], lv[1], lv[2]};
      std::sort(key.begin(), key.end());
      if (std::binary_search(existing.begin(), existing.end(), key)) continue;
      tris.insert(tris.end(), {lv[0], lv[2], lv[1]});
      existing.insert(std::upper_bound(existing.begin(), existing.end(), key), key);
      continue;
    }
    const int32_t ci = int32_t(verts.size() / 3);
    verts.insert(verts.end(), {c[0], c[1], c[2]});
    for (auto& w : weights) {
      float ws = 0.f;
      for (int32_t v : lv)
        if (size_t(v) < w.size()) ws += w[size_t(v)];
      while (w.size() < size_t(ci)) w.push_back(0.f);
      w.push_back(ws * invk);
    }
    for (size_t i = 0; i < k; ++i) tris.insert(tris.end(), {lv[(i + 1) % k], lv[i], ci});
  }
}
}  // namespace

tc_status tc_bake_bone_sdf(const float* mesh_verts, uint32_t nv, const int32_t* mesh_tris, uint32_t nt,
                           uint32_t n_bones, const float* bone_weights, const float* bind_matrices,
                           uint32_t resolution, float margin, float weight_threshold, float blend_k, float friction,
                           float thickness, float restitution, int close_open_boundaries, int device, tc_bake** out) {
  return guard([&] {
    need(out != nullptr, "out required");
    *out = nullptr;
    need(resolution >= 1, "resolution must be >= 1");
    need((nv == 0 || mesh_verts) && (nt == 0 || mesh_tris) && (n_bones == 0 || (bone_weights && bind_matrices)),
         "arrays required");
    std::vector<float> verts(mesh_verts, mesh_verts + 3 * size_t(nv));
    std::vector<int32_t> tris(mesh_tris, mesh_tris + 3 * size_t(nt));
    std::vector<std::vector<float>> weights(n_bones);
    for (uint32_t b = 0; b < n_bones; ++b) weights[b].assign(bone_weights + size_t(b) * nv, bone_weights + size_t(b + 1) * nv);
    if (close_open_boundaries) close_open_loops(verts, tris, weights);
    const size_t NV = verts.size() / 3, NT = tris.size() / 3;
    const std::vector<uint64_t> open = open_boundary_edges(tris.data(), NT, NV);
    std::vector<uint32_t> active;
    for (uint32_t b = 0; b < n_bones; ++b) {
      float mx = 0.f;
      for (float w : weights[b]) mx = std::fmax(mx, w);
      if (mx > weight_threshold) active.push_back(b);
    }
    if (active.empty()) throw TcError(TC_ERR_CUDA, "GPU SDF bake failed: no bone has skin weights above the threshold");
    // compute_3d_atlas_layout (sdf_baker.rs:137-164)
    const size_t na = active.size();
    const size_t ncols = std::max<size_t>(size_t(std::ceil(std::pow(double(na), 1.0 / 3.0))), 1);
    const size_t nrows = std::max<size_t>(size_t(std::ceil(std::sqrt(double((na + ncols - 1) / ncols)))), 1);
    const size_t nlay = std::max<size_t>((na + ncols * nrows - 1) / (ncols * nrows), 1);
    const size_t max_tile = std::max(std::max(ncols, nrows), nlay);
    const size_t res = max_tile * resolution > 2048 ? std::max<size_t>(2048 / max_tile, 16) : resolution;
    tc_bake* R = new tc_bake();
    std::unique_ptr<tc_bake> guard_r(R);
    R->w = uint32_t(ncols * res); R->h = uint32_t(nrows * res); R->d = uint32_t(nlay * res);
    std::vector<BakeTri> all;
    std::vector<BakeParams> params;
    std::vector<uint32_t> starts, counts, pbone;
    for (size_t ob = 0; ob < na; ++ob) {
      const uint32_t sb = active[ob];
      const float* M = bind_matrices + 16 * size_t(sb);
      R->active.push_back(sb);
      R->bind.insert(R->bind.end(), M, M + 16);
      float mn[3] = {INFINITY, INFINITY, INFINITY}, mxp[3] = {-INFINITY, -INFINITY, -INFINITY};
      size_t valid = 0;
      for (size_t v = 0; v < weights[sb].size(); ++v)
        if (weights[sb][v] > weight_threshold && v < NV) {
          float pl[3];
          tp_rowmajor(M, &verts[3 * v], pl);
          for (int k = 0; k < 3; ++k) { mn[k] = std::fmin(mn[k], pl[k]); mxp[k] = std::fmax(mxp[k], pl[k]); }
          ++valid;
        }
      if (!valid) for (int k = 0; k < 3; ++k) { mn[k] = -0.1f; mxp[k] = 0.1f; }
      float size[3];
      for (int k = 0; k < 3; ++k) size[k] = std::fmax(mxp[k] - mn[k], 0.05f);
      for (int k = 0; k < 3; ++k) {
        const float pad = size[k] * margin + std::fmax(thickness, 0.f);
        mn[k] -= pad;
        mxp[k] += pad;
        size[k] = mxp[k] - mn[k];
      }
      const size_t bpl = ncols * nrows;
      const uint32_t l = uint32_t(ob / bpl), rem = uint32_t(ob % bpl), r = uint32_t(rem / ncols), c = uint32_t(rem % ncols);
      const float sl[3] = {1.0f / size[0], 1.0f / size[1], 1.0f / size[2]};
      const float ol[3] = {-mn[0] / size[0], -mn[1] / size[1], -mn[2] / size[2]};
      float row[20];
      row[0] = mn[0]; row[1] = mn[1]; row[2] = mn[2]; row[3] = float(ob);
      row[4] = mxp[0]; row[5] = mxp[1]; row[6] = mxp[2]; row[7] = float(res);
      row[8] = sl[0] / float(ncols); row[9] = sl[1] / float(nrows); row[10] = sl[2] / float(nlay); row[11] = blend_k;
      row[12] = (ol[0] + float(c)) / float(ncols); row[13] = (ol[1] + float(r)) / float(nrows);
      row[14] = (ol[2] + float(l)) / float(nlay); row[15] = 0.f;
      row[16] = friction; row[17] = thickness; row[18] = restitution; row[19] = weight_threshold;
      R->infos.insert(R->infos.end(), row, row + 20);
      const uint32_t ts = uint32_t(all.size());
      for (size_t t = 0; t < NT; ++t) {
        const int32_t* q = &tris[3 * t];
        if (q[0] < 0 || q[1] < 0 || q[2] < 0 || size_t(q[0]) >= NV || size_t(q[1]) >= NV || size_t(q[2]) >= NV) continue;
        const float w0 = size_t(q[0]) < weights[sb].size() ? weights[sb][size_t(q[0])] : 0.f;
        const float w1 = size_t(q[1]) < weights[sb].size() ? weights[sb][size_t(q[1])] : 0.f;
        const float w2 = size_t(q[2]) < weights[sb].size() ? weights[sb][size_t(q[2])] : 0.f;
        if (!(w0 > 0.f || w1 > 0.f || w2 > 0.f)) continue;
        float p0[3], p1[3], p2[3];
        tp_rowmajor(M, &verts[3 * size_t(q[0])], p0);
        tp_rowmajor(M, &verts[3 * size_t(q[1])], p1);
        tp_rowmajor(M, &verts[3 * size_t(q[2])], p2);
        float tmin[3], tmax[3];
        for (int k = 0; k < 3; ++k) {
          tmin[k] = std::fmin(std::fmin(p0[k], p1[k]), p2[k]);
          tmax[k] = std::fmax(std::fmax(p0[k], p1[k]), p2[k]);
        }
        const bool overlap = tmin[0] <= mxp[0] && tmax[0] >= mn[0] && tmin[1] <= mxp[1] && tmax[1] >= mn[1] &&
                             tmin[2] <= mxp[2] && tmax[2] >= mn[2];
        if (!overlap) continue;
        const float e01[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]};
        const float e02[3] = {p2[0] - p0[0], p2[1] - p0[1], p2[2] - p0[2]};
        float cr[3], nn[3];
        h_cross(e01, e02, cr);
        h_normalize(cr, nn);
        const uint32_t bm = bmask_of(open, q[0], q[1], q[2]);
        all.push_back(BakeTri{make_float4(p0[0], p0[1], p0[2], w0), make_float4(p1[0], p1[1], p1[2], w1),
                              make_float4(p2[0], p2[1], p2[2], w2), make_float4(nn[0], nn[1], nn[2], float(bm))});
      }
      const uint32_t tc = uint32_t(all.size()) - ts;
      params.push_back(BakeParams{{mn[0], mn[1], mn[2]}, ts, {mxp[0], mxp[1], mxp[2]}, tc, c, r, l, uint32_t(res),
                                  R->w, R->h, R->d, 0u});
      starts.push_back(ts);
      counts.push_back(tc);
      pbone.push_back(uint32_t(ob));
    }
    if (all.empty())
      all.push_back(BakeTri{make_float4(0, 0, 0, 0), make_float4(0, 0, 0, 0), make_float4(0, 0, 0, 0), make_float4(0, 1, 0, 0)});
    TC_CK(cudaSetDevice(device));
    cudaStream_t st = nullptr;
    TC_CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    struct StreamGuard { cudaStream_t s; ~StreamGuard() { cudaStreamSynchronize(s); cudaStreamDestroy(s); } } sg{st};
    tcloth::BakeGpu G;
    G.nt = uint32_t(all.size());
    G.tris.upload(all, st);
    G.setup_tiles(tcloth::make_bake_tiles(starts, counts), st);
    {
      std::vector<float> cent(3 * all.size());
      for (size_t t = 0; t < all.size(); ++t) {
        const tcloth::BakeTri& q = all[t];
        cent[3 * t] = (q.p0w0.x + q.p1w1.x + q.p2w2.x) / 3.0f;
        cent[3 * t + 1] = (q.p0w0.y + q.p1w1.y + q.p2w2.y) / 3.0f;
        cent[3 * t + 2] = (q.p0w0.z + q.p1w1.z + q.p2w2.z) / 3.0f;
      }
      G.setup_spatial(tcloth::bake_spatial_perm(cent, starts, counts, G.nt), starts, counts, st);
    }
    tcloth::DBuf<uint32_t> atlas;
    const size_t nvox = size_t(R->w) * R->h * R->d;
    atlas.alloc(nvox);
    TC_CK(cudaMemsetAsync(atlas.p, 0, nvox * 4, st));
    G.bake(params, pbone, atlas.p, st);
    R->texels.resize(nvox);
    TC_CK(cudaMemcpyAsync(R->texels.data(), atlas.p, nvox * 4, cudaMemcpyDeviceToHost, st));
    TC_CK(cudaStreamSynchronize(st));
    TC_CK(cudaGetLastError());
    *out = guard_r.release();
  });
}

// bake_mesh_sdf_gpu (lib.rs:1349-1416; sdf_baker.rs:939-1060, :1114-1326):
// the signed distance field of one mesh over its padded bounding box.
namespace {
// The host half of every single-mesh bake: mesh_sdf_domain (sdf_baker.rs:939-982),
// mesh_sdf_bone_info (:984-1016) and collect_mesh_bake_triangles (:1018-1060).
struct MeshBakeSetup {
  float lo[3], hi[3], size[3];
  uint32_t dim[3];
  std::vector<float> infos;
  std::vector<tcloth::BakeTri> tris;
};
MeshBakeSetup mesh_bake_setup(const std::vector<float>& verts, const std::vector<int32_t>& tris, float voxel_size,
                              float margin, float friction, float thickness, float restitution) {
  MeshBakeSetup S;
  const size_t NV = verts.size() / 3, NT = tris.size() / 3;
  for (int k = 0; k < 3; ++k) { S.lo[k] = INFINITY; S.hi[k] = -INFINITY; }
  for (size_t v = 0; v < NV; ++v)
    for (int k = 0; k < 3; ++k) { S.lo[k] = std::fmin(S.lo[k], verts[3 * v + k]); S.hi[k] = std::fmax(S.hi[k], verts[3 * v + k]); }
  const float vs = std::fmax(voxel_size, 0.001f);
  for (int k = 0; k < 3; ++k) {
    S.size[k] = std::fmax(S.hi[k] - S.lo[k], 0.05f);
    const float pad = (std::fmax(S.size[k] * margin, 0.04f) + std::fmax(thickness, 0.f)) + 0.02f;
    S.lo[k] -= pad;
    S.hi[k] += pad;
    S.size[k] = S.hi[k] - S.lo[k];
    const float raw = std::ceil(S.size[k] / vs);
    const double r = (raw == raw && raw > 0.f) ? double(raw) : 0.0;
    S.dim[k] = uint32_t(std::min(std::max(r, 8.0), 2048.0));
  }
  S.infos.assign(20, 0.f);
  for (int k = 0; k < 3; ++k) {
    S.infos[k] = S.lo[k];
    S.infos[4 + k] = S.hi[k];
    S.infos[8 + k] = 1.0f / S.size[k];
    S.infos[12 + k] = -S.lo[k] / S.size[k];
  }
  S.infos[7] = float(S.dim[0]);
  S.infos[16] = friction; S.infos[17] = thickness; S.infos[18] = restitution;
  for (size_t t = 0; t < NT; ++t) {
    const int32_t i0 = tris[3 * t], i1 = tris[3 * t + 1], i2 = tris[3 * t + 2];
    if (i0 < 0 || i1 < 0 || i2 < 0 || size_t(i0) >= NV || size_t(i1) >= NV || size_t(i2) >= NV) continue;
    const float* p0 = &verts[3 * size_t(i0)];
    const float* p1 = &verts[3 * size_t(i1)];
    const float* p2 = &verts[3 * size_t(i2)];
    const float e1[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]};
    const float e2[3] = {p2[0] - p0[0], p2[1] - p0[1], p2[2] - p0[2]};
    const float c[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
    const float l2 = c[0] * c[0] + c[1] * c[1] + c[2] * c[2];
    float nrm[3] = {0.f, 1.f, 0.f};
    if (l2 > 1e-12f) {
      const float il = 1.0f / std::sqrt(l2);
      nrm[0] = c[0] * il; nrm[1] = c[1] * il; nrm[2] = c[2] * il;
    }
    S.tris.push_back(tcloth::BakeTri{make_float4(p0[0], p0[1], p0[2], 0.f), make_float4(p1[0], p1[1], p1[2], 0.f),
                                     make_float4(p2[0], p2[1], p2[2], 0.f), make_float4(nrm[0], nrm[1], nrm[2], 0.f)});
  }
  if (S.tris.empty())
    S.tris.push_back(tcloth::BakeTri{make_float4(0, 0, 0, 0), make_float4(0, 0, 0, 0), make_float4(0, 0, 0, 0),
                                     make_float4(0, 1, 0, 0)});
  return S;
}
// triangles on the device with their culling spheres (one tile run)
void mesh_bake_upload(const MeshBakeSetup& S, tcloth::BakeGpu& G, cudaStream_t st) {
  G.nt = uint32_t(S.tris.size());
  G.tris.upload(S.tris, st);
  G.setup_tiles(tcloth::make_bake_tiles({0u}, {G.nt}), st);
  tcloth::k_bone_tri_spheres<<<(G.nt + 255) / 256, 256, 0, st>>>(G.nt, G.tris.p, G.sph.p);
  tcloth::k_bone_tile_spheres<<<(G.ntiles + 127) / 128, 128, 0, st>>>(G.ntiles, G.tile_first.p, G.tile_cnt.p, G.sph.p,
                                                                       G.tsph.p);
}
tcloth::MeshBakeParams mesh_bake_params(const MeshBakeSetup& S, uint32_t ntri) {
  return tcloth::MeshBakeParams{{S.lo[0], S.lo[1], S.lo[2]}, {S.hi[0], S.hi[1], S.hi[2]}, S.dim[0], S.dim[1], S.dim[2],
                                ntri};
}
uint32_t brick_blocks(const uint32_t dim[3]) {
  return ((dim[0] + 7) / 8) * ((dim[1] + 7) / 8) * ((dim[2] + 3) / 4);
}
struct OwnStream {
  cudaStream_t s = nullptr;
  explicit OwnStream(int device) {
    TC_CK(cudaSetDevice(device));
    TC_CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  }
  ~OwnStream() { cudaStreamSynchronize(s); cudaStreamDestroy(s); }
};
// the coarse pass (bake_mesh_sdf_coarse_ext, sdf_baker.rs:1350-1600): domain
// at max(voxel x 4, 0.001), packed distance and the 8 nearest triangles per
// coarse voxel; device buffers are left in G / dist / near8 for the fine pass
struct CoarseBake {
  MeshBakeSetup S;
  float coarse_voxel = 0.f;
  tcloth::BakeGpu G;
  tcloth::DBuf<uint32_t> dist, near8;
};
void coarse_bake(const std::vector<float>& verts, const std::vector<int32_t>& tris, float voxel_size, float margin,
                 float friction, float thickness, float restitution, CoarseBake& C, cudaStream_t st) {
  C.coarse_voxel = std::fmax(voxel_size * 4.0f, 0.001f);
  C.S = mesh_bake_setup(verts, tris, C.coarse_voxel, margin, friction, thickness, restitution);
  mesh_bake_upload(C.S, C.G, st);
  const size_t nvox = size_t(C.S.dim[0]) * C.S.dim[1] * C.S.dim[2];
  C.dist.alloc(nvox);
  C.near8.alloc(nvox * 8);
  tcloth::k_mesh_bake_coarse<<<brick_blocks(C.S.dim), 256, 0, st>>>(mesh_bake_params(C.S, C.G.nt), C.G.tris.p,
                                                                    C.G.sph.p, C.G.tsph.p, C.dist.p, C.near8.p);
  TC_CK(cudaGetLastError());
}
}  // namespace

tc_status tc_bake_mesh_sdf(const float* mesh_verts, uint32_t nv, const int32_t* mesh_tris, uint32_t nt,
                           float voxel_size, float margin, float friction, float thickness, float restitution,
                           int close_open_boundaries, int device, tc_bake** out) {
  return guard([&] {
    need(out != nullptr, "out required");
    *out = nullptr;
    if (nv == 0) throw TcError(TC_ERR_CUDA, "GPU mesh SDF bake failed: the mesh has no vertices");
    need(mesh_verts != nullptr && (nt == 0 || mesh_tris != nullptr), "arrays required");
    std::vector<float> verts(mesh_verts, mesh_verts + 3 * size_t(nv));
    std::vector<int32_t> tris(mesh_tris, mesh_tris + 3 * size_t(nt));
    std::vector<std::vector<float>> no_weights;
    if (close_open_boundaries) close_open_loops(verts, tris, no_weights);
    const MeshBakeSetup S = mesh_bake_setup(verts, tris, voxel_size, margin, friction, thickness, restitution);
    std::unique_ptr<tc_bake> R(new tc_bake);
    R->w = S.dim[0]; R->h = S.dim[1]; R->d = S.dim[2];
    R->infos = S.infos;
    OwnStream os(device);
    tcloth::BakeGpu G;
    mesh_bake_upload(S, G, os.s);
    const size_t nvox = size_t(S.dim[0]) * S.dim[1] * S.dim[2];
    tcloth::DBuf<uint32_t> vox;
    vox.alloc(nvox);
    tcloth::k_mesh_bake<<<brick_blocks(S.dim), 256, 0, os.s>>>(mesh_bake_params(S, G.nt), G.tris.p, G.sph.p, G.tsph.p,
                                                                vox.p);
    R->texels.resize(nvox);
    TC_CK(cudaMemcpyAsync(R->texels.data(), vox.p, nvox * 4, cudaMemcpyDeviceToHost, os.s));
    TC_CK(cudaStreamSynchronize(os.s));
    TC_CK(cudaGetLastError());
    *out = R.release();
  });
}

tc_status tc_bake_mesh_sdf_coarse(const float* mesh_verts, uint32_t nv, const int32_t* mesh_tris, uint32_t nt,
                                  float voxel_size, float margin, float friction, float thickness, float restitution,
                                  int device, tc_bake** out) {
  return guard([&] {
    need(out != nullptr, "out required");
    *out = nullptr;
    if (nv == 0) throw TcError(TC_ERR_CUDA, "GPU coarse-grid bake failed: the mesh has no vertices");
    need(mesh_verts != nullptr && (nt == 0 || mesh_tris != nullptr), "arrays required");
    std::vector<float> verts(mesh_verts, mesh_verts + 3 * size_t(nv));
    std::vector<int32_t> tris(mesh_tris, mesh_tris + 3 * size_t(nt));
    std::vector<std::vector<float>> no_weights;
    close_open_loops(verts, tris, no_weights);  // bake_mesh_sdf_coarse always caps
    OwnStream os(device);
    CoarseBake C;
    coarse_bake(verts, tris, voxel_size, margin, friction, thickness, restitution, C, os.s);
    std::unique_ptr<tc_bake> R(new tc_bake);
    R->w = C.S.dim[0]; R->h = C.S.dim[1]; R->d = C.S.dim[2];
    R->infos = C.S.infos;
    R->coarse_voxel = C.coarse_voxel;
    const size_t nvox = size_t(R->w) * R->h * R->d;
    R->texels.resize(nvox);
    R->nearest.resize(nvox * 8);
    TC_CK(cudaMemcpyAsync(R->texels.data(), C.dist.p, nvox * 4, cudaMemcpyDeviceToHost, os.s));
    TC_CK(cudaMemcpyAsync(R->nearest.data(), C.near8.p, nvox * 32, cudaMemcpyDeviceToHost, os.s));
    TC_CK(cudaStreamSynchronize(os.s));
    TC_CK(cudaGetLastError());
    *out = R.release();
  });
}

tc_status tc_bake_mesh_sdf_hierarchical(const float* mesh_verts, uint32_t nv, const int32_t* mesh_tris, uint32_t nt,
                                        float voxel_size, float margin, float friction, float thickness,
                                        float restitution, int close_open_boundaries, int device, tc_bake** out) {
  return guard([&] {
    need(out != nullptr, "out required");
    *out = nullptr;
    if (nv == 0) throw TcError(TC_ERR_CUDA, "GPU hierarchical mesh SDF bake failed: the mesh has no vertices");
    need(mesh_verts != nullptr && (nt == 0 || mesh_tris != nullptr), "arrays required");
    std::vector<float> verts(mesh_verts, mesh_verts + 3 * size_t(nv));
    std::vector<int32_t> tris(mesh_tris, mesh_tris + 3 * size_t(nt));
    std::vector<std::vector<float>> no_weights;
    if (close_open_boundaries) close_open_loops(verts, tris, no_weights);
    const MeshBakeSetup S = mesh_bake_setup(verts, tris, voxel_size, margin, friction, thickness, restitution);
    OwnStream os(device);
    CoarseBake C;
    coarse_bake(verts, tris, voxel_size, margin, friction, thickness, restitution, C, os.s);
    // band = 4 fine voxels, at most two coarse cells (sdf_baker.rs:1655-1667)
    const float h_fine = std::fmax(std::fmax(S.size[0] / float(S.dim[0]), S.size[1] / float(S.dim[1])),
                                   S.size[2] / float(S.dim[2]));
    const float band = 4.0f * h_fine;
    const float h_coarse_min = std::fmin(std::fmin(S.size[0] / float(C.S.dim[0]), S.size[1] / float(C.S.dim[1])),
                                         S.size[2] / float(C.S.dim[2]));
    if (band > 2.0f * h_coarse_min) {
      char msg[160];
      std::snprintf(msg, sizeof msg, "GPU hierarchical mesh SDF bake failed: band (%.4f m) too wide for the coarse "
                    "cell (%.4f m)", band, h_coarse_min);
      throw TcError(TC_ERR_CUDA, msg);
    }
    std::unique_ptr<tc_bake> R(new tc_bake);
    R->w = S.dim[0]; R->h = S.dim[1]; R->d = S.dim[2];
    R->infos = S.infos;
    const size_t nvox = size_t(S.dim[0]) * S.dim[1] * S.dim[2];
    tcloth::DBuf<uint32_t> vox;
    vox.alloc(nvox);
    const tcloth::HierFineParams H{C.S.dim[0], C.S.dim[1], C.S.dim[2], band};
    tcloth::k_mesh_bake_fine<<<unsigned((nvox + 127) / 128), 128, 0, os.s>>>(mesh_bake_params(S, C.G.nt), H,
                                                                            C.G.tris.p, C.dist.p, C.near8.p, vox.p);
    R->texels.resize(nvox);
    TC_CK(cudaMemcpyAsync(R->texels.data(), vox.p, nvox * 4, cudaMemcpyDeviceToHost, os.s));
    TC_CK(cudaStreamSynchronize(os.s));
    TC_CK(cudaGetLastError());
    *out = R.release();
  });
}

tc_status tc_bake_get_nearest(tc_bake* b, uint32_t* nearest, float* coarse_voxel) {
  return guard([&] {
    need(b != nullptr, "bake result required");
    if (nearest) std::memcpy(nearest, b->nearest.data(), b->nearest.size() * 4);
    if (coarse_voxel) *coarse_voxel = b->coarse_voxel;
  });
}

tc_status tc_compute_combined_inv_masses(const float* positions, uint32_t n, const uint32_t* faces, uint32_t nf,
                                         const uint32_t* strand_edges, uint32_t ns, const float* pin_weights,
                                         uint32_t npin, float areal_density, float linear_density, float* out) {
  return guard([&] {
    need(out != nullptr && (n == 0 || positions != nullptr), "positions and output required");
    const std::vector<float> w = tcloth::combined_inv_masses(positions, n, faces, faces ? nf : 0u, strand_edges,
                                                             strand_edges ? ns : 0u, pin_weights,
                                                             pin_weights ? npin : 0u, areal_density, linear_density);
    std::copy(w.begin(), w.end(), out);
  });
}
tc_status tc_color_edge_pairs(uint32_t num_vertices, const uint32_t* pairs, uint32_t np, uint32_t* colors) {
  return guard([&] {
    need(np == 0 || (pairs != nullptr && colors != nullptr), "pairs and colours required");
    const std::vector<uint32_t> c = tcloth::color_edge_pairs(num_vertices, pairs, np);
    std::copy(c.begin(), c.end(), colors);
  });
}

tc_status tc_find_triangle_intersections(const float* positions, uint32_t n, const uint32_t* faces, uint32_t nf,
                                         int ignore_adjacent, float cell_size, const uint32_t* sewing, uint32_t nsew,
                                         uint32_t* pairs, uint32_t capacity, uint32_t* count) {
  return guard([&] {
    need(count != nullptr, "count required");
    need((positions != nullptr || n == 0) && (faces != nullptr || nf == 0), "positions and faces required");
    need(capacity == 0 || pairs != nullptr, "pairs required when capacity > 0");
    const std::vector<uint32_t> r = tcloth::find_triangle_intersections(
        positions, n, faces, nf, ignore_adjacent != 0, cell_size, sewing, sewing ? nsew : 0);
    const uint32_t k = uint32_t(r.size() / 2);
    *count = k;
    std::copy(r.begin(), r.begin() + 2 * size_t(std::min(k, capacity)), pairs);
  });
}

tc_status tc_bake_dims(tc_bake* b, uint32_t out[4]) {
  return guard([&] {
    need(b && out, "bake result and output required");
    out[0] = b->w; out[1] = b->h; out[2] = b->d; out[3] = uint32_t(b->active.size());
  });
}

tc_status tc_bake_get(tc_bake* b, uint32_t* texels, float* infos, uint32_t* active, float* bind) {
  return guard([&] {
    need(b != nullptr, "bake result required");
    if (texels) std::memcpy(texels, b->texels.data(), b->texels.size() * 4);
    if (infos) std::memcpy(infos, b->infos.data(), b->infos.size() * 4);
    if (active) std::memcpy(active, b->active.data(), b->active.size() * 4);
    if (bind) std::memcpy(bind, b->bind.data(), b->bind.size() * 4);
  });
}

tc_status tc_bake_destroy(tc_bake* b) {
  delete b;
  return TC_OK;
}

// ---- kernel variants of the self-collision pass (results identical)
tc_status tc_set_self_collision_variant(tc_sim* s, uint32_t ee_variant) {
  return guard([&] {
    need(ee_variant <= 2u,
         "ee_variant: 0 (warp per edge, pair list), 1 (grouped by cell) or 2 (warp per edge, contact in the warp)");
    Sim& m = S(s);
    m.ee_grouped = ee_variant == 1u;
    m.ee_list = ee_variant == 0u;
    m.mark();
  });
}

tc_status tc_set_ee_pair_list_capacity(tc_sim* s, uint64_t entries) {
  return guard([&] {
    Sim& m = S(s);
    need(entries <= 0xffffffffull, "entries: at most 2^32 - 1");
    if (entries > m.ee_q.n && m.ee_q.p) {
      TC_CK(cudaStreamSynchronize(m.st));
      m.ee_q.alloc(size_t(entries));
    }
    m.ee_list_entries = size_t(entries);
    m.mark();
  });
}

// ---- autotuned knobs
tc_status tc_set_launch_block(tc_sim* s, uint32_t threads) {
  return guard([&] {
    need(threads == 64 || threads == 128 || threads == 256 || threads == 512 || threads == 1024,
         "threads per block: 64, 128, 256, 512 or 1024");
    Sim& m = S(s);
    m.col_block = threads;
    m.mark();
  });
}
// spatial-hash cell size (pipelines.rs:898-912 computes the default); a
// different cell changes which neighbours the self-collision passes see, so
// it is a physics setting, not a launch shape.  cell <= 0 restores the
// reference formula's value.
tc_status tc_set_hash_cell_size(tc_sim* s, float cell) {
  return guard([&] {
    Sim& m = S(s);
    need(std::isfinite(cell), "cell size must be finite");
    m.m.cell = cell > 0.f ? cell : m.cell_ref;
    m.ce_stale = true;  // the collider-edge grid uses the same cell
    m.mark();
  });
}

// ---- narrow-phase pair lists of the direct self-collision pass
tc_status tc_set_pair_recording(tc_sim* s, int enable, uint32_t max_vt_pairs, uint32_t max_ee_pairs) {
  return guard([&] {
    Sim& m = S(s);
    if (enable) {
      need(max_vt_pairs > 0 && max_ee_pairs > 0, "pair record capacities must be positive");
      m.rec_vt.alloc(max_vt_pairs);
      m.rec_ee.alloc(max_ee_pairs);
      m.rec_n.alloc(2);
      m.rec_vt_cap = max_vt_pairs;
      m.rec_ee_cap = max_ee_pairs;
      TC_CK(cudaMemsetAsync(m.rec_n.p, 0, 2 * sizeof(uint32_t), m.st));
    }
    m.rec_pairs = enable != 0;
    m.mark();
  });
}
tc_status tc_get_pair_lists(tc_sim* s, uint32_t* vt, uint32_t vt_capacity, uint32_t* ee, uint32_t ee_capacity,
                            uint32_t counts[2]) {
  return guard([&] {
    Sim& m = S(s);
    need(counts != nullptr, "counts required");
    need(m.rec_pairs, "pair recording is off (tc_set_pair_recording)");
    uint32_t c[2];
    TC_CK(cudaMemcpyAsync(c, m.rec_n.p, sizeof c, cudaMemcpyDeviceToHost, m.st));
    TC_CK(cudaStreamSynchronize(m.st));
    counts[0] = c[0];
    counts[1] = c[1];
    need(c[0] <= m.rec_vt_cap && c[1] <= m.rec_ee_cap,
         "the pair record overflowed its capacity; enable it again with larger capacities");
    need(vt_capacity >= c[0] || vt == nullptr, "vt output too small for the recorded pairs");
    need(ee_capacity >= c[1] || ee == nullptr, "ee output too small for the recorded pairs");
    if (vt && c[0]) {
      std::vector<std::array<uint32_t, 4>> h(c[0]);
      TC_CK(cudaMemcpy(h.data(), m.rec_vt.p, size_t(c[0]) * 16, cudaMemcpyDeviceToHost));
      for (auto& r : h) std::sort(r.begin() + 1, r.end());
      std::sort(h.begin(), h.end());
      std::memcpy(vt, h.data(), size_t(c[0]) * 16);
    }
    if (ee && c[1]) {
      std::vector<std::array<uint32_t, 2>> h(c[1]);
      TC_CK(cudaMemcpy(h.data(), m.rec_ee.p, size_t(c[1]) * 8, cudaMemcpyDeviceToHost));
      for (auto& r : h) std::sort(r.begin(), r.end());
      std::sort(h.begin(), h.end());
      std::memcpy(ee, h.data(), size_t(c[1]) * 8);
    }
  });
}

// ---- settings record (simulation/config_impl.rs, cloth_py lib.rs:3029-3047)
tc_status tc_set_workgroup_size(tc_sim* s, uint32_t wg) {
  return guard([&] { S(s).wg_size = wg == 64 ? 64u : 32u; });
}
tc_status tc_set_areal_density(tc_sim* s, float density) {
  return guard([&] {
    if (std::isfinite(density)) S(s).areal_density = std::min(std::max(density, 0.f), 100.f);
  });
}
tc_status tc_set_coupled_self_collision_options(tc_sim* s, uint32_t mode, uint32_t relaxation_iters) {
  return guard([&] {
    need(mode == 0, "coupled self-collision modes 1-3 are not built");
    S(s).relax_iters = relaxation_iters;
  });
}
tc_status tc_get_config_json(tc_sim* s, char* buf, size_t capacity, size_t* length) {
  return guard([&] {
    need(length != nullptr, "length required");
    const std::string j = tcloth::settings_json(S(s).settings());
    *length = j.size();
    if (buf && capacity) {
      const size_t k = std::min(j.size(), capacity - 1);
      std::memcpy(buf, j.data(), k);
      buf[k] = '\0';
    }
  });
}
tc_status tc_get_config_hash(tc_sim* s, uint64_t* hash) {
  return guard([&] {
    need(hash != nullptr, "hash required");
    *hash = tcloth::settings_hash(tcloth::settings_json(S(s).settings()));
  });
}

// ---- diagnostics of the latest self-collision pass: pairs handed to the
// deferred edge-edge CCD kernel, and the queue capacity
tc_status tc_get_ccd_queue(tc_sim* s, uint32_t out[2]) {
  return guard([&] {
    Sim& m = S(s);
    need(out != nullptr, "out required");
    uint32_t q = 0;
    if (m.ccd_n.p) {
      TC_CK(cudaMemcpyAsync(&q, m.ccd_n.p, sizeof q, cudaMemcpyDeviceToHost, m.st));
      TC_CK(cudaStreamSynchronize(m.st));
    }
    out[0] = q;
    out[1] = uint32_t(m.ccd_q.n);
  });
}

// ---- adaptive substeps and iterations (mod.rs:723-790, dispatch.rs:477-607)
tc_status tc_set_adaptive_substep_options(tc_sim* s, int enabled, uint32_t min_substeps, uint32_t max_substeps) {
  return guard([&] {
    Sim& m = S(s);
    if (enabled) m.adaptive_enable_buffers();
    m.ad.set_options(enabled != 0, min_substeps, max_substeps);
    m.mark();
  });
}
tc_status tc_set_auto_compensate_iterations(tc_sim* s, int enabled) {
  return guard([&] { S(s).ad.auto_compensate = enabled != 0; });
}
tc_status tc_set_strain_adaptive_options(tc_sim* s, int enabled, float tolerance) {
  return guard([&] { S(s).ad.set_strain_options(enabled != 0, tolerance); });
}
tc_status tc_note_external_displacement(tc_sim* s, float disp) {
  return guard([&] { S(s).ad.note_external(disp); });
}
tc_status tc_get_adaptive_state(tc_sim* s, float out[6]) {
  return guard([&] {
    Sim& m = S(s);
    need(out != nullptr, "out required");
    out[0] = float(m.ad.effective_substeps);
    out[1] = float(m.ad.effective_iterations > 0 ? m.ad.effective_iterations : m.iters);
    out[2] = m.ad.last_strain;
    out[3] = m.ad.last_max_disp;
    out[4] = m.ad.mesh_char_len;
    out[5] = float(m.ad.mesh_diameter_hops);
  });
}
// Pure evaluation of the decision rules, for tests: in = {enabled, min, max,
// base, previous effective substeps (0 = none), char length, thickness, gx,
// gy, gz, max displacement, external displacement, strain adaptive,
// tolerance, last strain, auto compensate, solver iterations, diameter hops};
// out = {effective substeps, effective iterations for iter_substeps substeps
// (0 = for the substeps just chosen)}.
tc_status tc_adaptive_eval(float dt, uint32_t requested, uint32_t iter_substeps, const float in[18], uint32_t out[2]) {
  return guard([&] {
    need(in != nullptr && out != nullptr, "in and out required");
    tcloth::AdaptiveCtl a;
    a.enabled = in[0] != 0.f;
    a.min_substeps = uint32_t(in[1]);
    a.max_substeps = uint32_t(in[2]);
    a.base_substeps = uint32_t(in[3]);
    a.effective_substeps = uint32_t(in[4]);
    a.mesh_char_len = in[5];
    a.cloth_thickness = in[6];
    const float g[3] = {in[7], in[8], in[9]};
    a.last_max_disp = in[10];
    a.pending_external = in[11];
    a.strain_adaptive = in[12] != 0.f;
    a.strain_tolerance = in[13];
    a.last_strain = in[14];
    a.auto_compensate = in[15] != 0.f;
    a.mesh_diameter_hops = uint32_t(in[17]);
    out[0] = a.substeps(dt, requested, g, 3);
    out[1] = a.iterations(uint32_t(in[16]), iter_substeps ? iter_substeps : out[0]);
  });
}

// ---- self-collision substep intervals (mod.rs:1071-1088)
tc_status tc_set_self_collision_substep_interval(tc_sim* s, uint32_t interval) {
  return guard([&] { Sim& m = S(s); m.sc_interval = std::max(interval, 1u); m.mark(); });
}
tc_status tc_set_self_collision_ee_substep_interval(tc_sim* s, uint32_t interval) {
  return guard([&] { Sim& m = S(s); m.ee_interval = interval; m.mark(); });
}
tc_status tc_get_self_collision_intervals(tc_sim* s, uint32_t out[2]) {
  return guard([&] {
    Sim& m = S(s);
    need(out != nullptr, "out required");
    out[0] = m.sc_interval;
    out[1] = m.ee_interval;
  });
}

// ---- learned warm start
uint32_t tc_ws_param_count(void) { return tcloth::kP_N; }

tc_status tc_ws_enable(tc_sim* s, int enable, uint32_t k_replaced, float res_thresh) {
  return guard([&] {
    Sim& m = S(s);
    if (!enable) { if (m.ws.on) m.mark(); m.ws.on = false; return; }
    need(m.can_persist(), "the warm start needs cooperative launch (persistent solver)");
    need(k_replaced >= 1 && k_replaced < m.iters, "k_replaced must be in [1, solver iterations - 1]");
    need(std::isfinite(res_thresh) || res_thresh > 0.f, "res_thresh must be a number or +inf");
    m.ws_setup();
    m.ws.on = true;
    m.ws.k = k_replaced;
    m.ws.res_thresh = res_thresh;
    m.mark();
  });
}

tc_status tc_ws_set_kernel(tc_sim* s, uint32_t kind) {
  return guard([&] {
    need(kind <= 1u, "kind: 0 (tcgen05) or 1 (mma.sync)");
    Sim& m = S(s);
    m.ws_setup();
    m.ws.net.tc = kind == 0u;
    m.mark();
  });
}

tc_status tc_ws_record(tc_sim* s, uint32_t capacity, uint32_t every) {
  return guard([&] {
    Sim& m = S(s);
    need(every >= 1, "every must be >= 1");
    m.ws_setup();
    const size_t n = m.n;
    if (capacity == 0) {  // stop recording, keep the snapshots
      m.ws.rec_cap = m.ws.rec_count;
      return;
    }
    {
      m.ws.rec_feat.alloc(size_t(capacity) * n * tcloth::kWsF);
      m.ws.rec_target.alloc(size_t(capacity) * n * 3);
      m.ws.rec_mask.alloc(size_t(capacity) * n);
    }
    m.ws.rec_cap = capacity;
    m.ws.rec_count = 0;
    m.ws.rec_every = every;
    m.ws.rec_phase = 0;
    TC_CK(cudaMemsetAsync(m.ws.dprev.p, 0, n * sizeof(float4), m.st));
    TC_CK(cudaStreamSynchronize(m.st));
  });
}

tc_status tc_ws_recorded(tc_sim* s, uint32_t* count) {
  return guard([&] { Sim& m = S(s); need(count != nullptr, "count required"); *count = m.ws.rec_count; });
}

tc_status tc_ws_train(tc_sim* s, uint32_t epochs, float lr, uint64_t seed, float* loss_first, float* loss_last) {
  return guard([&] {
    Sim& m = S(s);
    need(lr > 0.f && std::isfinite(lr), "lr must be positive");
    m.ws_train(epochs, lr, seed, loss_first, loss_last);
  });
}

tc_status tc_ws_get_params(tc_sim* s, float* out, size_t len) {
  return guard([&] {
    Sim& m = S(s);
    need(out != nullptr && len >= tcloth::kP_N, "output array too small");
    m.ws_setup();
    m.ws.net.get_params(out);
  });
}

tc_status tc_ws_set_params(tc_sim* s, const float* params, size_t len) {
  return guard([&] {
    Sim& m = S(s);
    need(params != nullptr && len == tcloth::kP_N, "params must hold tc_ws_param_count() floats");
    for (size_t i = 0; i < len; ++i) need(std::isfinite(params[i]), "params must be finite");
    m.ws_setup();
    m.ws.net.set_params(params);
    m.ws.normalized = true;
  });
}

tc_status tc_ws_set_relative_threshold(tc_sim* s, float ratio) {
  return guard([&] {
    Sim& m = S(s);
    need(std::isfinite(ratio) && ratio >= 0.f, "ratio must be finite and non-negative");
    m.ws.res_ratio = ratio;
    m.mark();
  });
}

tc_status tc_ws_stats(tc_sim* s, double out[4]) {
  return guard([&] {
    Sim& m = S(s);
    need(out != nullptr, "out required");
    unsigned int fb = 0;
    float rm = 0.f, rp = 0.f;
    if (m.ws.ready) {
      TC_CK(cudaMemcpyAsync(&fb, m.ws.fallbacks.p, sizeof fb, cudaMemcpyDeviceToHost, m.st));
      TC_CK(cudaMemcpyAsync(&rm, m.ws.res_max.p, sizeof rm, cudaMemcpyDeviceToHost, m.st));
      TC_CK(cudaMemcpyAsync(&rp, m.ws.res_pred.p, sizeof rp, cudaMemcpyDeviceToHost, m.st));
      TC_CK(cudaStreamSynchronize(m.st));
    }
    out[0] = double(m.ws.substeps_run);
    out[1] = double(fb);
    out[2] = double(rm);
    out[3] = m.ws.res_ratio > 0.f ? double(std::fmax(m.ws.res_ratio * rp, m.ws_res_floor())) : double(m.ws.res_thresh);
  });
}

tc_status tc_ws_reset_stats(tc_sim* s) {
  return guard([&] {
    Sim& m = S(s);
    m.ws.substeps_run = 0;
    if (m.ws.ready) {
      TC_CK(cudaMemsetAsync(m.ws.fallbacks.p, 0, sizeof(unsigned int), m.st));
      TC_CK(cudaStreamSynchronize(m.st));
    }
  });
}

tc_status tc_mlp_grad(uint32_t n, const float* feat, const uint32_t* adj_off, const uint32_t* adj_idx,
                      const float* target, const float* mask, const float* params, float* loss, float* grads,
                      float* y, float* y_infer, int device) {
  return guard([&] {
    need(n > 0 && feat && adj_off && target && mask && params && loss && grads && y, "all arrays are required");
    const uint32_t na = adj_off[n];
    need(na == 0 || adj_idx != nullptr, "adj_idx required");
    need(adj_off[0] == 0, "adj_off[0] must be 0");
    for (uint32_t i = 0; i < n; ++i) need(adj_off[i + 1] >= adj_off[i], "adj_off must be non-decreasing");
    for (uint32_t q = 0; q < na; ++q) need(adj_idx[q] < n, "adjacency index out of range");
    TC_CK(cudaSetDevice(device));
    cudaStream_t st = nullptr;
    TC_CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    struct StreamGuard { cudaStream_t s; ~StreamGuard() { cudaStreamSynchronize(s); cudaStreamDestroy(s); } } sg{st};
    tcloth::DBuf<uint32_t> d_off, d_idx;
    tcloth::DBuf<float> d_t, d_m, d_loss;
    tcloth::DBuf<__nv_bfloat16> d_f;
    std::vector<__nv_bfloat16> hf(size_t(n) * tcloth::kWsF);
    for (size_t e = 0; e < hf.size(); ++e) hf[e] = __float2bfloat16(feat[e]);
    d_off.upload(adj_off, n + 1, st);
    d_idx.upload(adj_idx, na, st);
    d_t.upload(target, size_t(n) * 3, st);
    d_m.upload(mask, n, st);
    d_f.upload(hf, st);
    d_loss.alloc(1);
    TC_CK(cudaMemsetAsync(d_loss.p, 0, sizeof(float), st));
    tcloth::Mlp net;
    net.setup(st, n, d_off.p, d_idx.p);
    net.set_ell(adj_off, adj_idx);
    net.alloc_train();
    net.set_params(params);
    tcloth::DBuf<int> d_err;
    d_err.alloc(1);
    TC_CK(cudaMemsetAsync(d_err.p, 0, sizeof(int), st));
    net.err = d_err.p;
    net.forward(d_f.p, true, d_t.p, d_m.p, d_loss.p);
    net.backward();
    TC_CK(cudaMemcpyAsync(loss, d_loss.p, sizeof(float), cudaMemcpyDeviceToHost, st));
    TC_CK(cudaMemcpyAsync(grads, net.gw.p, tcloth::kP_N * sizeof(float), cudaMemcpyDeviceToHost, st));
    TC_CK(cudaMemcpyAsync(y, net.y.p, size_t(n) * 3 * sizeof(float), cudaMemcpyDeviceToHost, st));
    tcloth::DBuf<float> d_yi;
    if (y_infer) {
      d_yi.alloc(size_t(n) * 3);
      net.infer(d_f.p, nullptr, nullptr, d_yi.p, nullptr, nullptr, nullptr);
      TC_CK(cudaMemcpyAsync(y_infer, d_yi.p, size_t(n) * 3 * sizeof(float), cudaMemcpyDeviceToHost, st));
    }
    int herr = 0;
    TC_CK(cudaMemcpyAsync(&herr, d_err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    TC_CK(cudaStreamSynchronize(st));
    if (herr) throw TcError(TC_ERR_TIMEOUT, "a tensor-core completion wait of the network timed out");
    TC_CK(cudaGetLastError());
  });
}

}  // extern "C"

// ===================================================================
// Spatial-hash build without any allocation
// ===================================================================
// For callers that cannot allocate device memory themselves: a host
// application that owns every device buffer through its own allocator (for
// example a DCC tool or game-engine plugin), a thread that must not call
// cudaMalloc / cudaFree because they synchronise the device, or a
// memory-capped service.  Their scratch space is this file-scope array,
// sized for the largest cloth the reference's hash supports (its table is
// capped at 65,536 buckets); every GPU that loads the library holds it
// (about 1.6 MB) until the process exits.
namespace {
constexpr uint32_t kStaticMaxElems = 262144;  // vertices (or edges) per call
constexpr uint32_t kStaticMaxTable = 65536;   // hash buckets per call
constexpr uint32_t kStaticTiles = kStaticMaxTable / 1024;
struct StaticHashScratch {
  uint32_t keys[kStaticMaxElems];
  uint32_t counts[kStaticMaxTable + 1];
  uint32_t cursor[kStaticMaxTable + 1];
  uint32_t tile_sum[kStaticTiles];
};
}  // namespace
static __device__ __align__(256) StaticHashScratch g_static_hash_scratch;

// bucket key of each position (the count pass of spatial_grid_sort.wgsl:44-52)
__global__ void k_static_hash_count(uint32_t n, const float4* __restrict__ pos, float cell, uint32_t table,
                                    uint32_t* __restrict__ keys, uint32_t* __restrict__ counts) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const tcloth::I3 c = tcloth::cell_of(tcloth::mk(pos[i]), cell);
  const uint32_t h = tcloth::hash3(c.x, c.y, c.z, table);
  keys[i] = h;
  atomicAdd(&counts[h], 1u);
}

static StaticHashScratch* static_scratch_for_current_device() {
  // One device address per device, looked up on the first call with that
  // device current (the host-side name of the array is not a device address).
  // Threads making their first call on one device at the same time both look
  // the address up and publish the same value; the atomics make that a
  // well-defined race.  The address belongs to the device's primary context:
  // after a reset of that context (cudaDeviceReset) the library must be used
  // from a fresh process.
  static std::atomic<StaticHashScratch*> ptrs[64] = {};
  int dev = 0;
  TC_CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) throw TcError(TC_ERR_CUDA, "device index out of range for the static scratch table");
  StaticHashScratch* cached = ptrs[dev].load(std::memory_order_acquire);
  if (!cached) {
    void* p = nullptr;
    TC_CK(cudaGetSymbolAddress(&p, g_static_hash_scratch));
    cached = static_cast<StaticHashScratch*>(p);
    ptrs[dev].store(cached, std::memory_order_release);
  }
  return cached;
}

extern "C" tc_status tc_hash_build_static(const float* positions, uint32_t n, float cell_size, uint32_t table_size,
                                          uint32_t* cell_starts, uint32_t* sorted, void* stream) {
  return guard([&] {
    need(n <= kStaticMaxElems, "tc_hash_build_static: n exceeds the static scratch limit of 262144 elements");
    need(table_size >= 1024 && table_size <= kStaticMaxTable,
         "tc_hash_build_static: table_size must be in [1024, 65536]");
    need(cell_size > 0.f, "tc_hash_build_static: cell_size must be positive");
    need(cell_starts != nullptr && (sorted != nullptr || n == 0) && (positions != nullptr || n == 0),
         "tc_hash_build_static: positions, cell_starts and sorted are required");
    need(reinterpret_cast<uintptr_t>(positions) % 16 == 0,
         "tc_hash_build_static: positions must be 16-byte aligned (rows of 4 floats read as float4)");
    StaticHashScratch* sc = static_scratch_for_current_device();
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const float4* pos = reinterpret_cast<const float4*>(positions);
    const uint32_t T = table_size;
    // the array keeps the previous call's contents: zero what must start at zero
    TC_CK(cudaMemsetAsync(sc->counts, 0, (T + 1) * sizeof(uint32_t), st));
    TC_CK(cudaMemsetAsync(sc->cursor, 0, (T + 1) * sizeof(uint32_t), st));
    if (n) k_static_hash_count<<<(n + 255) / 256, 256, 0, st>>>(n, pos, cell_size, T, sc->keys, sc->counts);
    const uint32_t ntiles = (T + 1023) / 1024;
    tcloth::k_scan_blocks<<<ntiles, 1024, 0, st>>>(T, sc->counts, cell_starts, sc->tile_sum);
    tcloth::k_scan_finish<<<ntiles, 1024, 0, st>>>(T, ntiles, sc->tile_sum, cell_starts);
    if (n) tcloth::k_hash_scatter<<<(n + 255) / 256, 256, 0, st>>>(n, sc->keys, cell_starts, sc->cursor, sorted);
    tcloth::k_hash_sort_buckets<<<(T + 255) / 256, 256, 0, st>>>(T, cell_starts, sorted);
    TC_CK(cudaGetLastError());
  });
}
