// Learned warm start: a graph MLP that predicts each vertex's constraint
// correction for the coming substep (new; no counterpart in the reference).
//
// Network (per vertex i, neighbours N(i) from the adjacency CSR):
//   X0 = features_i (16, bf16)
//   H0 = SiLU(X0 W0 + b0)                              64
//   X1 = [H0_i, mean_{j in N(i)} H0_j]  (bf16)         128
//   H1 = SiLU(X1 W1 + b1)                              64
//   X2 = [H1_i, mean_{j in N(i)} H1_j]                 128
//   H2 = SiLU(X2 W2 + b2)                              64
//   Y  = H2 W3 + b3                                    3 (fp32)
// Weights are bf16 for the tensor cores (fp32 master copies for Adam),
// every product accumulates in fp32 (mma.sync.m16n8k16 .bf16 -> .f32).
// Rounding points (mirrored by the CPU reference of the tests): features,
// weights, H and the neighbour means are rounded to bf16; Z, dY and all
// gradient accumulations stay fp32; dZ is rounded to bf16 before its GEMMs.
#pragma once
#include <cuda_bf16.h>

#include "vmath.cuh"

namespace tcloth {

constexpr int kWsF = 16;   // input features
constexpr int kWsH = 64;   // hidden width
constexpr int kWsRows = 64;  // vertices per block tile (4 warps x 16 rows)

// fp32 parameter blob: weights row-major [in][out], then the bias
constexpr uint32_t kP_W0 = 0, kP_b0 = 1024, kP_W1 = 1088, kP_b1 = 9280, kP_W2 = 9344, kP_b2 = 17536,
                   kP_W3 = 17600, kP_b3 = 17792, kP_N = 17795;
// transposed bf16 copies [out][in] of W0..W2 for the forward GEMM's B operand
constexpr uint32_t kT_W0 = 0, kT_W1 = 1024, kT_W2 = 9216, kT_N = 17408;

__device__ __forceinline__ float silu(float z) { return z / (1.0f + expf(-z)); }
__device__ __forceinline__ float silu_grad(float z) {
  const float s = 1.0f / (1.0f + expf(-z));
  return s * (1.0f + z * (1.0f - s));
}

__device__ __forceinline__ uint32_t pack_bf16(__nv_bfloat16 lo, __nv_bfloat16 hi) {
  return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

// D(16x8, f32) += A(16x16, bf16, row) * B(16x8, bf16, col)
__device__ __forceinline__ void mma_bf16_16816(float d[4], const uint32_t a[4], const uint32_t b[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// Fragments from shared memory.  A is row-major [row][k] (ld in elements),
// Bt is n-major [n][k]: element (k, n) of B at Bt[n * ld + k].
__device__ __forceinline__ void load_a_frag(uint32_t a[4], const __nv_bfloat16* A, int ld, int row0, int k0, int lane) {
  const int g = lane >> 2, t = lane & 3;
  const __nv_bfloat16* r0 = A + (row0 + g) * ld + k0 + 2 * t;
  const __nv_bfloat16* r1 = A + (row0 + g + 8) * ld + k0 + 2 * t;
  a[0] = *reinterpret_cast<const uint32_t*>(r0);
  a[1] = *reinterpret_cast<const uint32_t*>(r1);
  a[2] = *reinterpret_cast<const uint32_t*>(r0 + 8);
  a[3] = *reinterpret_cast<const uint32_t*>(r1 + 8);
}
__device__ __forceinline__ void load_b_frag(uint32_t b[2], const __nv_bfloat16* Bt, int ld, int n0, int k0, int lane) {
  const int g = lane >> 2, t = lane & 3;
  const __nv_bfloat16* c = Bt + (n0 + g) * ld + k0 + 2 * t;
  b[0] = *reinterpret_cast<const uint32_t*>(c);
  b[1] = *reinterpret_cast<const uint32_t*>(c + 8);
}
// A^T fragment where the stored matrix is S[k][m] (row-major, ld): A(m, k) = S[k][m].
__device__ __forceinline__ void load_at_frag(uint32_t a[4], const __nv_bfloat16* S, int ld, int m0, int k0, int lane) {
  const int g = lane >> 2, t = lane & 3;
  auto at = [&](int m, int k) { return S[k * ld + m]; };
  a[0] = pack_bf16(at(m0 + g, k0 + 2 * t), at(m0 + g, k0 + 2 * t + 1));
  a[1] = pack_bf16(at(m0 + g + 8, k0 + 2 * t), at(m0 + g + 8, k0 + 2 * t + 1));
  a[2] = pack_bf16(at(m0 + g, k0 + 2 * t + 8), at(m0 + g, k0 + 2 * t + 9));
  a[3] = pack_bf16(at(m0 + g + 8, k0 + 2 * t + 8), at(m0 + g + 8, k0 + 2 * t + 9));
}
// B fragment where the stored matrix is S[k][n] (row-major, ld): B(k, n) = S[k][n].
__device__ __forceinline__ void load_bk_frag(uint32_t b[2], const __nv_bfloat16* S, int ld, int n0, int k0, int lane) {
  const int g = lane >> 2, t = lane & 3;
  b[0] = pack_bf16(S[(k0 + 2 * t) * ld + n0 + g], S[(k0 + 2 * t + 1) * ld + n0 + g]);
  b[1] = pack_bf16(S[(k0 + 2 * t + 8) * ld + n0 + g], S[(k0 + 2 * t + 9) * ld + n0 + g]);
}

struct MlpLayerArgs {
  uint32_t n;
  int kin;                      // 16 (layer 0) or 128 (message-passing layers)
  const __nv_bfloat16* x_feat;  // layer 0 input [n][16]
  const __nv_bfloat16* h_prev;  // rounds: previous hidden [n][64]
  const uint32_t* adj_off;
  const uint32_t* adj_idx;
  const __nv_bfloat16* wt;      // [64][kin] (transposed weights)
  const float* bias;            // [64]
  __nv_bfloat16* x_out;         // optional: the assembled input [n][kin] (training)
  float* z_out;                 // optional: pre-activations [n][64] (training)
  __nv_bfloat16* h_out;         // [n][64], or null when the head is fused
  // fused head (inference, last layer): Y = H W3 + b3, then p += Y L on
  // free vertices (x4.w > 0) when p4 is given, else Y to y_out
  const __nv_bfloat16* w3;      // [64][3] or null
  const float* b3;
  float* y_out;
  const float4* x4;
  float4* p4;
  const float* local_len;
};

__device__ __forceinline__ void bf16x8_to_f32(const uint4 u, float f[8]) {
  const uint32_t w[4] = {u.x, u.y, u.z, u.w};
  for (int q = 0; q < 4; ++q) {
    f[2 * q] = __uint_as_float(w[q] << 16);
    f[2 * q + 1] = __uint_as_float(w[q] & 0xFFFF0000u);
  }
}
__device__ __forceinline__ uint4 f32_to_bf16x8(const float f[8]) {
  uint32_t w[4];
  for (int q = 0; q < 4; ++q) w[q] = pack_bf16(__float2bfloat16(f[2 * q]), __float2bfloat16(f[2 * q + 1]));
  return make_uint4(w[0], w[1], w[2], w[3]);
}

// One layer forward: assemble the 64-row input tile (features, or self +
// neighbour mean; 16-byte loads of 8 bf16, four neighbours in flight), with
// 256 threads; then 4 warps multiply by W on the tensor cores (mma.sync
// m16n8k16, fp32 accumulators), add bias, SiLU; the output tile is staged in
// shared memory and stored with 16-byte stores.
constexpr int kWsFwdThreads = 256;
__global__ void __launch_bounds__(kWsFwdThreads) k_mlp_layer_fwd(MlpLayerArgs a) {
  __shared__ __align__(16) __nv_bfloat16 xs[kWsRows][128 + 8];
  __shared__ __align__(16) __nv_bfloat16 ws[kWsH][128 + 8];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t row0 = blockIdx.x * kWsRows;
  const int kin = a.kin, kv = kin / 8;  // 16-byte vectors per row
  for (int e = tid; e < kWsH * kv; e += blockDim.x)
    *reinterpret_cast<uint4*>(&ws[e / kv][(e % kv) * 8]) = __ldg(reinterpret_cast<const uint4*>(a.wt) + e);
  if (kin == kWsF) {
    for (int e = tid; e < kWsRows * 2; e += blockDim.x) {
      const int r = e >> 1, c = (e & 1) * 8;
      const uint32_t v = row0 + r;
      *reinterpret_cast<uint4*>(&xs[r][c]) =
          v < a.n ? __ldg(reinterpret_cast<const uint4*>(a.x_feat + size_t(v) * kWsF + c)) : make_uint4(0, 0, 0, 0);
    }
  } else {
    // self part and neighbour mean; each thread owns (row, 8-column group)
    for (int e = tid; e < kWsRows * 8; e += blockDim.x) {
      const int r = e >> 3, cg = (e & 7) * 8;
      const uint32_t v = row0 + r;
      uint4 self = make_uint4(0, 0, 0, 0), mean = make_uint4(0, 0, 0, 0);
      if (v < a.n) {
        self = __ldg(reinterpret_cast<const uint4*>(a.h_prev + size_t(v) * kWsH + cg));
        float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        const uint32_t b = __ldg(a.adj_off + v), en = __ldg(a.adj_off + v + 1);
        auto row = [&](uint32_t j) { return __ldg(reinterpret_cast<const uint4*>(a.h_prev + size_t(j) * kWsH + cg)); };
        auto add = [&](const uint4 u) {
          float f[8];
          bf16x8_to_f32(u, f);
#pragma unroll
          for (int c = 0; c < 8; ++c) acc[c] += f[c];
        };
        uint32_t q = b;
        for (; q + 4 <= en; q += 4) {  // same summation order as one at a time
          const uint32_t j0 = __ldg(a.adj_idx + q), j1 = __ldg(a.adj_idx + q + 1), j2 = __ldg(a.adj_idx + q + 2),
                         j3 = __ldg(a.adj_idx + q + 3);
          const uint4 u0 = row(j0), u1 = row(j1), u2 = row(j2), u3 = row(j3);
          add(u0);
          add(u1);
          add(u2);
          add(u3);
        }
        for (; q < en; ++q) add(row(__ldg(a.adj_idx + q)));
        const float inv = en > b ? 1.0f / float(en - b) : 0.0f;
        for (int c = 0; c < 8; ++c) acc[c] *= inv;
        mean = f32_to_bf16x8(acc);
      }
      *reinterpret_cast<uint4*>(&xs[r][cg]) = self;
      *reinterpret_cast<uint4*>(&xs[r][kWsH + cg]) = mean;
    }
  }
  __syncthreads();
  if (a.x_out) {
    for (int e = tid; e < kWsRows * kv; e += blockDim.x) {
      const int r = e / kv, c = (e % kv) * 8;
      if (row0 + r < a.n) *reinterpret_cast<uint4*>(a.x_out + size_t(row0 + r) * kin + c) = *reinterpret_cast<const uint4*>(&xs[r][c]);
    }
  }
  if (a.x_out) __syncthreads();  // the epilogue below rewrites xs rows
  if (warp >= kWsRows / 16) return;  // 4 warps x 16 rows do the products
  float acc[8][4];
#pragma unroll
  for (int nt = 0; nt < 8; ++nt)
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[nt][q] = 0.f;
  for (int k0 = 0; k0 < kin; k0 += 16) {
    uint32_t af[4];
    load_a_frag(af, &xs[0][0], 128 + 8, warp * 16, k0, lane);
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      uint32_t bf[2];
      load_b_frag(bf, &ws[0][0], 128 + 8, nt * 8, k0, lane);
      mma_bf16_16816(acc[nt], af, bf);
    }
  }
  const int g = lane >> 2, t = lane & 3;
  float y0[3] = {0.f, 0.f, 0.f}, y1[3] = {0.f, 0.f, 0.f};  // fused head partials, rows g and g + 8
  // the epilogue overwrites this warp's own 16 rows of xs only
  __syncwarp();
#pragma unroll
  for (int nt = 0; nt < 8; ++nt)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int r = warp * 16 + g + (q >> 1) * 8, c = nt * 8 + 2 * t + (q & 1);
      const uint32_t v = row0 + r;
      const float z = acc[nt][q] + __ldg(a.bias + c);
      if (a.z_out && v < a.n) a.z_out[size_t(v) * kWsH + c] = z;
      const __nv_bfloat16 h = __float2bfloat16(silu(z));
      xs[r][c] = h;
      if (a.w3) {
        const float hf = __bfloat162float(h);
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          const float wv = __bfloat162float(a.w3[c * 3 + j]);
          if (q >> 1) y1[j] += hf * wv;
          else y0[j] += hf * wv;
        }
      }
    }
  __syncwarp();
  if (a.w3) {
    for (int j = 0; j < 3; ++j) {
      y0[j] += __shfl_xor_sync(0xffffffffu, y0[j], 1);
      y0[j] += __shfl_xor_sync(0xffffffffu, y0[j], 2);
      y1[j] += __shfl_xor_sync(0xffffffffu, y1[j], 1);
      y1[j] += __shfl_xor_sync(0xffffffffu, y1[j], 2);
    }
    if (t < 2) {
      const uint32_t v = row0 + warp * 16 + g + t * 8;
      if (v < a.n) {
        const float Y[3] = {(t ? y1[0] : y0[0]) + a.b3[0], (t ? y1[1] : y0[1]) + a.b3[1],
                            (t ? y1[2] : y0[2]) + a.b3[2]};
        if (a.y_out)
          for (int j = 0; j < 3; ++j) a.y_out[size_t(v) * 3 + j] = Y[j];
        if (a.p4 && a.x4[v].w > 0.f) {
          const float L = fmaxf(a.local_len[v], 1e-6f);
          float4 p = a.p4[v];
          p.x += Y[0] * L;
          p.y += Y[1] * L;
          p.z += Y[2] * L;
          a.p4[v] = p;
        }
      }
    }
  }
  if (a.h_out) {
    for (int e = lane; e < 16 * 8; e += 32) {
      const int r = warp * 16 + (e >> 3), c = (e & 7) * 8;
      if (row0 + r < a.n)
        *reinterpret_cast<uint4*>(a.h_out + size_t(row0 + r) * kWsH + c) = *reinterpret_cast<const uint4*>(&xs[r][c]);
    }
  }
}

// Head: Y = H2 W3 + b3 (fp32 accumulation of bf16 products).  With targets,
// also dY = 2 (Y - T) m / (3 M) (mean squared error over the M free vertices,
// mask m) and the loss.
__global__ void k_mlp_head(uint32_t n, const __nv_bfloat16* __restrict__ h2, const __nv_bfloat16* __restrict__ w3,
                           const float* __restrict__ b3, float* __restrict__ y, const float* __restrict__ target,
                           const float* __restrict__ mask, float inv_count, float* __restrict__ dy,
                           float* __restrict__ loss) {
  const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  float l = 0.f;
  if (v < n) {
    for (int c = 0; c < 3; ++c) {
      float s = 0.f;
      for (int k = 0; k < kWsH; ++k) s += __bfloat162float(h2[size_t(v) * kWsH + k]) * __bfloat162float(w3[k * 3 + c]);
      s += b3[c];
      y[size_t(v) * 3 + c] = s;
      if (target) {
        const float m = mask ? mask[v] : 1.0f;
        const float d = (s - target[size_t(v) * 3 + c]) * m;
        dy[size_t(v) * 3 + c] = 2.0f * d * inv_count / 3.0f;
        l += d * d;
      }
    }
  }
  if (target) {
    for (int o = 16; o > 0; o >>= 1) l += __shfl_down_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, l * inv_count / 3.0f);
  }
}

// Head backward: dH2 = dY W3^T (fp32), dW3 += H2^T dY, db3 += sum dY.
__global__ void k_mlp_head_bwd(uint32_t n, const __nv_bfloat16* __restrict__ h2, const __nv_bfloat16* __restrict__ w3,
                               const float* __restrict__ dy, float* __restrict__ dh2, float* __restrict__ dw3,
                               float* __restrict__ db3) {
  __shared__ float s_dw[kWsH * 3];
  __shared__ float s_db[3];
  for (int e = threadIdx.x; e < kWsH * 3; e += blockDim.x) s_dw[e] = 0.f;
  if (threadIdx.x < 3) s_db[threadIdx.x] = 0.f;
  __syncthreads();
  const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v < n) {
    const float d0 = dy[size_t(v) * 3], d1 = dy[size_t(v) * 3 + 1], d2 = dy[size_t(v) * 3 + 2];
    for (int k = 0; k < kWsH; ++k) {
      const float w0 = __bfloat162float(w3[k * 3]), w1 = __bfloat162float(w3[k * 3 + 1]), w2 = __bfloat162float(w3[k * 3 + 2]);
      dh2[size_t(v) * kWsH + k] = d0 * w0 + d1 * w1 + d2 * w2;
      const float h = __bfloat162float(h2[size_t(v) * kWsH + k]);
      atomicAdd(&s_dw[k * 3], h * d0);
      atomicAdd(&s_dw[k * 3 + 1], h * d1);
      atomicAdd(&s_dw[k * 3 + 2], h * d2);
    }
    atomicAdd(&s_db[0], d0);
    atomicAdd(&s_db[1], d1);
    atomicAdd(&s_db[2], d2);
  }
  __syncthreads();
  for (int e = threadIdx.x; e < kWsH * 3; e += blockDim.x) atomicAdd(&dw3[e], s_dw[e]);
  if (threadIdx.x < 3) atomicAdd(&db3[threadIdx.x], s_db[threadIdx.x]);
}

// dZ = dH * SiLU'(Z), rounded to bf16 for the tensor-core GEMMs; db += sum dZ.
__global__ void k_mlp_act_bwd(uint32_t n, const float* __restrict__ dh, const float* __restrict__ z,
                              __nv_bfloat16* __restrict__ dz, float* __restrict__ db) {
  __shared__ float s_db[kWsH];
  if (threadIdx.x < kWsH) s_db[threadIdx.x] = 0.f;
  __syncthreads();
  const size_t e = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e < size_t(n) * kWsH) {
    const float g = dh[e] * silu_grad(z[e]);
    dz[e] = __float2bfloat16(g);
    atomicAdd(&s_db[e % kWsH], g);
  }
  __syncthreads();
  if (threadIdx.x < kWsH) atomicAdd(&db[threadIdx.x], s_db[threadIdx.x]);
}

// Weight gradient dW[kin][64] += X^T dZ over a 64-row tile (tensor cores),
// and input gradient dX[n][kin] = dZ W^T.
struct MlpBwdArgs {
  uint32_t n;
  int kin;
  const __nv_bfloat16* x;    // [n][kin]
  const __nv_bfloat16* dz;   // [n][64]
  const __nv_bfloat16* w;    // [kin][64] (row-major weights = n-major for dZ W^T)
  float* dw;                 // [kin][64]
  float* dx;                 // [n][kin] or null
};
__global__ void __launch_bounds__(128) k_mlp_layer_bwd(MlpBwdArgs a) {
  __shared__ __align__(16) __nv_bfloat16 xs[kWsRows][128 + 8];
  __shared__ __align__(16) __nv_bfloat16 ds[kWsRows][kWsH + 8];
  __shared__ __align__(16) __nv_bfloat16 wsm[128][kWsH + 8];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t row0 = blockIdx.x * kWsRows;
  const int kin = a.kin;
  for (int e = tid; e < kWsRows * kin; e += blockDim.x) {
    const int r = e / kin, c = e % kin;
    xs[r][c] = row0 + r < a.n ? a.x[size_t(row0 + r) * kin + c] : __float2bfloat16(0.f);
  }
  for (int e = tid; e < kWsRows * kWsH; e += blockDim.x) {
    const int r = e / kWsH, c = e % kWsH;
    ds[r][c] = row0 + r < a.n ? a.dz[size_t(row0 + r) * kWsH + c] : __float2bfloat16(0.f);
  }
  for (int e = tid; e < kin * kWsH; e += blockDim.x) wsm[e / kWsH][e % kWsH] = a.w[e];
  __syncthreads();
  const int g = lane >> 2, t = lane & 3;
  // dW: M = kin (16-row tiles over warps), N = 64, K = 64 rows of the tile
  for (int mt = warp; mt < kin / 16; mt += 4) {
    float acc[8][4];
    for (int nt = 0; nt < 8; ++nt)
      for (int q = 0; q < 4; ++q) acc[nt][q] = 0.f;
    for (int k0 = 0; k0 < kWsRows; k0 += 16) {
      uint32_t af[4];
      load_at_frag(af, &xs[0][0], 128 + 8, mt * 16, k0, lane);
      for (int nt = 0; nt < 8; ++nt) {
        uint32_t bf[2];
        load_bk_frag(bf, &ds[0][0], kWsH + 8, nt * 8, k0, lane);
        mma_bf16_16816(acc[nt], af, bf);
      }
    }
    for (int nt = 0; nt < 8; ++nt)
      for (int q = 0; q < 4; ++q) {
        const int r = mt * 16 + g + (q >> 1) * 8, c = nt * 8 + 2 * t + (q & 1);
        atomicAdd(&a.dw[r * kWsH + c], acc[nt][q]);
      }
  }
  if (!a.dx) return;
  // dX: M = 64 rows (16 per warp), N = kin, K = 64
  for (int nt = 0; nt < kin / 8; ++nt) {
    float acc[4] = {0.f, 0.f, 0.f, 0.f};
    for (int k0 = 0; k0 < kWsH; k0 += 16) {
      uint32_t af[4], bf[2];
      load_a_frag(af, &ds[0][0], kWsH + 8, warp * 16, k0, lane);
      load_b_frag(bf, &wsm[0][0], kWsH + 8, nt * 8, k0, lane);
      mma_bf16_16816(acc, af, bf);
    }
    for (int q = 0; q < 4; ++q) {
      const int r = warp * 16 + g + (q >> 1) * 8, c = nt * 8 + 2 * t + (q & 1);
      if (row0 + r < a.n) a.dx[size_t(row0 + r) * kin + c] = acc[q];
    }
  }
}

// dH_prev[j] = dX[j][0:64] + sum_{i in N(j)} dX[i][64:128] / deg(i)
// (the adjacency is symmetric, so the transpose of the mean is a gather).
__global__ void k_mlp_agg_bwd(uint32_t n, const float* __restrict__ dx, const uint32_t* __restrict__ adj_off,
                              const uint32_t* __restrict__ adj_idx, float* __restrict__ dh_prev) {
  const size_t e = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= size_t(n) * kWsH) return;
  const uint32_t j = uint32_t(e / kWsH), c = uint32_t(e % kWsH);
  float s = dx[size_t(j) * 128 + c];
  for (uint32_t q = adj_off[j]; q < adj_off[j + 1]; ++q) {
    const uint32_t i = adj_idx[q];
    const uint32_t deg = adj_off[i + 1] - adj_off[i];
    s += dx[size_t(i) * 128 + kWsH + c] / float(deg);
  }
  dh_prev[e] = s;
}

// Adam on fp32 master weights; refreshes the bf16 copy (optionally transposed
// [cols][rows] for the forward GEMM's n-major B operand).
__global__ void k_adam(uint32_t cnt, float* __restrict__ w, const float* __restrict__ gw, float* __restrict__ m,
                       float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2,
                       __nv_bfloat16* __restrict__ wb, __nv_bfloat16* __restrict__ wbt, uint32_t rows, uint32_t cols) {
  const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= cnt) return;
  const float g = gw[e];
  const float mm = b1 * m[e] + (1.0f - b1) * g;
  const float vv = b2 * v[e] + (1.0f - b2) * g * g;
  m[e] = mm;
  v[e] = vv;
  const float nw = w[e] - lr * (mm / c1) / (sqrtf(vv / c2) + eps);
  w[e] = nw;
  if (wb) wb[e] = __float2bfloat16(nw);
  if (wbt) wbt[(e % cols) * rows + e / cols] = __float2bfloat16(nw);
}

// bf16 copies of the fp32 master blob (row-major, and transposed W0..W2)
__global__ void k_ws_refresh(const float* __restrict__ w, __nv_bfloat16* __restrict__ wb,
                             __nv_bfloat16* __restrict__ wbt) {
  const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= kP_N) return;
  const __nv_bfloat16 b = __float2bfloat16(w[e]);
  wb[e] = b;
  if (e < kP_b0) wbt[kT_W0 + (e % kWsH) * kWsF + e / kWsH] = b;
  else if (e >= kP_W1 && e < kP_b1) { const uint32_t q = e - kP_W1; wbt[kT_W1 + (q % kWsH) * 128 + q / kWsH] = b; }
  else if (e >= kP_W2 && e < kP_b2) { const uint32_t q = e - kP_W2; wbt[kT_W2 + (q % kWsH) * 128 + q / kWsH] = b; }
}

}  // namespace tcloth

namespace tcloth {

// Per-vertex input features, all lengths divided by the vertex's local edge
// length L (local_len): previous substep's constraint correction, the first
// Jacobi move of the edge constraints around the vertex (gathered over the
// adjacency with rest lengths), the signed distance and normal to the nearest
// primitive collider, velocity * dt, |g| dt^2, a free-vertex flag and a bias.
struct WsFeatArgs {
  uint32_t n;
  const float4* x4;
  const float4* p4;
  const float4* v4;
  const float4* dprev;      // previous substep's correction (p_iter - p_pred)
  const float* local_len;
  const uint32_t* adj_off;
  const uint32_t* adj_idx;
  const float* adj_rest;    // rest length of each adjacency entry
  const Prim* prims;
  uint32_t nprims;
  const uint32_t* vinst;     // batched instances: vertex -> instance (or null)
  const uint2* inst_prims;   // instance -> (first primitive, count)
  float dt, g_dt2;
  __nv_bfloat16* feat;      // [n][16]
};
__device__ __forceinline__ float prim_sdf(const Prim& c, V3 p, V3& nrm) {
  const uint32_t type = __float_as_uint(c.h.w);
  if (type == 0u) {
    const V3 d = p - mk(c.a);
    const float l = length(d);
    nrm = l > kEps ? d / l : mk(0.f, 1.f, 0.f);
    return l - c.h.z;
  }
  if (type == 1u) {
    const V3 A = mk(c.a), ab = mk(c.b) - A;
    const float l2 = dot(ab, ab);
    const float t = l2 > kEps ? clampf(dot(p - A, ab) / l2, 0.f, 1.f) : 0.f;
    const V3 d = p - (A + ab * t);
    const float l = length(d);
    nrm = l > kEps ? d / l : mk(0.f, 1.f, 0.f);
    return l - c.h.z;
  }
  const V3 B = mk(c.b);
  nrm = B / length(B);
  return dot(p - mk(c.a), nrm);
}
__global__ void k_ws_features(WsFeatArgs a) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const float4 xi4 = a.x4[i], pi4 = a.p4[i], vi4 = a.v4[i];
  const V3 pi = mk(pi4);
  const float wi = xi4.w;
  const float L = fmaxf(a.local_len[i], 1e-6f);
  const float invL = 1.0f / L;
  const float4 dp = a.dprev[i];
  V3 jac = mk(0.f, 0.f, 0.f);
  for (uint32_t q = a.adj_off[i]; q < a.adj_off[i + 1]; ++q) {
    const uint32_t j = a.adj_idx[q];
    const float4 pj4 = a.p4[j];
    const float wj = a.x4[j].w;
    const V3 d = pi - mk(pj4);
    const float dl = length(d);
    const float ws = wi + wj;
    if (dl > kEps && ws > kEps) jac = jac + d * ((a.adj_rest[q] - dl) / dl * (wi / ws));
  }
  float sdf = 1.0f;
  V3 n = mk(0.f, 0.f, 0.f);
  uint32_t kb = 0, ke = a.nprims;
  if (a.vinst) {
    const uint2 r = a.inst_prims[a.vinst[i]];
    kb = r.x;
    ke = r.x + r.y;
  }
  for (uint32_t k = kb; k < ke; ++k) {
    V3 nk;
    const float s = (prim_sdf(a.prims[k], pi, nk) - pi4.w) * invL;
    if (k == kb || s < sdf) { sdf = s; n = nk; }
  }
  sdf = clampf(sdf, -4.f, 4.f);
  float f[kWsF] = {dp.x * invL, dp.y * invL, dp.z * invL, jac.x * invL, jac.y * invL, jac.z * invL, sdf,
                   n.x, n.y, n.z, vi4.x * a.dt * invL, vi4.y * a.dt * invL, vi4.z * a.dt * invL,
                   a.g_dt2 * invL, wi > 0.f ? 1.f : 0.f, 1.f};
  for (int c = 0; c < kWsF; ++c) a.feat[size_t(i) * kWsF + c] = __float2bfloat16(f[c]);
}

__global__ void k_copy4(uint32_t n, const float4* __restrict__ src, float4* __restrict__ dst) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = src[i];
}
// correction of this substep's iterations: dprev = p - p_pred; optional
// training target (dprev / L) and mask (free vertex).
__global__ void k_ws_correction(uint32_t n, const float4* __restrict__ p4, const float4* __restrict__ ppred,
                                const float4* __restrict__ x4, const float* __restrict__ local_len,
                                float4* __restrict__ dprev, float* __restrict__ target, float* __restrict__ mask) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 p = p4[i], q = ppred[i];
  const float4 d = make_float4(p.x - q.x, p.y - q.y, p.z - q.z, 0.f);
  dprev[i] = d;
  if (target) {
    const float invL = 1.0f / fmaxf(local_len[i], 1e-6f);
    target[size_t(i) * 3] = d.x * invL;
    target[size_t(i) * 3 + 1] = d.y * invL;
    target[size_t(i) * 3 + 2] = d.z * invL;
    mask[i] = x4[i].w > 0.f ? 1.f : 0.f;
  }
}

}  // namespace tcloth
