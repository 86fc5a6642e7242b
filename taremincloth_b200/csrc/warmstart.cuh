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

#include "tcgen05.cuh"
#include "vmath.cuh"

namespace tcloth {

constexpr int kWsF = 16;   // input features
constexpr int kWsH = 64;   // hidden width
constexpr int kWsRows = 64;  // vertices per block tile (4 warps x 16 rows)
constexpr uint32_t kWsTcSpin = 1u << 22;  // polls (64 ns sleep each) of a tcgen05 MMA completion wait

// fp32 parameter blob: weights row-major [in][out], then the bias; then the
// normalizer, which training does not change (its gradient is zero): the
// per-feature input scales FS[16] and the output scale YS (features enter
// layer 0 as bf16(feature * FS); the network predicts correction / (L YS))
constexpr uint32_t kP_W0 = 0, kP_b0 = 1024, kP_W1 = 1088, kP_b1 = 9280, kP_W2 = 9344, kP_b2 = 17536,
                   kP_W3 = 17600, kP_b3 = 17792, kP_FS = 17795, kP_YS = 17811, kP_N = 17812;
// transposed bf16 copies [out][in] of W0..W2 for the forward GEMM's B operand
constexpr uint32_t kT_W0 = 0, kT_W1 = 1024, kT_W2 = 9216, kT_N = 17408;

// SiLU with the fast exponential and division intrinsics (the activation is
// rounded to bf16 next, which absorbs their few-ulp error); z below about
// -88 gives an infinite exponential and a zero quotient.
__device__ __forceinline__ float silu(float z) { return __fdividef(z, 1.0f + __expf(-z)); }
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
// The same fragments with ldmatrix (one instruction per 16x16 A tile, one
// per two 8-column B tiles): lane l supplies the address of row l % 8 of
// 8x8 matrix l / 8; rows must start on 16 bytes.
__device__ __forceinline__ void ldsm_x4(uint32_t r[4], const __nv_bfloat16* p) {
  const uint32_t a = static_cast<uint32_t>(__cvta_generic_to_shared(p));
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(a));
}
// A fragment of rows row0..row0+15, k0..k0+15 (matrices: rows 0-7 / 8-15 x k 0-7 / 8-15)
__device__ __forceinline__ void ldsm_a(uint32_t a[4], const __nv_bfloat16* A, int ld, int row0, int k0, int lane) {
  const int m = lane >> 3, r = lane & 7;
  ldsm_x4(a, A + (row0 + (m & 1) * 8 + r) * ld + k0 + (m >> 1) * 8);
}
// B fragments of columns n0..n0+7 (b[0..1]) and n0+8..n0+15 (b[2..3]) from Bt[n][k]
__device__ __forceinline__ void ldsm_b2(uint32_t b[4], const __nv_bfloat16* Bt, int ld, int n0, int k0, int lane) {
  const int m = lane >> 3, r = lane & 7;
  ldsm_x4(b, Bt + (n0 + (m >> 1) * 8 + r) * ld + k0 + (m & 1) * 8);
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
  const float* fscale;          // layer 0: per-feature scales [16], or null
  const __nv_bfloat16* h_prev;  // rounds: previous hidden [n][64]
  const uint32_t* adj_off;
  const uint32_t* adj_idx;
  const __nv_bfloat16* wt;      // [64][kin] (transposed weights)
  const float* bias;            // [64]
  __nv_bfloat16* x_out;         // optional: the assembled input [n][kin] (training)
  float* z_out;                 // optional: pre-activations [n][64] (training)
  __nv_bfloat16* h_out;         // [n][64]
};

__device__ __forceinline__ float out_scale(const float* ys) {
  const float v = ys ? *ys : 1.f;
  return v > 0.f ? v : 1.f;
}

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
      uint4 u = v < a.n ? __ldg(reinterpret_cast<const uint4*>(a.x_feat + size_t(v) * kWsF + c)) : make_uint4(0, 0, 0, 0);
      if (a.fscale) {
        float f[8];
        bf16x8_to_f32(u, f);
#pragma unroll
        for (int q = 0; q < 8; ++q) f[q] *= __ldg(a.fscale + c + q);
        u = f32_to_bf16x8(f);
      }
      *reinterpret_cast<uint4*>(&xs[r][c]) = u;
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
      xs[r][c] = __float2bfloat16(silu(z));
    }
  __syncwarp();
  if (a.h_out) {
    for (int e = lane; e < 16 * 8; e += 32) {
      const int r = warp * 16 + (e >> 3), c = (e & 7) * 8;
      if (row0 + r < a.n)
        *reinterpret_cast<uint4*>(a.h_out + size_t(row0 + r) * kWsH + c) = *reinterpret_cast<const uint4*>(&xs[r][c]);
    }
  }
}

// Head: Y = H2 W3 + b3 (fp32 accumulation of bf16 products).  With targets,
// also dY = 2 (Y - T / YS) m / (3 n) (mean squared error against the
// normalised target, mask m of free vertices) and the loss.
__global__ void k_mlp_head(uint32_t n, const __nv_bfloat16* __restrict__ h2, const __nv_bfloat16* __restrict__ w3,
                           const float* __restrict__ b3, float* __restrict__ y, const float* __restrict__ target,
                           const float* __restrict__ mask, const float* __restrict__ yscale, float inv_count,
                           float* __restrict__ dy, float* __restrict__ loss) {
  const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  float l = 0.f;
  const float ys = out_scale(yscale);
  if (v < n) {
    for (int c = 0; c < 3; ++c) {
      float s = 0.f;
      for (int k = 0; k < kWsH; ++k) s += __bfloat162float(h2[size_t(v) * kWsH + k]) * __bfloat162float(w3[k * 3 + c]);
      s += b3[c];
      y[size_t(v) * 3 + c] = s;
      if (target) {
        const float m = mask ? mask[v] : 1.0f;
        const float d = (s - target[size_t(v) * 3 + c] / ys) * m;
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

// Backward of a 128-wide layer on the tcgen05 tensor cores.  Persistent CTAs
// of 256 threads take tiles of 128 rows; per tile they stage, as K-major core
// matrices: X^T (M = 128 inputs x K = 128 rows) and dZ^T (N = 64 x K = 128
// rows) for dW, and dZ (M = 128 rows x K = 64) for dX; W (N = 128 x K = 64)
// is staged once.  Thread 0 issues 4 MMAs of dX = dZ W^T into TMEM columns
// 64-191 (fresh per tile) and 8 MMAs of dW += X^T dZ into columns 0-63,
// which accumulate over all of the CTA's tiles; one commit per tile.  dX
// rows go out from the per-tile epilogue, and each CTA adds its dW to the
// global sum once at the end.  A completion wait that runs out of polls sets
// *err = 2.  Grid: the resident CTAs (2 per SM: 80 KB of shared memory,
// 256 TMEM columns each).
struct MlpBwdTcArgs {
  uint32_t n;
  const __nv_bfloat16* x;   // [n][128]
  const __nv_bfloat16* dz;  // [n][64]
  const __nv_bfloat16* w;   // [128][64] row-major weights
  float* dw;                // [128][64], added to
  float* dx;                // [n][128] or null
  int* err;
};
constexpr uint32_t kWsBwdCols = 256;
constexpr uint32_t kWsBwdSmem = 128 * 128 * 2 + 64 * 128 * 2 + 128 * 64 * 2 + 128 * 64 * 2;
__global__ void __launch_bounds__(256, 2) k_mlp_layer_bwd_tc(MlpBwdTcArgs a) {
  extern __shared__ __align__(128) uint8_t bw_dsm[];
  uint8_t* adw = bw_dsm;                    // X^T  [128 inputs][K 128 rows]
  uint8_t* bdw = adw + 128 * 128 * 2;       // dZ^T [64 outputs][K 128 rows]
  uint8_t* adx = bdw + 64 * 128 * 2;        // dZ   [128 rows][K 64]
  uint8_t* bdx = adx + 128 * 64 * 2;        // W    [128 inputs][K 64]
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tslot;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (int e = tid; e < 128 * 8; e += blockDim.x)  // W row c, 8 outputs per uint4
    *reinterpret_cast<uint4*>(bdx + cm_offset(e >> 3, (e & 7) * 8, 64)) = __ldg(reinterpret_cast<const uint4*>(a.w) + e);
  if (warp == 0) tmem_alloc(&tslot, kWsBwdCols);
  if (tid == 0) mbar_init(&mbar, 1);
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = tslot;
  const uint32_t a_dw = smem_addr(adw), b_dw = smem_addr(bdw), a_dx = smem_addr(adx), b_dx = smem_addr(bdx);
  constexpr uint32_t id_dw = idesc_bf16_f32(128, 64), id_dx = idesc_bf16_f32(128, 128);
  const uint32_t ntiles = (a.n + 127) / 128;
  const int quad = warp & 3, half = warp >> 2;
  uint32_t parity = 0;
  bool ok = true, any = false;
  auto pair = [](uint16_t lo, uint16_t hi) { return uint32_t(lo) | (uint32_t(hi) << 16); };
  for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const uint32_t row0 = tile * 128;
    // X^T: rows 2p, 2p + 1 and inputs c0 .. c0 + 7 per item (1024 items)
    for (int e = tid; e < 64 * 16; e += blockDim.x) {
      const int rp = e & 63, c0 = (e >> 6) * 8, r = 2 * rp;
      const uint32_t v0 = row0 + r, v1 = v0 + 1;
      const uint4 u0 = v0 < a.n ? __ldg(reinterpret_cast<const uint4*>(a.x + size_t(v0) * 128 + c0)) : make_uint4(0, 0, 0, 0);
      const uint4 u1 = v1 < a.n ? __ldg(reinterpret_cast<const uint4*>(a.x + size_t(v1) * 128 + c0)) : make_uint4(0, 0, 0, 0);
      const uint16_t* h0 = reinterpret_cast<const uint16_t*>(&u0);
      const uint16_t* h1 = reinterpret_cast<const uint16_t*>(&u1);
#pragma unroll
      for (int i = 0; i < 8; ++i) *reinterpret_cast<uint32_t*>(adw + cm_offset(c0 + i, r, 128)) = pair(h0[i], h1[i]);
    }
    // dZ^T (rows 2p, 2p + 1, outputs n0 .. n0 + 7) and dZ itself
    for (int e = tid; e < 64 * 8; e += blockDim.x) {
      const int rp = e & 63, n0 = (e >> 6) * 8, r = 2 * rp;
      const uint32_t v0 = row0 + r, v1 = v0 + 1;
      const uint4 u0 = v0 < a.n ? __ldg(reinterpret_cast<const uint4*>(a.dz + size_t(v0) * kWsH + n0)) : make_uint4(0, 0, 0, 0);
      const uint4 u1 = v1 < a.n ? __ldg(reinterpret_cast<const uint4*>(a.dz + size_t(v1) * kWsH + n0)) : make_uint4(0, 0, 0, 0);
      const uint16_t* h0 = reinterpret_cast<const uint16_t*>(&u0);
      const uint16_t* h1 = reinterpret_cast<const uint16_t*>(&u1);
#pragma unroll
      for (int i = 0; i < 8; ++i) *reinterpret_cast<uint32_t*>(bdw + cm_offset(n0 + i, r, 128)) = pair(h0[i], h1[i]);
      *reinterpret_cast<uint4*>(adx + cm_offset(r, n0, 64)) = u0;
      *reinterpret_cast<uint4*>(adx + cm_offset(r + 1, n0, 64)) = u1;
    }
    fence_async_smem();
    tc_fence_before();  // the previous tile's TMEM reads come before this tile's MMAs
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
#pragma unroll
      for (uint32_t s = 0; s < 4; ++s)
        mma_bf16(tbase + 64, smem_desc(a_dx + 256 * s, 128, 1024), smem_desc(b_dx + 256 * s, 128, 1024), id_dx, s > 0);
#pragma unroll
      for (uint32_t s = 0; s < 8; ++s)
        mma_bf16(tbase, smem_desc(a_dw + 256 * s, 128, 2048), smem_desc(b_dw + 256 * s, 128, 2048), id_dw,
                 any || s > 0);
      mma_commit(&mbar);
    }
    any = true;
    ok = __syncthreads_and(mbar_wait(&mbar, parity, kWsTcSpin));
    if (!ok) break;
    parity ^= 1u;
    tc_fence_after();
    if (a.dx) {
      const uint32_t r = quad * 32 + lane, v = row0 + r;
#pragma unroll
      for (int c0 = 0; c0 < 64; c0 += 32) {
        float z[32];
        const uint32_t taddr = tbase + (uint32_t(quad * 32) << 16) + 64u + uint32_t(half * 64 + c0);
        tmem_ld16(taddr, z);
        tmem_ld16(taddr + 16, z + 16);
        if (v < a.n) {
          float4* o = reinterpret_cast<float4*>(a.dx + size_t(v) * 128 + half * 64 + c0);
#pragma unroll
          for (int q = 0; q < 8; ++q) o[q] = make_float4(z[4 * q], z[4 * q + 1], z[4 * q + 2], z[4 * q + 3]);
        }
      }
    }
  }
  if (ok && any) {
    // dW rows (TMEM lanes) c = 32 quad + lane, outputs 32 half .. 32 half + 31
    const uint32_t c = quad * 32 + lane;
    float z[32];
    const uint32_t taddr = tbase + (uint32_t(quad * 32) << 16) + uint32_t(half * 32);
    tmem_ld16(taddr, z);
    tmem_ld16(taddr + 16, z + 16);
#pragma unroll
    for (int k = 0; k < 32; ++k) atomicAdd(&a.dw[c * kWsH + half * 32 + k], z[k]);
  }
  if (!ok) {
    if (tid == 0 && a.err) atomicExch(a.err, 2);
    mbar_wait(&mbar, parity, kWsTcSpin);  // the MMAs still in flight, if any
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tbase, kWsBwdCols);
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

// Normalizer statistics of recorded snapshots: per block, over the rows
// blockIdx.x, blockIdx.x + gridDim.x, ... of the free vertices (mask), the
// sums of squares of the 16 features and of the target, and the row count;
// a fixed grid and fixed reduction order make the result reproducible.
constexpr int kWsMomBlocks = 296, kWsMom = kWsF + 2;
__global__ void __launch_bounds__(256) k_ws_moments(size_t rows, const __nv_bfloat16* __restrict__ feat,
                                                    const float* __restrict__ target, const float* __restrict__ mask,
                                                    float* __restrict__ part) {
  float acc[kWsMom];
#pragma unroll
  for (int c = 0; c < kWsMom; ++c) acc[c] = 0.f;
  for (size_t r = size_t(blockIdx.x) * blockDim.x + threadIdx.x; r < rows; r += size_t(gridDim.x) * blockDim.x) {
    if (mask[r] <= 0.f) continue;
    float f[8];
    for (int h = 0; h < 2; ++h) {
      bf16x8_to_f32(__ldg(reinterpret_cast<const uint4*>(feat + r * kWsF) + h), f);
#pragma unroll
      for (int q = 0; q < 8; ++q) acc[h * 8 + q] += f[q] * f[q];
    }
    for (int q = 0; q < 3; ++q) acc[kWsF] += target[r * 3 + q] * target[r * 3 + q];
    acc[kWsF + 1] += 1.f;
  }
  __shared__ float red[8][kWsMom];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int c = 0; c < kWsMom; ++c) {
    float t = acc[c];
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    if (lane == 0) red[warp][c] = t;
  }
  __syncthreads();
  if (threadIdx.x < kWsMom) {
    float t = 0.f;
    for (int w = 0; w < int(blockDim.x >> 5); ++w) t += red[w][threadIdx.x];
    part[size_t(blockIdx.x) * kWsMom + threadIdx.x] = t;
  }
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
__device__ __forceinline__ void ws_feature_row(const WsFeatArgs& a, uint32_t i, float f[kWsF]) {
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
  const float g[kWsF] = {dp.x * invL, dp.y * invL, dp.z * invL, jac.x * invL, jac.y * invL, jac.z * invL, sdf,
                         n.x, n.y, n.z, vi4.x * a.dt * invL, vi4.y * a.dt * invL, vi4.z * a.dt * invL,
                         a.g_dt2 * invL, wi > 0.f ? 1.f : 0.f, 1.f};
#pragma unroll
  for (int c = 0; c < kWsF; ++c) f[c] = g[c];
}
// features of every vertex (bf16) for the recorded training snapshots
__global__ void k_ws_features(WsFeatArgs a) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  float f[kWsF];
  ws_feature_row(a, i, f);
  for (int c = 0; c < kWsF; ++c) a.feat[size_t(i) * kWsF + c] = __float2bfloat16(f[c]);
}

// ---------------------------------------------------------------------------
// Inference kernels.  Same products and rounding points as the training
// forward (k_mlp_layer_fwd; the fused head sums in another order), organised
// for throughput on large graphs: layer 0 computes the features in the
// kernel (and keeps the predicted positions); the message-passing layers run
// persistent over 64-row tiles with W^T staged in shared memory once per
// block, all 8 warps on the tensor cores (two per 16 rows, 32 output columns
// each); each row's neighbour list comes from an ELL table (degree, then the
// first 15 neighbours in adjacency order; the CSR serves the rest), so the
// neighbour rows of a vertex are all in flight at once.
constexpr int kWsEll = 16;
constexpr int kWsL0Rows = 256;  // layer 0: one vertex per thread

struct MlpInferArgs {
  uint32_t n;
  // layer 0
  const __nv_bfloat16* x_feat;  // given features [n][16], or null: computed from fa
  WsFeatArgs fa;
  float4* ppred;                // with computed features: copy of p before the move
  const float* fscale;
  // message-passing layers
  const __nv_bfloat16* h_prev;
  const uint32_t* ell;          // [n][16]
  const uint32_t* adj_off;
  const uint32_t* adj_idx;
  const __nv_bfloat16* wt;      // W^T [64][kin]
  const float* bias;
  __nv_bfloat16* h_out;         // or null with the fused head
  const __nv_bfloat16* w3;
  const float* b3;
  const float* yscale;
  float* y_out;
  const float4* x4;
  float4* p4;
  const float* local_len;
  int* err;  // tcgen05 kernels: set to 2 when an MMA completion wait ran out (may be null)
  // training forward (k_mlp_infer_mp_tc without the head): the gathered X
  // rows [n][128] and Z = X W + b [n][64] (both may be null)
  __nv_bfloat16* x_out;
  float* z_out;
};

// Layer 0: X0 = bf16(bf16(features) * FS), H0 = bf16(SiLU(X0 W0 + b0)).
__global__ void __launch_bounds__(kWsL0Rows) k_mlp_infer_l0(MlpInferArgs a) {
  __shared__ __align__(16) union {
    __nv_bfloat16 x[kWsL0Rows][kWsF + 8];
    __nv_bfloat16 h[kWsL0Rows][kWsH + 8];
  } sm;
  __shared__ __align__(16) __nv_bfloat16 wt[kWsH][kWsF + 8];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t row0 = blockIdx.x * kWsL0Rows, v = row0 + tid;
  for (int e = tid; e < kWsH * 2; e += blockDim.x)
    *reinterpret_cast<uint4*>(&wt[e >> 1][(e & 1) * 8]) = __ldg(reinterpret_cast<const uint4*>(a.wt) + e);
  float f[kWsF];
  if (v < a.n) {
    if (a.x_feat) {
      bf16x8_to_f32(__ldg(reinterpret_cast<const uint4*>(a.x_feat + size_t(v) * kWsF)), f);
      bf16x8_to_f32(__ldg(reinterpret_cast<const uint4*>(a.x_feat + size_t(v) * kWsF) + 1), f + 8);
    } else {
      ws_feature_row(a.fa, v, f);
#pragma unroll
      for (int c = 0; c < kWsF; ++c) f[c] = __bfloat162float(__float2bfloat16(f[c]));
      a.ppred[v] = a.fa.p4[v];
    }
#pragma unroll
    for (int c = 0; c < kWsF; ++c) f[c] *= __ldg(a.fscale + c);
  } else {
#pragma unroll
    for (int c = 0; c < kWsF; ++c) f[c] = 0.f;
  }
  *reinterpret_cast<uint4*>(&sm.x[tid][0]) = f32_to_bf16x8(f);
  *reinterpret_cast<uint4*>(&sm.x[tid][8]) = f32_to_bf16x8(f + 8);
  __syncthreads();
  // each warp: rows warp*32 .. +31, two 16-row tiles, one k step
  uint32_t af[2][4];
  load_a_frag(af[0], &sm.x[0][0], kWsF + 8, warp * 32, 0, lane);
  load_a_frag(af[1], &sm.x[0][0], kWsF + 8, warp * 32 + 16, 0, lane);
  __syncthreads();  // sm.x is overwritten by the outputs below
  const int g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      float acc[4] = {0.f, 0.f, 0.f, 0.f};
      uint32_t bf[2];
      load_b_frag(bf, &wt[0][0], kWsF + 8, nt * 8, 0, lane);
      mma_bf16_16816(acc, af[mt], bf);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int r = warp * 32 + mt * 16 + g + (q >> 1) * 8, c = nt * 8 + 2 * t + (q & 1);
        sm.h[r][c] = __float2bfloat16(silu(acc[q] + __ldg(a.bias + c)));
      }
    }
  __syncthreads();
  for (int e = tid; e < kWsL0Rows * 8; e += blockDim.x) {
    const int r = e >> 3, c = (e & 7) * 8;
    if (row0 + r < a.n)
      *reinterpret_cast<uint4*>(a.h_out + size_t(row0 + r) * kWsH + c) = *reinterpret_cast<const uint4*>(&sm.h[r][c]);
  }
}

// Neighbour mean of one (vertex, 8-column group): bf16(mean_{j in N(i)} H_j)
// summed in adjacency order (as the training forward), up to eight
// neighbour rows in flight.
__device__ __forceinline__ uint4 ws_neighbour_mean(const MlpInferArgs& a, uint32_t v, int cg) {
  auto row = [&](uint32_t j) { return __ldg(reinterpret_cast<const uint4*>(a.h_prev + size_t(j) * kWsH + cg)); };
  const uint4* er = reinterpret_cast<const uint4*>(a.ell + size_t(v) * kWsEll);
  const uint4 e0 = __ldg(er), e1 = __ldg(er + 1), e2 = __ldg(er + 2), e3 = __ldg(er + 3);
  const uint32_t idx[15] = {e0.y, e0.z, e0.w, e1.x, e1.y, e1.z, e1.w, e2.x, e2.y, e2.z, e2.w, e3.x, e3.y, e3.z, e3.w};
  const uint32_t deg = e0.x, d1 = min(deg, 15u);
  float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  auto add = [&](const uint4 u) {
    float fv[8];
    bf16x8_to_f32(u, fv);
#pragma unroll
    for (int c = 0; c < 8; ++c) acc[c] += fv[c];
  };
#pragma unroll
  for (int q0 = 0; q0 < 15; q0 += 8) {
    if (uint32_t(q0) >= d1) break;
    uint4 u[8];
#pragma unroll
    for (int k = 0; k < 8; ++k)
      if (q0 + k < 15 && uint32_t(q0 + k) < d1) u[k] = row(idx[q0 + k]);
#pragma unroll
    for (int k = 0; k < 8; ++k)
      if (q0 + k < 15 && uint32_t(q0 + k) < d1) add(u[k]);
  }
  if (deg > 15u) {
    const uint32_t b = __ldg(a.adj_off + v), en = __ldg(a.adj_off + v + 1);
    for (uint32_t q = b + 15u; q < en; ++q) add(row(__ldg(a.adj_idx + q)));
  }
  const float inv = deg ? 1.0f / float(deg) : 0.0f;
#pragma unroll
  for (int c = 0; c < 8; ++c) acc[c] *= inv;
  return f32_to_bf16x8(acc);
}
// Message-passing layer: X = [H_i, bf16(mean_j H_j)], H' = bf16(SiLU(X W + b)),
// or with w3 the head Y = H' W3 + b3 and p += Y YS L on free vertices.
__global__ void __launch_bounds__(256, 3) k_mlp_infer_mp(MlpInferArgs a) {
  __shared__ __align__(16) __nv_bfloat16 xs[kWsRows][128 + 8];
  __shared__ __align__(16) __nv_bfloat16 ws[kWsH][128 + 8];
  __shared__ float ypart[2][kWsRows][3];  // fused head: partial sums of the two column halves
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int e = tid; e < kWsH * 16; e += blockDim.x)
    *reinterpret_cast<uint4*>(&ws[e >> 4][(e & 15) * 8]) = __ldg(reinterpret_cast<const uint4*>(a.wt) + e);
  const uint32_t ntiles = (a.n + kWsRows - 1) / kWsRows;
  auto row = [&](uint32_t j, int cg) { return __ldg(reinterpret_cast<const uint4*>(a.h_prev + size_t(j) * kWsH + cg)); };
  const int g = lane >> 2, t = lane & 3;
  const int wr = (warp & 3) * 16, wn = (warp >> 2) * 4;  // warp: rows wr..wr+15, columns (wn..wn+3) x 8
  for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const uint32_t row0 = tile * kWsRows;
#pragma unroll 1
    for (int m = 0; m < 2; ++m) {
      const int r = (tid >> 3) + 32 * m, cg = (tid & 7) * 8;
      const uint32_t v = row0 + r;
      uint4 self = make_uint4(0, 0, 0, 0), mean = make_uint4(0, 0, 0, 0);
      if (v < a.n) {
        self = row(v, cg);
        mean = ws_neighbour_mean(a, v, cg);
      }
      *reinterpret_cast<uint4*>(&xs[r][cg]) = self;
      *reinterpret_cast<uint4*>(&xs[r][kWsH + cg]) = mean;
    }
    __syncthreads();
    float acc[4][4];
#pragma unroll
    for (int nt = 0; nt < 4; ++nt)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[nt][q] = 0.f;
#pragma unroll
    for (int k0 = 0; k0 < 128; k0 += 16) {
      uint32_t af[4], bf[2][4];
      ldsm_a(af, &xs[0][0], 128 + 8, wr, k0, lane);
      ldsm_b2(bf[0], &ws[0][0], 128 + 8, wn * 8, k0, lane);
      ldsm_b2(bf[1], &ws[0][0], 128 + 8, wn * 8 + 16, k0, lane);
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) mma_bf16_16816(acc[nt], af, &bf[nt >> 1][(nt & 1) * 2]);
    }
    __syncthreads();  // every warp has read its input rows before any output is written over them
    float y0[3] = {0.f, 0.f, 0.f}, y1[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int nt = 0; nt < 4; ++nt)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int r = wr + g + (q >> 1) * 8, c = (wn + nt) * 8 + 2 * t + (q & 1);
        const __nv_bfloat16 h = __float2bfloat16(silu(acc[nt][q] + __ldg(a.bias + c)));
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
    if (a.w3) {
      for (int j = 0; j < 3; ++j) {
        y0[j] += __shfl_xor_sync(0xffffffffu, y0[j], 1);
        y0[j] += __shfl_xor_sync(0xffffffffu, y0[j], 2);
        y1[j] += __shfl_xor_sync(0xffffffffu, y1[j], 1);
        y1[j] += __shfl_xor_sync(0xffffffffu, y1[j], 2);
      }
      if (t < 2)
        for (int j = 0; j < 3; ++j) ypart[warp >> 2][wr + g + t * 8][j] = t ? y1[j] : y0[j];
      __syncthreads();
      if (tid < kWsRows) {
        const uint32_t v = row0 + tid;
        if (v < a.n) {
          const float Y[3] = {ypart[0][tid][0] + ypart[1][tid][0] + a.b3[0],
                              ypart[0][tid][1] + ypart[1][tid][1] + a.b3[1],
                              ypart[0][tid][2] + ypart[1][tid][2] + a.b3[2]};
          if (a.y_out)
            for (int j = 0; j < 3; ++j) a.y_out[size_t(v) * 3 + j] = Y[j];
          if (a.p4 && a.x4[v].w > 0.f) {
            const float L = fmaxf(a.local_len[v], 1e-6f), ys = out_scale(a.yscale);
            float4 p = a.p4[v];
            p.x += Y[0] * ys * L;
            p.y += Y[1] * ys * L;
            p.z += Y[2] * ys * L;
            a.p4[v] = p;
          }
        }
      }
    } else {
      __syncthreads();
      for (int e = tid; e < kWsRows * 8; e += blockDim.x) {
        const int r = e >> 3, c = (e & 7) * 8;
        if (row0 + r < a.n)
          *reinterpret_cast<uint4*>(a.h_out + size_t(row0 + r) * kWsH + c) = *reinterpret_cast<const uint4*>(&xs[r][c]);
      }
    }
    __syncthreads();  // xs is rewritten by the next tile's gather
  }
}

// The same message-passing layer on the tcgen05 tensor cores.  A CTA of 256
// threads takes tiles of 128 vertices: the threads gather
// X = [H_i, bf16(mean_j H_j)] (128 x 128 bf16, four (row, 8-column) pieces
// per thread) into shared memory as core matrices (layout below),
// thread 0 issues eight MMAs of K = 16 into a 128 x 64 fp32 accumulator in
// tensor memory (TMEM lane = tile row) and commits them to an mbarrier, and
// the epilogue reads the accumulator back with tcgen05.ld: warps w and w + 4
// share lane quadrant w, taking columns 0-31 and 32-63 (bias, SiLU, bf16;
// or the fused head, whose two column halves meet in shared memory).  W^T
// stays in shared memory for the CTA's lifetime.  A completion wait that
// runs out of polls sets *err = 2 and ends the kernel after one more bounded
// wait, freeing its TMEM.
constexpr int kWsTcRows = 128;
constexpr int kWsTcThreads = 256;
constexpr int kWsTcMinBlocks = 3;  // CTAs per SM (launch bounds: 80 registers)
constexpr uint32_t kWsTcCols = 64;         // TMEM columns: the fp32 accumulator
// X tile layout: K chunk c of all 16 row groups is one run of 16 core
// matrices (2,048 bytes), and the runs are kWsTcLbo = 2,064 bytes apart
// (the descriptor's leading byte offset; stride byte offset 128).  The 16
// extra bytes put the 8 chunks of one row, which a quarter-warp stores at
// once, in 8 different bank groups.
constexpr uint32_t kWsTcLbo = 16 * 128 + 16;
constexpr uint32_t kWsTcXBytes = 16 * kWsTcLbo;
constexpr uint32_t kWsTcSmemMp = kWsTcXBytes + kWsH * 128 * 2;  // X tile + W^T
__device__ __forceinline__ uint32_t xs_offset(uint32_t row, uint32_t k) {
  return (k >> 3) * kWsTcLbo + (row >> 3) * 128u + (row & 7u) * 16u + (k & 7u) * 2u;
}
__global__ void __launch_bounds__(kWsTcThreads, kWsTcMinBlocks) k_mlp_infer_mp_tc(MlpInferArgs a) {
  extern __shared__ __align__(128) uint8_t ws_dsm[];
  uint8_t* xs = ws_dsm;                 // X tile [128 rows][K 128] (xs_offset)
  uint8_t* wsm = ws_dsm + kWsTcXBytes;  // W^T [64 outputs][K 128] (cm_offset)
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tslot;
  __shared__ float ypart[kWsTcRows][3];  // fused head: columns 32-63 of each row
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (int e = tid; e < kWsH * 16; e += blockDim.x)
    *reinterpret_cast<uint4*>(wsm + cm_offset(e >> 4, (e & 15) * 8, 128)) =
        __ldg(reinterpret_cast<const uint4*>(a.wt) + e);
  if (warp == 0) tmem_alloc(&tslot, kWsTcCols);
  if (tid == 0) mbar_init(&mbar, 1);
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = tslot, xa = smem_addr(xs), wa = smem_addr(wsm);
  constexpr uint32_t idesc = idesc_bf16_f32(kWsTcRows, kWsH);
  auto row = [&](uint32_t j, int cg) { return __ldg(reinterpret_cast<const uint4*>(a.h_prev + size_t(j) * kWsH + cg)); };
  const uint32_t ntiles = (a.n + kWsTcRows - 1) / kWsTcRows;
  const int quad = warp & 3, half = warp >> 2, er = quad * 32 + lane;  // epilogue: row er, columns 32 half ..
  uint32_t parity = 0;
  bool ok = true;
  for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const uint32_t row0 = tile * kWsTcRows;
#pragma unroll 1
    for (int m = 0; m < 4; ++m) {
      const int r = (tid >> 3) + 32 * m, cg = (tid & 7) * 8;
      const uint32_t v = row0 + r;
      uint4 self = make_uint4(0, 0, 0, 0), mean = make_uint4(0, 0, 0, 0);
      if (v < a.n) {
        self = row(v, cg);
        mean = ws_neighbour_mean(a, v, cg);
      }
      *reinterpret_cast<uint4*>(xs + xs_offset(r, cg)) = self;
      *reinterpret_cast<uint4*>(xs + xs_offset(r, kWsH + cg)) = mean;
      if (a.x_out && v < a.n) {
        *reinterpret_cast<uint4*>(a.x_out + size_t(v) * 128 + cg) = self;
        *reinterpret_cast<uint4*>(a.x_out + size_t(v) * 128 + kWsH + cg) = mean;
      }
    }
    fence_async_smem();
    tc_fence_before();  // the previous tile's TMEM reads come before this tile's MMAs
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
#pragma unroll
      for (uint32_t s = 0; s < 8; ++s)
        mma_bf16(tbase, smem_desc(xa + 2 * s * kWsTcLbo, kWsTcLbo, 128), smem_desc(wa + 256 * s, 128, 2048), idesc,
                 s > 0);
      mma_commit(&mbar);
    }
    ok = __syncthreads_and(mbar_wait(&mbar, parity, kWsTcSpin));
    if (!ok) break;
    parity ^= 1u;
    tc_fence_after();
    float z[32];
    const uint32_t taddr = tbase + (uint32_t(quad * 32) << 16) + uint32_t(half * 32);
    tmem_ld16(taddr, z);
    tmem_ld16(taddr + 16, z + 16);
    const uint32_t v = row0 + er;
    const int c0 = half * 32;
    if (a.w3) {
      float y[3] = {0.f, 0.f, 0.f};
#pragma unroll
      for (int c = 0; c < 32; ++c) {
        const float h = __bfloat162float(__float2bfloat16(silu(z[c] + __ldg(a.bias + c0 + c))));
#pragma unroll
        for (int j = 0; j < 3; ++j) y[j] += h * __bfloat162float(a.w3[(c0 + c) * 3 + j]);
      }
      if (half)
        for (int j = 0; j < 3; ++j) ypart[er][j] = y[j];
      __syncthreads();
      if (!half && v < a.n) {
        const float Y[3] = {(y[0] + ypart[er][0]) + a.b3[0], (y[1] + ypart[er][1]) + a.b3[1],
                            (y[2] + ypart[er][2]) + a.b3[2]};
        if (a.y_out)
          for (int j = 0; j < 3; ++j) a.y_out[size_t(v) * 3 + j] = Y[j];
        if (a.p4 && a.x4[v].w > 0.f) {
          const float L = fmaxf(a.local_len[v], 1e-6f), ys = out_scale(a.yscale);
          float4 p = a.p4[v];
          p.x += Y[0] * ys * L;
          p.y += Y[1] * ys * L;
          p.z += Y[2] * ys * L;
          a.p4[v] = p;
        }
      }
    } else if (v < a.n) {
#pragma unroll
      for (int cg = 0; cg < 32; cg += 8) {
        float zb[8], hv[8];
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          zb[c] = z[cg + c] + __ldg(a.bias + c0 + cg + c);
          hv[c] = silu(zb[c]);
        }
        if (a.z_out) {
          float4* zo = reinterpret_cast<float4*>(a.z_out + size_t(v) * kWsH + c0 + cg);
          zo[0] = make_float4(zb[0], zb[1], zb[2], zb[3]);
          zo[1] = make_float4(zb[4], zb[5], zb[6], zb[7]);
        }
        *reinterpret_cast<uint4*>(a.h_out + size_t(v) * kWsH + c0 + cg) = f32_to_bf16x8(hv);
      }
    }
  }
  if (!ok) {
    if (tid == 0 && a.err) atomicExch(a.err, 2);
    mbar_wait(&mbar, parity, kWsTcSpin);  // the MMAs still in flight, if any
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tbase, kWsTcCols);
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
