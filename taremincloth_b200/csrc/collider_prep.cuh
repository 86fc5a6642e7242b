// Mesh-collider upload on the device (simulation/mod.rs:2613-2670): the
// triangles arrive as host floats; packing, the Morton order of the
// centroids (stable), the per-triangle bounding spheres and the three
// conservative culling levels (groups of 16, 256 and 4,096 sorted triangles)
// are computed here, in the stream ahead of the frame, so that an upload
// costs the host one copy into pinned memory.  Every value equals the one
// the host computation it replaces gave, bit for bit: the float operations
// run in the same order without contraction (--fmad=false), the reductions
// are minima and maxima (exact in any order, NaN skipped the way the host's
// std::fmin / std::min skip it), and the radix sort is stable.
#pragma once
#include "solver_kernels.cuh"

namespace tcloth {

// one triangle from 9 floats (+ 4 attribute floats: friction, thickness,
// restitution, flags), as the host packed it
__global__ void k_col_pack(uint32_t T, const float* __restrict__ t9, const float* __restrict__ attr, float fric,
                           float thick, float rest, uint32_t flags0, MeshTri* __restrict__ out) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= T) return;
  const float* q = t9 + 9 * size_t(t);
  float f = fric, th = thick, r = rest;
  uint32_t flags = flags0;
  if (attr) {
    f = attr[4 * size_t(t)];
    th = attr[4 * size_t(t) + 1];
    r = attr[4 * size_t(t) + 2];
    const float fl = roundf(attr[4 * size_t(t) + 3]);
    flags = fl > 0.f ? (fl >= 4294967295.f ? 0xFFFFFFFFu : uint32_t(fl)) : 0u;
  }
  out[t] = MeshTri{make_float4(q[0], q[1], q[2], f), make_float4(q[3], q[4], q[5], th),
                   make_float4(q[6], q[7], q[8], r), make_float4(__uint_as_float(flags), 0.f, 0.f, 0.f)};
}

__device__ __forceinline__ float col_cen(const MeshTri& t, int a) {
  const float* p0 = &t.p0f.x;
  const float* p1 = &t.p1t.x;
  const float* p2 = &t.p2r.x;
  return (p0[a] + p1[a] + p2[a]) / 3.0f;
}

// box[0..2] = minimum centroid, box[3..5] = 1 / max(extent, 1e-5); one block
__global__ void __launch_bounds__(1024) k_col_bounds(uint32_t T, const MeshTri* __restrict__ raw,
                                                     float* __restrict__ box) {
  __shared__ float smin[3][1024], smax[3][1024];
  float lo[3] = {3.4028235e38f, 3.4028235e38f, 3.4028235e38f}, hi[3] = {-3.4028235e38f, -3.4028235e38f, -3.4028235e38f};
  for (uint32_t t = threadIdx.x; t < T; t += blockDim.x) {
    const MeshTri q = raw[t];
    for (int a = 0; a < 3; ++a) {
      const float c = col_cen(q, a);
      lo[a] = fminf(lo[a], c);
      hi[a] = fmaxf(hi[a], c);
    }
  }
  for (int a = 0; a < 3; ++a) {
    smin[a][threadIdx.x] = lo[a];
    smax[a][threadIdx.x] = hi[a];
  }
  __syncthreads();
  for (uint32_t h = blockDim.x / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h)
      for (int a = 0; a < 3; ++a) {
        smin[a][threadIdx.x] = fminf(smin[a][threadIdx.x], smin[a][threadIdx.x + h]);
        smax[a][threadIdx.x] = fmaxf(smax[a][threadIdx.x], smax[a][threadIdx.x + h]);
      }
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int a = 0; a < 3; ++a) {
      box[a] = smin[a][0];
      box[3 + a] = 1.f / fmaxf(smax[a][0] - smin[a][0], 1e-5f);
    }
}

__device__ __forceinline__ uint32_t col_expand10(uint32_t v) {
  v = (v * 0x00010001u) & 0xFF0000FFu;
  v = (v * 0x00000101u) & 0x0F00F00Fu;
  v = (v * 0x00000011u) & 0xC30C30C3u;
  v = (v * 0x00000005u) & 0x49249249u;
  return v;
}
__device__ __forceinline__ uint32_t col_quant(float f) {  // saturating float -> uint32
  if (!(f > 0.f)) return 0u;
  if (f >= 4294967295.f) return 0xFFFFFFFFu;
  return uint32_t(f);
}
__global__ void k_col_codes(uint32_t T, const MeshTri* __restrict__ raw, const float* __restrict__ box,
                            uint32_t* __restrict__ code, uint32_t* __restrict__ idx) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= T) return;
  const MeshTri q = raw[t];
  uint32_t c[3];
  for (int a = 0; a < 3; ++a)
    c[a] = col_quant(fminf(fmaxf((col_cen(q, a) - box[a]) * box[3 + a], 0.f), 1.f) * 1023.f);
  code[t] = (col_expand10(c[0]) << 2) | (col_expand10(c[1]) << 1) | col_expand10(c[2]);
  idx[t] = t;
}

// triangles in Morton order and their bounding spheres (centroid, widest
// vertex distance + thickness)
__global__ void k_col_gather(uint32_t T, const MeshTri* __restrict__ raw, const uint32_t* __restrict__ ord,
                             MeshTri* __restrict__ sorted, float4* __restrict__ bd) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= T) return;
  const MeshTri q = raw[ord[t]];
  sorted[t] = q;
  const float cx = col_cen(q, 0), cy = col_cen(q, 1), cz = col_cen(q, 2);
  auto d2 = [&](const float4& p) {
    const float ax = p.x - cx, ay = p.y - cy, az = p.z - cz;
    return ax * ax + ay * ay + az * az;
  };
  const float r = sqrtf(fmaxf(fmaxf(d2(q.p0f), d2(q.p1t)), d2(q.p2r))) + q.p1t.w;
  bd[t] = make_float4(cx, cy, cz, r);
}

// one block per group of `gs` consecutive spheres: a sphere around the box of
// the spheres widened 1.5x, in double, widened again by 1e-5 relative + 1e-7
__device__ __forceinline__ double col_dmin(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double col_dmax(double a, double b) { return (a < b) ? b : a; }
__global__ void __launch_bounds__(256) k_col_groups(uint32_t T, uint32_t gs, const float4* __restrict__ bd,
                                                    float4* __restrict__ out) {
  __shared__ double sl[3][256], sh[3][256];
  __shared__ double sC[3];
  const uint32_t b = blockIdx.x * gs, e = min(T, b + gs);
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (uint32_t t = b + threadIdx.x; t < e; t += blockDim.x) {
    const float4 s = bd[t];
    const double R = 1.5 * double(s.w);
    const double c[3] = {s.x, s.y, s.z};
    for (int a = 0; a < 3; ++a) {
      lo[a] = col_dmin(lo[a], c[a] - R);
      hi[a] = col_dmax(hi[a], c[a] + R);
    }
  }
  for (int a = 0; a < 3; ++a) {
    sl[a][threadIdx.x] = lo[a];
    sh[a][threadIdx.x] = hi[a];
  }
  __syncthreads();
  for (uint32_t h = blockDim.x / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h)
      for (int a = 0; a < 3; ++a) {
        sl[a][threadIdx.x] = col_dmin(sl[a][threadIdx.x], sl[a][threadIdx.x + h]);
        sh[a][threadIdx.x] = col_dmax(sh[a][threadIdx.x], sh[a][threadIdx.x + h]);
      }
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int a = 0; a < 3; ++a) sC[a] = (sl[a][0] + sh[a][0]) * 0.5;
  __syncthreads();
  const double C[3] = {sC[0], sC[1], sC[2]};
  double Rg = 0.0;
  for (uint32_t t = b + threadIdx.x; t < e; t += blockDim.x) {
    const float4 s = bd[t];
    const double dx = s.x - C[0], dy = s.y - C[1], dz = s.z - C[2];
    Rg = col_dmax(Rg, sqrt(dx * dx + dy * dy + dz * dz) + 1.5 * double(s.w));
  }
  __syncthreads();
  sl[0][threadIdx.x] = Rg;
  __syncthreads();
  for (uint32_t h = blockDim.x / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) sl[0][threadIdx.x] = col_dmax(sl[0][threadIdx.x], sl[0][threadIdx.x + h]);
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double rg = sl[0][0] * (1.0 + 1e-5) + 1e-7;
    out[blockIdx.x] = make_float4(float(C[0]), float(C[1]), float(C[2]), float(rg));
  }
}

}  // namespace tcloth
