// rm_atrous.cu - the a-trous edge-aware filter (pathtrace.metal:1315-1354) as a
// shared-memory tiled kernel, fused with the tonemap (:1355-1363) on its last
// pass.
//
// This file is compiled WITH fused multiply-add: the filter's weights go
// through exp2 and rsqrt approximations anyway, so its parity with the CPU
// oracle is a tolerance (1e-4 relative on 99.9 % of pixels), and contraction
// only shortens the dependency chains.  Per tap the kernel reads four shared
// memory records (position|kind, normal|luma, colour|albedo.r, albedo.gb);
// the 5 x 5 footprint's HBM bytes are read once per tile.  Taps outside the
// image or on pixels of kind 0 hold a zero normal in the tile, so their weight
// pow16(max(n.n0, 0)) x exp2(<= 0) is exactly 0 and the reference's explicit
// skips (bounds, kind) need no test per tap.
#include <cuda_runtime.h>

#include "rm_device.cuh"
#include "rm_launch.h"

namespace rmd {

namespace {

constexpr int kTX = 32, kTY = 8;

__device__ __forceinline__ float luma(float r, float g, float b) { return 0.2126f * r + 0.7152f * g + 0.0722f * b; }

__device__ __forceinline__ float3 ld3(const float* __restrict__ a, uint32_t i) {
  return make_float3(a[size_t(i) * 3], a[size_t(i) * 3 + 1], a[size_t(i) * 3 + 2]);
}
__device__ __forceinline__ void st3(float* __restrict__ a, uint32_t i, float x, float y, float z) {
  a[size_t(i) * 3] = x; a[size_t(i) * 3 + 1] = y; a[size_t(i) * 3 + 2] = z;
}

// |d| from d.d: d2 / sqrt(d2), 0 for d2 = 0 (the clamp keeps rsqrt finite)
__device__ __forceinline__ float fast_len(float d2) { return d2 * rsqrtf(fmaxf(d2, 1e-30f)); }

template <int STEP>
__global__ void __launch_bounds__(kTX* kTY) k_denoise_atrous_tiled(Params p, GBufSoA gb, const float* __restrict__ in,
                                                                   float* __restrict__ out, uint8_t* __restrict__ rgb) {
  constexpr int R = 2 << STEP;  // halo: 2 taps x stride
  constexpr int SW = kTX + 2 * R, SH = kTY + 2 * R;
  __shared__ float4 s_pk[SH][SW];  // pos, kind
  __shared__ float4 s_nl[SH][SW];  // normal, luma
  __shared__ float4 s_ca[SH][SW];  // colour rgb, albedo r
  __shared__ float2 s_ag[SH][SW];  // albedo g, b
  const int W = p.width, H = p.height;
  const int x0 = blockIdx.x * kTX, y0 = blockIdx.y * kTY;
  const int tid = threadIdx.y * kTX + threadIdx.x;
  for (int k = tid; k < SW * SH; k += kTX * kTY) {
    const int lx = k % SW, ly = k / SW;
    const int gx = x0 + lx - R, gy = y0 + ly - R;
    float4 pk = make_float4(0.f, 0.f, 0.f, __int_as_float(0));
    float4 nl = make_float4(0.f, 0.f, 0.f, 0.f), ca = nl;
    float2 ag = make_float2(0.f, 0.f);
    if (gx >= 0 && gy >= 0 && gx < W && gy < H) {
      const uint32_t n = uint32_t(gy) * uint32_t(W) + uint32_t(gx);
      pk = gb.pos_kind[n];
      if (__float_as_int(pk.w) != 0) {
        const float4 N = gb.nor_rough[n], A = gb.alb_met[n];
        const float3 c = ld3(in, n);
        nl = make_float4(N.x, N.y, N.z, luma(c.x, c.y, c.z));
        ca = make_float4(c.x, c.y, c.z, A.x);
        ag = make_float2(A.y, A.z);
      }
    }
    s_pk[ly][lx] = pk; s_nl[ly][lx] = nl; s_ca[ly][lx] = ca; s_ag[ly][lx] = ag;
  }
  __syncthreads();
  const int x = x0 + threadIdx.x, y = y0 + threadIdx.y;
  if (x >= W || y >= H) return;
  const uint32_t id = uint32_t(y) * uint32_t(W) + uint32_t(x);
  const int cx = threadIdx.x + R, cy = threadIdx.y + R;
  const float4 P0 = s_pk[cy][cx];
  float rx = 0, ry = 0, rz = 0;
  if (__float_as_int(P0.w) != 0) {
    const float4 N0 = s_nl[cy][cx], C0 = s_ca[cy][cx];
    const float2 A0 = s_ag[cy][cx];
    const float l0 = N0.w;
    float dcx = P0.x - p.camera.x, dcy = P0.y - p.camera.y, dcz = P0.z - p.camera.z;
    const float dc = sqrtf(dcx * dcx + dcy * dcy + dcz * dcz);
    // exp(-a)*exp(-b)*exp(-c) as one exp2 of the scaled sum
    const float kz = -1.4426950408889634f / (0.1f * dc + 1e-4f);
    const float kl = -1.4426950408889634f / (0.3f * fmaxf(l0, 0.5f) + 1e-3f);
    const float ka = -1.4426950408889634f * 4.0f;
    float sx = 0, sy = 0, sz = 0, wsum = 0;
#pragma unroll
    for (int dy = -2; dy <= 2; ++dy) {
#pragma unroll
      for (int dx = -2; dx <= 2; ++dx) {
        const int ly = cy + dy * (1 << STEP), lx = cx + dx * (1 << STEP);
        const float4 P = s_pk[ly][lx];
        const float4 N = s_nl[ly][lx], C = s_ca[ly][lx];
        const float2 A = s_ag[ly][lx];
        float nd = N.x * N0.x + (N.y * N0.y + N.z * N0.z);
        float wn = rm_pow16f(fmaxf(nd, 0.0f));
        float ex = P.x - P0.x, ey = P.y - P0.y, ez = P.z - P0.z;
        float ax = C.w - C0.w, ay = A.x - A0.x, az = A.y - A0.y;
        float e = fast_len(ex * ex + ey * ey + ez * ez) * kz + fabsf(N.w - l0) * kl +
                  fast_len(ax * ax + ay * ay + az * az) * ka;
        float w = wn * exp2f(e);
        sx += w * C.x; sy += w * C.y; sz += w * C.z;
        wsum += w;
      }
    }
    if (wsum > 1e-12f) { const float iw = 1.0f / wsum; rx = sx * iw; ry = sy * iw; rz = sz * iw; }
    else { rx = C0.x; ry = C0.y; rz = C0.z; }
  }
  st3(out, id, rx, ry, rz);
  if (rgb) {
    rgb[size_t(id) * 3] = tonemap8(rx); rgb[size_t(id) * 3 + 1] = tonemap8(ry); rgb[size_t(id) * 3 + 2] = tonemap8(rz);
  }
}

}  // namespace

cudaError_t launch_atrous_tiled(int step, const Params& p, const GBufSoA& gb, const float* in, float* out,
                                uint8_t* rgb, cudaStream_t st) {
  const dim3 blk(kTX, kTY), grd((p.width + kTX - 1) / kTX, (p.height + kTY - 1) / kTY);
  if (step == 0) k_denoise_atrous_tiled<0><<<grd, blk, 0, st>>>(p, gb, in, out, rgb);
  else k_denoise_atrous_tiled<1><<<grd, blk, 0, st>>>(p, gb, in, out, rgb);
  return cudaGetLastError();
}

}  // namespace rmd
