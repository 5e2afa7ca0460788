// rm_denoise.cu - edge-guided spatiotemporal denoiser and tonemap (sm_100a).
//
// The reference runs, after ReSTIR shading, a temporal pass, two 5x5 a-trous
// passes and a tonemap (src/engine/pathtrace.metal:1259-1363, chained by
// src/engine/metal.mm:321-366).  These are screen-space passes over SoA
// G-buffer planes (float4 pos|kind, normal|rough, albedo|metallic): the bound
// is HBM bandwidth, so every pixel is read with 128-bit loads and the second
// a-trous pass writes the RGB8 image itself (the tonemap is fused into it).
//
// The temporal pass and the tonemap are exact (bit-equal to the CPU oracle).
// The a-trous weights use the hardware exp2 through __expf on the sum of the
// three exponents, exp(-a)*exp(-b)*exp(-c) = exp(-(a+b+c)); this is the one
// stage of the path whose parity is a tolerance (1e-4 relative), not bits.
#include <cuda_runtime.h>

#include "rm_device.cuh"
#include "rm_launch.h"

namespace rmd {

__device__ __forceinline__ float luma(float r, float g, float b) { return 0.2126f * r + 0.7152f * g + 0.0722f * b; }

__device__ __forceinline__ float3 ld3(const float* __restrict__ a, uint32_t i) {
  return make_float3(a[size_t(i) * 3], a[size_t(i) * 3 + 1], a[size_t(i) * 3 + 2]);
}
__device__ __forceinline__ void st3(float* __restrict__ a, uint32_t i, float x, float y, float z) {
  a[size_t(i) * 3] = x; a[size_t(i) * 3 + 1] = y; a[size_t(i) * 3 + 2] = z;
}

// K6 denoise_temporal (pathtrace.metal:1263-1314)
__global__ void __launch_bounds__(256) k_denoise_temporal(Params p, GBufSoA gb, GBufSoA hg,
                                                          const float* __restrict__ cur,
                                                          const float* __restrict__ hist, float* __restrict__ out) {
  const uint32_t id = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t npix = uint32_t(p.width) * uint32_t(p.height);
  if (id >= npix) return;
  const int x = int(id % uint32_t(p.width)), y = int(id / uint32_t(p.width));
  const float3 c = ld3(cur, id);
  const float4 PK = gb.pos_kind[id];
  if (p.hasHistory == 0 || __float_as_int(PK.w) != 1) { st3(out, id, c.x, c.y, c.z); return; }
  float mnx = c.x, mny = c.y, mnz = c.z, mxx = c.x, mxy = c.y, mxz = c.z;
  for (int dy = -1; dy <= 1; ++dy)
    for (int dx = -1; dx <= 1; ++dx) {
      int nx = x + dx, ny = y + dy;
      if (nx < 0 || ny < 0 || nx >= p.width || ny >= p.height) continue;
      const float3 v = ld3(cur, uint32_t(ny) * uint32_t(p.width) + uint32_t(nx));
      mnx = fminf(mnx, v.x); mny = fminf(mny, v.y); mnz = fminf(mnz, v.z);
      mxx = fmaxf(mxx, v.x); mxy = fmaxf(mxy, v.y); mxz = fmaxf(mxz, v.z);
    }
  float ox = c.x, oy = c.y, oz = c.z;
  const rm_camera& pc = p.prevCamera;
  float pdx = PK.x - pc.x, pdy = PK.y - pc.y, pdz = PK.z - pc.z;
  float ccx = pc.m0 * pdx + pc.m3 * pdy + pc.m6 * pdz;
  float ccy = pc.m1 * pdx + pc.m4 * pdy + pc.m7 * pdz;
  float ccz = pc.m2 * pdx + pc.m5 * pdy + pc.m8 * pdz;
  if (ccz > 1e-6f) {
    float ppx = pc.focal * ccx / ccz + float(p.width) * 0.5f;
    float ppy = float(p.height) * 0.5f - pc.focal * ccy / ccz;
    if (ppx >= 0.0f && ppx < float(p.width) && ppy >= 0.0f && ppy < float(p.height)) {
      const uint32_t hidx = uint32_t(int(floorf(ppy))) * uint32_t(p.width) + uint32_t(int(floorf(ppx)));
      const float4 HK = hg.pos_kind[hidx];
      if (__float_as_int(HK.w) == 1) {
        const float4 HN = hg.nor_rough[hidx];
        const float4 CN = gb.nor_rough[id];
        float ddx = PK.x - HK.x, ddy = PK.y - HK.y, ddz = PK.z - HK.z;
        float dd = sqrtf(ddx * ddx + ddy * ddy + ddz * ddz);
        float dcx = PK.x - p.camera.x, dcy = PK.y - p.camera.y, dcz = PK.z - p.camera.z;
        float dc = sqrtf(dcx * dcx + dcy * dcy + dcz * dcz);
        if (dd < 0.02f * dc + 1e-3f && (CN.x * HN.x + (CN.y * HN.y + CN.z * HN.z)) > 0.9f) {
          const float3 h = ld3(hist, hidx);
          float hx = fminf(fmaxf(h.x, mnx), mxx), hy = fminf(fmaxf(h.y, mny), mxy), hz = fminf(fmaxf(h.z, mnz), mxz);
          ox = hx + (c.x - hx) * 0.2f; oy = hy + (c.y - hy) * 0.2f; oz = hz + (c.z - hz) * 0.2f;
        }
      }
    }
  }
  st3(out, id, ox, oy, oz);
}

// K7 denoise_atrous (pathtrace.metal:1315-1354); when rgb != nullptr the
// tonemap of K8 (:1355-1363) is applied to the result as well.
__global__ void __launch_bounds__(256) k_denoise_atrous(Params p, GBufSoA gb, const float* __restrict__ in,
                                                        float* __restrict__ out, int step, uint8_t* __restrict__ rgb) {
  const uint32_t id = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t npix = uint32_t(p.width) * uint32_t(p.height);
  if (id >= npix) return;
  const int x = int(id % uint32_t(p.width)), y = int(id / uint32_t(p.width));
  const float4 P0 = gb.pos_kind[id];
  float rx = 0, ry = 0, rz = 0;
  if (__float_as_int(P0.w) != 0) {
    const float3 c0 = ld3(in, id);
    const float4 N0 = gb.nor_rough[id], A0 = gb.alb_met[id];
    const float l0 = luma(c0.x, c0.y, c0.z);
    float dcx = P0.x - p.camera.x, dcy = P0.y - p.camera.y, dcz = P0.z - p.camera.z;
    const float dc = sqrtf(dcx * dcx + dcy * dcy + dcz * dcz);
    const float inv_z = 1.0f / (0.1f * dc + 1e-4f);
    const float inv_l = 1.0f / (0.3f * fmaxf(l0, 0.5f) + 1e-3f);
    const int stride = 1 << step;
    float sx = 0, sy = 0, sz = 0, wsum = 0;
#pragma unroll
    for (int dy = -2; dy <= 2; ++dy) {
      const int ny = y + dy * stride;
      if (ny < 0 || ny >= p.height) continue;
#pragma unroll
      for (int dx = -2; dx <= 2; ++dx) {
        const int nx = x + dx * stride;
        if (nx < 0 || nx >= p.width) continue;
        const uint32_t n = uint32_t(ny) * uint32_t(p.width) + uint32_t(nx);
        const float4 P = gb.pos_kind[n];
        if (__float_as_int(P.w) == 0) continue;
        const float4 N = gb.nor_rough[n], A = gb.alb_met[n];
        const float3 c = ld3(in, n);
        float nd = N.x * N0.x + (N.y * N0.y + N.z * N0.z);
        float wn = rm_pow16f(fmaxf(nd, 0.0f));
        float ex = P.x - P0.x, ey = P.y - P0.y, ez = P.z - P0.z;
        float ax = A.x - A0.x, ay = A.y - A0.y, az = A.z - A0.z;
        float e = sqrtf(ex * ex + ey * ey + ez * ez) * inv_z + fabsf(luma(c.x, c.y, c.z) - l0) * inv_l +
                  sqrtf(ax * ax + ay * ay + az * az) * 4.0f;
        float w = wn * __expf(-e);
        sx += w * c.x; sy += w * c.y; sz += w * c.z;
        wsum += w;
      }
    }
    if (wsum > 1e-12f) { const float iw = 1.0f / wsum; rx = sx * iw; ry = sy * iw; rz = sz * iw; }
    else { rx = c0.x; ry = c0.y; rz = c0.z; }
  }
  st3(out, id, rx, ry, rz);
  if (rgb) {
    rgb[size_t(id) * 3] = tonemap8(rx); rgb[size_t(id) * 3 + 1] = tonemap8(ry); rgb[size_t(id) * 3 + 2] = tonemap8(rz);
  }
}

// K8 denoise_tonemap (pathtrace.metal:1355-1363), used when the denoiser is off.
__global__ void __launch_bounds__(256) k_tonemap(const float* __restrict__ in, uint8_t* __restrict__ rgb, uint32_t n3) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n3) return;
  rgb[i] = tonemap8(in[i]);
}

// ---- tiled versions --------------------------------------------------------
//
// 32 x 8 pixels per block.  The neighbourhood of the tile (halo 1 for the
// temporal clamp, 2 * stride for a-trous) is staged once in shared memory with
// coalesced 128-bit loads, so each G-buffer / colour byte leaves HBM (or L2)
// about once instead of once per tap.

constexpr int kTX = 32, kTY = 8;

__global__ void __launch_bounds__(kTX* kTY) k_denoise_temporal_tiled(Params p, GBufSoA gb, GBufSoA hg,
                                                                     const float* __restrict__ cur,
                                                                     const float* __restrict__ hist,
                                                                     float* __restrict__ out) {
  __shared__ float3 sc[kTY + 2][kTX + 2];
  const int W = p.width, H = p.height;
  const int x0 = blockIdx.x * kTX, y0 = blockIdx.y * kTY;
  const int tid = threadIdx.y * kTX + threadIdx.x;
  for (int k = tid; k < (kTX + 2) * (kTY + 2); k += kTX * kTY) {
    const int lx = k % (kTX + 2), ly = k / (kTX + 2);
    const int gx = x0 + lx - 1, gy = y0 + ly - 1;
    float3 v = make_float3(0.f, 0.f, 0.f);
    if (gx >= 0 && gy >= 0 && gx < W && gy < H) v = ld3(cur, uint32_t(gy) * uint32_t(W) + uint32_t(gx));
    sc[ly][lx] = v;
  }
  __syncthreads();
  const int x = x0 + threadIdx.x, y = y0 + threadIdx.y;
  if (x >= W || y >= H) return;
  const uint32_t id = uint32_t(y) * uint32_t(W) + uint32_t(x);
  const float3 c = sc[threadIdx.y + 1][threadIdx.x + 1];
  const float4 PK = gb.pos_kind[id];
  if (p.hasHistory == 0 || __float_as_int(PK.w) != 1) { st3(out, id, c.x, c.y, c.z); return; }
  float mnx = c.x, mny = c.y, mnz = c.z, mxx = c.x, mxy = c.y, mxz = c.z;
#pragma unroll
  for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
    for (int dx = -1; dx <= 1; ++dx) {
      const int nx = x + dx, ny = y + dy;
      if (nx < 0 || ny < 0 || nx >= W || ny >= H) continue;
      const float3 v = sc[threadIdx.y + 1 + dy][threadIdx.x + 1 + dx];
      mnx = fminf(mnx, v.x); mny = fminf(mny, v.y); mnz = fminf(mnz, v.z);
      mxx = fmaxf(mxx, v.x); mxy = fmaxf(mxy, v.y); mxz = fmaxf(mxz, v.z);
    }
  float ox = c.x, oy = c.y, oz = c.z;
  const rm_camera& pc = p.prevCamera;
  float pdx = PK.x - pc.x, pdy = PK.y - pc.y, pdz = PK.z - pc.z;
  float ccx = pc.m0 * pdx + pc.m3 * pdy + pc.m6 * pdz;
  float ccy = pc.m1 * pdx + pc.m4 * pdy + pc.m7 * pdz;
  float ccz = pc.m2 * pdx + pc.m5 * pdy + pc.m8 * pdz;
  if (ccz > 1e-6f) {
    float ppx = pc.focal * ccx / ccz + float(W) * 0.5f;
    float ppy = float(H) * 0.5f - pc.focal * ccy / ccz;
    if (ppx >= 0.0f && ppx < float(W) && ppy >= 0.0f && ppy < float(H)) {
      const uint32_t hidx = uint32_t(int(floorf(ppy))) * uint32_t(W) + uint32_t(int(floorf(ppx)));
      const float4 HK = hg.pos_kind[hidx];
      if (__float_as_int(HK.w) == 1) {
        const float4 HN = hg.nor_rough[hidx];
        const float4 CN = gb.nor_rough[id];
        float ddx = PK.x - HK.x, ddy = PK.y - HK.y, ddz = PK.z - HK.z;
        float dd = sqrtf(ddx * ddx + ddy * ddy + ddz * ddz);
        float dcx = PK.x - p.camera.x, dcy = PK.y - p.camera.y, dcz = PK.z - p.camera.z;
        float dc = sqrtf(dcx * dcx + dcy * dcy + dcz * dcz);
        if (dd < 0.02f * dc + 1e-3f && (CN.x * HN.x + (CN.y * HN.y + CN.z * HN.z)) > 0.9f) {
          const float3 h = ld3(hist, hidx);
          float hx = fminf(fmaxf(h.x, mnx), mxx), hy = fminf(fmaxf(h.y, mny), mxy), hz = fminf(fmaxf(h.z, mnz), mxz);
          ox = hx + (c.x - hx) * 0.2f; oy = hy + (c.y - hy) * 0.2f; oz = hz + (c.z - hz) * 0.2f;
        }
      }
    }
  }
  st3(out, id, ox, oy, oz);
}

cudaError_t launch_denoise_stage(int stage, const Params& p, const GBufSoA& gb, const GBufSoA& hg, const float* in,
                                 const float* hist_in, float* out, uint8_t* rgb, cudaStream_t st) {
  const dim3 blk(kTX, kTY), grd((p.width + kTX - 1) / kTX, (p.height + kTY - 1) / kTY);
  if (stage == 0) {
    k_denoise_temporal_tiled<<<grd, blk, 0, st>>>(p, gb, hg, in, hist_in, out);
    return cudaGetLastError();
  }
  return launch_atrous_tiled(stage - 1, p, gb, in, out, rgb, st);
}

cudaError_t launch_tonemap(const float* hdr, uint8_t* rgb, uint32_t npix, cudaStream_t st) {
  const uint32_t n3 = npix * 3;
  k_tonemap<<<(n3 + 255) / 256, 256, 0, st>>>(hdr, rgb, n3);
  return cudaGetLastError();
}

}  // namespace rmd
