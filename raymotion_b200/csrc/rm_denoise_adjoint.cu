// rm_denoise_adjoint.cu - the denoiser's backward pass (pathtrace.metal:
// 1263-1354): the transpose of the temporal blend and of the two a-trous
// passes as functions of the colour they filter and of the G-buffer albedo in
// their weights, the G-buffer geometry and the history colour held (the
// frame's checkpoint).  It turns dL/d(denoised image) into dL/d(the ReSTIR
// shade's HDR image) and dL/d(G-buffer albedo), which the path-replay adjoint
// then takes.
//
// An a-trous pass is out_i = sum_j w_ij c_j / W_i, W_i = sum_j w_ij (out_i = c_i
// when W_i <= 1e-12; 0 on kind-0 pixels), with
//   w_ij = pow16(max(n_i.n_j, 0)) exp(-|p_j - p_i| / s_i) exp(-|l_j - l_i| / t_i)
//          exp(-|a_j - a_i| / 0.25),  l = luma(c), t_i = 0.3 max(l_i, 0.5) + 1e-3,
// so besides the linear term w_ij / W_i each colour moves the weights through
// its luma:  dL/dw_ij = g_i . (c_j - out_i) / W_i,  dw_ij/dl_j = -w_ij sgn(l_j -
// l_i) / t_i,  dw_ij/dl_i = w_ij (sgn(l_j - l_i) / t_i + |l_j - l_i| t_i' / t_i^2).
// The weights also move with the G-buffer albedo of both pixels (the first
// hit's material albedo times its texel): dw_ij/da_j = -w_ij u_ij / 0.25 and
// dw_ij/da_i = w_ij u_ij / 0.25, u_ij the unit vector of a_j - a_i; those
// gradients go to the materials through the path-replay adjoint, which knows
// each pixel's first hit.  The forward pass is recomputed here with the
// library's exp and sqrt (the oracle's exact form; the frame's own a-trous
// kernel uses exp2 / rsqrt approximations within 1e-4), keeping out_i and W_i
// for the backward.
#include <cuda_runtime.h>

#include "rm_device.cuh"
#include "rm_launch.h"

namespace rmd {

namespace {

__device__ __forceinline__ float lum(const float* c) { return 0.2126f * c[0] + 0.7152f * c[1] + 0.0722f * c[2]; }

// The weight of tap j for centre i (both kind != 0), the oracle's k_atrous.
__device__ __forceinline__ float atrous_w(const GBufSoA& gb, uint32_t i, uint32_t j, float dc_i, float li,
                                          float lj) {
  const float4 Pi = gb.pos_kind[i], Pj = gb.pos_kind[j];
  const float4 Ni = gb.nor_rough[i], Nj = gb.nor_rough[j];
  const float4 Ai = gb.alb_met[i], Aj = gb.alb_met[j];
  const float nd = Nj.x * Ni.x + (Nj.y * Ni.y + Nj.z * Ni.z);
  const float wn = rm_pow16f(fmaxf(nd, 0.0f));
  const float ex = Pj.x - Pi.x, ey = Pj.y - Pi.y, ez = Pj.z - Pi.z;
  const float wz = expf(-sqrtf(ex * ex + ey * ey + ez * ez) / (0.1f * dc_i + 1e-4f));
  const float wl = expf(-fabsf(lj - li) / (0.3f * fmaxf(li, 0.5f) + 1e-3f));
  const float ax = Aj.x - Ai.x, ay = Aj.y - Ai.y, az = Aj.z - Ai.z;
  const float wa = expf(-sqrtf(ax * ax + ay * ay + az * az) / 0.25f);
  return wn * wz * wl * wa;
}

// (a_j - a_i) / (0.25 |a_j - a_i|), zero for equal albedos: dlog wa_ij / da_i
__device__ __forceinline__ float3 alb_dir(const GBufSoA& gb, uint32_t i, uint32_t j) {
  const float4 Ai = gb.alb_met[i], Aj = gb.alb_met[j];
  const float ax = Aj.x - Ai.x, ay = Aj.y - Ai.y, az = Aj.z - Ai.z;
  const float l = sqrtf(ax * ax + ay * ay + az * az);
  if (!(l > 0.0f)) return make_float3(0.f, 0.f, 0.f);
  const float k = 1.0f / (0.25f * l);
  return make_float3(ax * k, ay * k, az * k);
}

__device__ __forceinline__ float cam_dist(const Params& p, const float4& P) {
  const float dx = P.x - p.camera.x, dy = P.y - p.camera.y, dz = P.z - p.camera.z;
  return sqrtf(dx * dx + dy * dy + dz * dz);
}

// forward a-trous pass: out and W per pixel (W < 0 marks out = c or 0)
__global__ void __launch_bounds__(256) k_atrous_fwd(Params p, GBufSoA gb, const float* __restrict__ in,
                                                    float* __restrict__ out, float* __restrict__ wsum, int step) {
  const uint32_t id = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t npix = uint32_t(p.width) * uint32_t(p.height);
  if (id >= npix) return;
  const int x = int(id % uint32_t(p.width)), y = int(id / uint32_t(p.width));
  const float4 P0 = gb.pos_kind[id];
  if (__float_as_int(P0.w) == 0) {
    out[size_t(id) * 3] = out[size_t(id) * 3 + 1] = out[size_t(id) * 3 + 2] = 0.0f;
    wsum[id] = -1.0f;
    return;
  }
  const float c0[3] = {in[size_t(id) * 3], in[size_t(id) * 3 + 1], in[size_t(id) * 3 + 2]};
  const float l0 = lum(c0), dc = cam_dist(p, P0);
  const int stride = 1 << step;
  float s[3] = {0.f, 0.f, 0.f}, W = 0.0f;
  for (int dy = -2; dy <= 2; ++dy)
    for (int dx = -2; dx <= 2; ++dx) {
      const int nx = x + dx * stride, ny = y + dy * stride;
      if (nx < 0 || ny < 0 || nx >= p.width || ny >= p.height) continue;
      const uint32_t n = uint32_t(ny) * uint32_t(p.width) + uint32_t(nx);
      if (__float_as_int(gb.pos_kind[n].w) == 0) continue;
      const float c[3] = {in[size_t(n) * 3], in[size_t(n) * 3 + 1], in[size_t(n) * 3 + 2]};
      const float w = atrous_w(gb, id, n, dc, l0, lum(c));
      for (int k = 0; k < 3; ++k) s[k] += w * c[k];
      W += w;
    }
  if (W > 1e-12f) {
    for (int k = 0; k < 3; ++k) out[size_t(id) * 3 + k] = s[k] / W;
    wsum[id] = W;
  } else {
    for (int k = 0; k < 3; ++k) out[size_t(id) * 3 + k] = c0[k];
    wsum[id] = -1.0f;
  }
}

// backward a-trous pass: g_in_j = sum over the centres i whose 5x5 footprint
// holds j of the linear and the weight terms, plus j's own luma term as a
// centre (gathered, one thread per j)
__global__ void __launch_bounds__(256) k_atrous_bwd(Params p, GBufSoA gb, const float* __restrict__ in,
                                                    const float* __restrict__ out, const float* __restrict__ wsum,
                                                    const float* __restrict__ g_out, float* __restrict__ g_in,
                                                    float* __restrict__ g_alb, int step) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t npix = uint32_t(p.width) * uint32_t(p.height);
  if (j >= npix) return;
  const int x = int(j % uint32_t(p.width)), y = int(j / uint32_t(p.width));
  float gj[3] = {0.f, 0.f, 0.f}, ga[3] = {0.f, 0.f, 0.f};
  const float4 Pj = gb.pos_kind[j];
  const int stride = 1 << step;
  const float cj[3] = {in[size_t(j) * 3], in[size_t(j) * 3 + 1], in[size_t(j) * 3 + 2]};
  const float lj = lum(cj);
  if (__float_as_int(Pj.w) != 0) {
    float dl_j = 0.0f;  // dL/d l_j through the weights of the centres around j and of j itself
    // j as a tap of centre i = j - offset (the footprint is symmetric)
    for (int dy = -2; dy <= 2; ++dy)
      for (int dx = -2; dx <= 2; ++dx) {
        const int ix = x - dx * stride, iy = y - dy * stride;
        if (ix < 0 || iy < 0 || ix >= p.width || iy >= p.height) continue;
        const uint32_t i = uint32_t(iy) * uint32_t(p.width) + uint32_t(ix);
        const float4 Pi = gb.pos_kind[i];
        if (__float_as_int(Pi.w) == 0) continue;
        const float Wi = wsum[i];
        const float gi[3] = {g_out[size_t(i) * 3], g_out[size_t(i) * 3 + 1], g_out[size_t(i) * 3 + 2]};
        if (!(Wi > 0.0f)) {  // out_i = c_i
          if (i == j) for (int k = 0; k < 3; ++k) gj[k] += gi[k];
          continue;
        }
        const float ci[3] = {in[size_t(i) * 3], in[size_t(i) * 3 + 1], in[size_t(i) * 3 + 2]};
        const float li = lum(ci);
        const float w = atrous_w(gb, i, j, cam_dist(p, Pi), li, lj);
        const float ti = 0.3f * fmaxf(li, 0.5f) + 1e-3f;
        float dw = 0.0f;  // dL/dw_ij
        for (int k = 0; k < 3; ++k) {
          gj[k] += gi[k] * w / Wi;
          dw += gi[k] * (cj[k] - out[size_t(i) * 3 + k]) / Wi;
        }
        const float sg = lj > li ? 1.0f : (lj < li ? -1.0f : 0.0f);
        dl_j += dw * (-w * sg / ti);
        // j's albedo in wa_ij: dlog wa_ij / da_j = -(a_j - a_i) / (0.25 |.|)
        const float3 u = alb_dir(gb, i, j);
        ga[0] -= dw * w * u.x; ga[1] -= dw * w * u.y; ga[2] -= dw * w * u.z;
      }
    // j as the centre: its luma in |l_k - l_j| and in t_j
    const float Wj = wsum[j];
    if (Wj > 0.0f) {
      const float gjo[3] = {g_out[size_t(j) * 3], g_out[size_t(j) * 3 + 1], g_out[size_t(j) * 3 + 2]};
      const float tj = 0.3f * fmaxf(lj, 0.5f) + 1e-3f, dtj = lj > 0.5f ? 0.3f : 0.0f;
      const float dcj = cam_dist(p, Pj);
      for (int dy = -2; dy <= 2; ++dy)
        for (int dx = -2; dx <= 2; ++dx) {
          const int nx = x + dx * stride, ny = y + dy * stride;
          if (nx < 0 || ny < 0 || nx >= p.width || ny >= p.height) continue;
          const uint32_t n = uint32_t(ny) * uint32_t(p.width) + uint32_t(nx);
          if (__float_as_int(gb.pos_kind[n].w) == 0) continue;
          const float cn[3] = {in[size_t(n) * 3], in[size_t(n) * 3 + 1], in[size_t(n) * 3 + 2]};
          const float ln = lum(cn);
          const float w = atrous_w(gb, j, n, dcj, lj, ln);
          float dw = 0.0f;
          for (int k = 0; k < 3; ++k) dw += gjo[k] * (cn[k] - out[size_t(j) * 3 + k]) / Wj;
          const float d = ln - lj;
          const float sg = d > 0.0f ? 1.0f : (d < 0.0f ? -1.0f : 0.0f);
          dl_j += dw * w * (sg / tj + fabsf(d) * dtj / (tj * tj));
          // j's albedo as the centre: dlog wa_jn / da_j = (a_n - a_j) / (0.25 |.|)
          const float3 u = alb_dir(gb, j, n);
          ga[0] += dw * w * u.x; ga[1] += dw * w * u.y; ga[2] += dw * w * u.z;
        }
    }
    gj[0] += dl_j * 0.2126f; gj[1] += dl_j * 0.7152f; gj[2] += dl_j * 0.0722f;
  }
  for (int k = 0; k < 3; ++k) {
    g_in[size_t(j) * 3 + k] = gj[k];
    g_alb[size_t(j) * 3 + k] += ga[k];
  }
}

// backward temporal pass: o = h' + (c - h') 0.2 with h' = clamp(h, mn, mx)
// over the 3x3 neighbourhood of the current colour; the history is held, a
// clamped channel's 0.8 goes to the neighbour that set the bound (the first
// in the forward scan).  g_cur must be zero on entry (the clamp terms are
// scattered).
__global__ void __launch_bounds__(256) k_temporal_bwd(Params p, GBufSoA gb, GBufSoA hg, const float* __restrict__ cur,
                                                      const float* __restrict__ hist,
                                                      const float* __restrict__ g_out, float* __restrict__ g_cur) {
  const uint32_t id = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t npix = uint32_t(p.width) * uint32_t(p.height);
  if (id >= npix) return;
  const float g[3] = {g_out[size_t(id) * 3], g_out[size_t(id) * 3 + 1], g_out[size_t(id) * 3 + 2]};
  const int x = int(id % uint32_t(p.width)), y = int(id / uint32_t(p.width));
  const float4 PK = gb.pos_kind[id];
  bool blend = false;
  uint32_t hidx = 0;
  if (p.hasHistory != 0 && __float_as_int(PK.w) == 1) {
    const rm_camera& pc = p.prevCamera;
    float pdx = PK.x - pc.x, pdy = PK.y - pc.y, pdz = PK.z - pc.z;
    float ccx = pc.m0 * pdx + pc.m3 * pdy + pc.m6 * pdz;
    float ccy = pc.m1 * pdx + pc.m4 * pdy + pc.m7 * pdz;
    float ccz = pc.m2 * pdx + pc.m5 * pdy + pc.m8 * pdz;
    if (ccz > 1e-6f) {
      float ppx = pc.focal * ccx / ccz + float(p.width) * 0.5f;
      float ppy = float(p.height) * 0.5f - pc.focal * ccy / ccz;
      if (ppx >= 0.0f && ppx < float(p.width) && ppy >= 0.0f && ppy < float(p.height)) {
        hidx = uint32_t(int(floorf(ppy))) * uint32_t(p.width) + uint32_t(int(floorf(ppx)));
        const float4 HK = hg.pos_kind[hidx];
        if (__float_as_int(HK.w) == 1) {
          const float4 HN = hg.nor_rough[hidx], CN = gb.nor_rough[id];
          float ddx = PK.x - HK.x, ddy = PK.y - HK.y, ddz = PK.z - HK.z;
          float dd = sqrtf(ddx * ddx + ddy * ddy + ddz * ddz);
          float dcx = PK.x - p.camera.x, dcy = PK.y - p.camera.y, dcz = PK.z - p.camera.z;
          float dc = sqrtf(dcx * dcx + dcy * dcy + dcz * dcz);
          blend = dd < 0.02f * dc + 1e-3f && (CN.x * HN.x + (CN.y * HN.y + CN.z * HN.z)) > 0.9f;
        }
      }
    }
  }
  if (!blend) {
    for (int k = 0; k < 3; ++k) atomicAdd(g_cur + size_t(id) * 3 + k, g[k]);
    return;
  }
  for (int k = 0; k < 3; ++k) {
    const float c = cur[size_t(id) * 3 + k];
    float mn = c, mx = c;
    uint32_t amn = id, amx = id;
    for (int dy = -1; dy <= 1; ++dy)
      for (int dx = -1; dx <= 1; ++dx) {
        const int nx = x + dx, ny = y + dy;
        if (nx < 0 || ny < 0 || nx >= p.width || ny >= p.height) continue;
        const uint32_t n = uint32_t(ny) * uint32_t(p.width) + uint32_t(nx);
        const float v = cur[size_t(n) * 3 + k];
        if (v < mn) { mn = v; amn = n; }
        if (v > mx) { mx = v; amx = n; }
      }
    const float h = hist[size_t(hidx) * 3 + k];
    atomicAdd(g_cur + size_t(id) * 3 + k, 0.2f * g[k]);
    if (h < mn) atomicAdd(g_cur + size_t(amn) * 3 + k, 0.8f * g[k]);
    else if (h > mx) atomicAdd(g_cur + size_t(amx) * 3 + k, 0.8f * g[k]);
  }
}

}  // namespace

cudaError_t launch_denoise_backward(const Params& p, const GBufSoA& gb, const GBufSoA& hg, const float* hdr,
                                    const float* hist_col, const float* dLdout, float* scratch, float* dLdhdr,
                                    float* dLdalb, cudaStream_t st) {
  const size_t npix = size_t(p.width) * size_t(p.height);
  const unsigned g = unsigned((npix + 255) / 256);
  // scratch: T, A0, A1, G1 (3 floats per pixel each), W0, W1 (1 each)
  float* T = scratch;
  float* A0 = T + npix * 3;
  float* A1 = A0 + npix * 3;
  float* G = A1 + npix * 3;
  float* W0 = G + npix * 3;
  float* W1 = W0 + npix;
  cudaError_t e = launch_denoise_stage(0, p, gb, hg, hdr, hist_col, T, nullptr, st);  // the frame's own temporal pass
  if (e != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(dLdalb, 0, npix * 3 * sizeof(float), st)) != cudaSuccess) return e;
  k_atrous_fwd<<<g, 256, 0, st>>>(p, gb, T, A0, W0, 0);
  k_atrous_fwd<<<g, 256, 0, st>>>(p, gb, A0, A1, W1, 1);
  k_atrous_bwd<<<g, 256, 0, st>>>(p, gb, A0, A1, W1, dLdout, G, dLdalb, 1);   // dL/dA0
  k_atrous_bwd<<<g, 256, 0, st>>>(p, gb, T, A0, W0, G, A1, dLdalb, 0);        // dL/dT (into A1)
  if ((e = cudaMemsetAsync(dLdhdr, 0, npix * 3 * sizeof(float), st)) != cudaSuccess) return e;
  k_temporal_bwd<<<g, 256, 0, st>>>(p, gb, hg, hdr, hist_col, A1, dLdhdr);
  return cudaGetLastError();
}

}  // namespace rmd
