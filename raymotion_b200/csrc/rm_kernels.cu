// rm_kernels.cu - frame kernels of the path-tracing hot path (sm_100a).
//
// Each kernel reproduces one Metal kernel of the reference
// (src/engine/pathtrace.metal, cited per kernel) on the device layout of
// rm_device.cuh.  Compiled with -fmad=false: on identical RNG streams the
// radiance equals the CPU oracle's bit for bit.
#include <cuda_runtime.h>

#include "rm_device.cuh"
#include "rm_launch.h"

namespace rmd {

// Warp-aggregated counter update; every lane of the warp must reach it.
__device__ __forceinline__ void warp_count(unsigned long long* ctr, uint32_t v) {
  unsigned long long s = __reduce_add_sync(0xffffffffu, v);
  if ((threadIdx.x & 31) == 0 && s) atomicAdd(ctr, s);
}

// Counters of a kernel: [0] path samples, [1] rays, [2] BVH nodes visited,
// [3] triangle tests.  Every lane of the warp must reach this.
__device__ __forceinline__ void flush_counts(unsigned long long* ctr, uint32_t samples, uint32_t rays,
                                             uint32_t nodes, uint32_t tests) {
  warp_count(ctr + 0, samples);
  warp_count(ctr + 1, rays);
  warp_count(ctr + 2, nodes);
  warp_count(ctr + 3, tests);
}

__device__ __forceinline__ void clamp3(const Params& p, float& r, float& g, float& b) {
  if (p.clamp_value > 0.0f) {
    r = fminf(r, p.clamp_value); g = fminf(g, p.clamp_value); b = fminf(b, p.clamp_value);
  }
}

// K1 render_paths (pathtrace.metal:739-769) for LANES == 1, and K2
// render_paths_simd (:773-815) for LANES in {8, 32}: LANES threads per pixel,
// each a strided subset of the samples, reduced with butterfly shuffles that
// never leave the pixel's lane group.
template <int LANES>
__global__ void __launch_bounds__(256) k_render_paths(Scene s, Params p, uint64_t seed, float* __restrict__ hdr,
                                                      uint8_t* __restrict__ rgb, uint32_t* __restrict__ dbg,
                                                      unsigned long long* ctr, uint32_t* err) {
  const uint64_t gid = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const uint32_t npix = uint32_t(p.width) * uint32_t(p.height);
  const uint32_t pixel = uint32_t(gid / LANES), lane = uint32_t(gid % LANES);
  uint32_t taken = 0, rays = 0, nodes = 0, tests = 0;
  if (pixel < npix) {
    const uint32_t x = pixel % uint32_t(p.width), y = pixel / uint32_t(p.width);
    Tracer pt(s, p, err);
    uint64_t sd = seed_pixel(seed, x, y);
    if (LANES > 1) sd ^= uint64_t(lane) * 0x94D049BB133111EBull;
    pt.rng.seed(sd);
    float sr = 0, sg = 0, sb = 0, sum_l = 0, sum_l2 = 0;
    int n = 0;
    if (LANES == 1) {
      for (int si = 0; si < p.spp; ++si) {
        float sx, sy, cr, cg, cb;
        pt.jitter(x, y, sx, sy);
        pt.sample_sensor(sx, sy, p.bounces, cr, cg, cb);
        clamp3(p, cr, cg, cb);
        sr += cr; sg += cg; sb += cb;
        ++n;
        if (p.adapt_min > 0) {
          float lum = cr * 0.2126f + cg * 0.7152f + cb * 0.0722f;
          sum_l += lum; sum_l2 += lum * lum;
          if (n >= p.adapt_min && n > 1 && n % p.adapt_step == 0) {
            float mean = sum_l / float(n);
            float var = fmaxf(0.0f, (sum_l2 - sum_l * mean) / float(n - 1));
            float thr = p.adapt_rel * mean + p.adapt_abs;
            if (var < thr * thr) break;
          }
        }
      }
      taken = uint32_t(n);
    } else {
      const uint32_t group = (threadIdx.x & 31u) / LANES;
      const uint32_t mask = LANES == 32 ? 0xffffffffu : (((1u << LANES) - 1u) << (group * LANES));
      for (uint32_t base = 0; base < uint32_t(p.spp); base += LANES) {
        float cr = 0, cg = 0, cb = 0;
        if (base + lane < uint32_t(p.spp)) {
          float sx, sy;
          pt.jitter(x, y, sx, sy);
          pt.sample_sensor(sx, sy, p.bounces, cr, cg, cb);
          clamp3(p, cr, cg, cb);
          ++taken;
        }
        float lum = cr * 0.2126f + cg * 0.7152f + cb * 0.0722f;
        float lum2 = lum * lum;
#pragma unroll
        for (int m = 1; m < LANES; m <<= 1) {
          cr += __shfl_xor_sync(mask, cr, m, LANES);
          cg += __shfl_xor_sync(mask, cg, m, LANES);
          cb += __shfl_xor_sync(mask, cb, m, LANES);
          lum += __shfl_xor_sync(mask, lum, m, LANES);
          lum2 += __shfl_xor_sync(mask, lum2, m, LANES);
        }
        sr += cr; sg += cg; sb += cb; sum_l += lum; sum_l2 += lum2;
        n = int(min(base + uint32_t(LANES), uint32_t(p.spp)));
        if (p.adapt_min > 0 && n >= p.adapt_min && n > 1 && n % p.adapt_step == 0) {
          float mean = sum_l / float(n);
          float var = fmaxf(0.0f, (sum_l2 - sum_l * mean) / float(n - 1));
          float thr = p.adapt_rel * mean + p.adapt_abs;
          if (var < thr * thr) break;
        }
      }
    }
    uint32_t st = pt.rng.state;
    if (LANES > 1) {
      const uint32_t group = (threadIdx.x & 31u) / LANES;
      const uint32_t mask = LANES == 32 ? 0xffffffffu : (((1u << LANES) - 1u) << (group * LANES));
#pragma unroll
      for (int m = 1; m < LANES; m <<= 1) st ^= __shfl_xor_sync(mask, st, m, LANES);
    }
    rays = pt.rays; nodes = pt.nodes; tests = pt.tests;
    if (lane == 0) {
      float cr = sr / float(n), cg = sg / float(n), cb = sb / float(n);
      if (hdr) { hdr[size_t(pixel) * 3] = cr; hdr[size_t(pixel) * 3 + 1] = cg; hdr[size_t(pixel) * 3 + 2] = cb; }
      if (rgb) {
        rgb[size_t(pixel) * 3] = tonemap8(cr); rgb[size_t(pixel) * 3 + 1] = tonemap8(cg);
        rgb[size_t(pixel) * 3 + 2] = tonemap8(cb);
      }
      if (dbg) { dbg[size_t(pixel) * 2] = st; dbg[size_t(pixel) * 2 + 1] = uint32_t(n); }
    }
  }
  __syncwarp();
  flush_counts(ctr, taken, rays, nodes, tests);
}

// ---------------------------------------------------------------- ReSTIR

__device__ __forceinline__ int gkind(const GBufSoA& g, uint32_t i) { return __float_as_int(g.pos_kind[i].w); }

// K3 restir_generate (pathtrace.metal:817-917).  Ten 128-thread blocks per SM
// (48 registers, ~360 bytes of spills): the 32 candidates' shadow rays are
// latency-bound, and the extra warps outweigh the spills (13.1 / 13.3 against
// 13.4 / 13.6 ms at eight blocks and 64 registers on the 720p frame; six
// blocks at 80 registers, 15.0 ms).
__global__ void __launch_bounds__(128, 10) k_restir_generate(Scene s, Params p, uint64_t seed, GBufSoA gb, ResSoA ri,
                                                         unsigned long long* ctr, uint32_t* err) {
  const uint32_t id = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t npix = uint32_t(p.width) * uint32_t(p.height);
  uint32_t taken = 0, rays = 0, nodes = 0, tests = 0;
  if (id < npix) {
    const uint32_t x = id % uint32_t(p.width), y = id / uint32_t(p.width);
    Tracer pt(s, p, err);
    pt.rng.seed(seed_pixel(seed, x, y));
    gb.pos_kind[id] = make_float4(0.f, 0.f, 0.f, __int_as_float(0));
    ri.sumwu_m_valid[id] = make_float4(0.f, 0.f, 0.f, 0.f);
    float sx = float(x) + 1e-12f + (p.resolution - 2e-12f) * pt.U() - float(p.width) * 0.5f;
    float sy = float(p.height) * 0.5f - (float(y) + 1e-12f + (p.resolution - 2e-12f) * pt.U());
    const rm_camera& c = p.camera;
    float f2 = c.focal * c.focal;
    float dinv = 1.0f / sqrtf(sx * sx + sy * sy + f2);
    float tx = sx * dinv, ty = sy * dinv, tz = c.focal * dinv;
    float rdx = tx * c.m0 + (ty * c.m1 + tz * c.m2);
    float rdy = tx * c.m3 + (ty * c.m4 + tz * c.m5);
    float rdz = tx * c.m6 + (ty * c.m7 + tz * c.m8);
    Hit hit = pt.cast_alpha_ray(c.x, c.y, c.z, rdx, rdy, rdz, kFar);
    if (hit.tri >= 0) {
      float pnx = hit.nix, pny = hit.niy, pnz = hit.niz;
      float geom = hit.ngx * pnx + (hit.ngy * pny + hit.ngz * pnz);
      if (geom < 0.0f) { pnx = -pnx; pny = -pny; pnz = -pnz; }
      float ndot = rdx * pnx + (rdy * pny + rdz * pnz);
      if (ndot > 0.0f) { pnx = -pnx; pny = -pny; pnz = -pnz; }
      float wox = -rdx, woy = -rdy, woz = -rdz;
      float rough = hit.rough; if (rough < 0.0f) rough = 0.0f; if (rough > 1.0f) rough = 1.0f;
      float metallic = s.tris[hit.tri].metallic;
      if (metallic < 0.0f) metallic = 0.0f;
      if (metallic > 1.0f) metallic = 1.0f;
      const bool diel = hit.ior > 1.0001f;
      gb.nor_rough[id] = make_float4(pnx, pny, pnz, rough);
      gb.alb_met[id] = make_float4(hit.ar, hit.ag, hit.ab, metallic);
      gb.wo_ior[id] = make_float4(wox, woy, woz, diel ? hit.ior : 1.0f);
      gb.emi[id] = make_float4(hit.er, hit.eg, hit.eb, 0.f);
      gb.pos_kind[id] = make_float4(hit.px, hit.py, hit.pz, __int_as_float(diel ? 3 : 1));
      if (!diel && p.lights != 0 && p.light_total > 1e-12f) {
        int Mc = p.restir_candidates; if (Mc < 1) Mc = 1; if (Mc > 32) Mc = 32;
        float r2 = rough; if (r2 < 0.02f) r2 = 0.02f;
        float alpha2 = (r2 * r2) * (r2 * r2);
        float spec_prob = 0.05f + 0.95f * metallic; if (spec_prob > 0.98f) spec_prob = 0.98f;
        if (metallic >= 0.999f) spec_prob = 1.0f;
        const float px = hit.px, py = hit.py, pz = hit.pz;
        float sumWs = 0, sumWu = 0, sel_lx = 0, sel_ly = 0, sel_lz = 0, sel_nx = 0, sel_ny = 0, sel_nz = 0;
        float sel_er = 0, sel_eg = 0, sel_eb = 0, sel_alpha = 1, sel_ph = 0;
        bool have = false;
        int sel_li = 0;  // light index of the selected sample (kept in the reservoir's free word)
        const float sox = px + pnx * 0.002f, soy = py + pny * 0.002f, soz = pz + pnz * 0.002f;
        const Tracer::BsdfPrep bp =
            Tracer::prep_bsdf(wox, woy, woz, pnx, pny, pnz, alpha2, metallic, hit.ar, hit.ag, hit.ab);
        for (int j = 0; j < Mc; ++j) {
          float pick = pt.U() * p.light_total;
          const int li = pt.pick_light(pick);
          const LightRec t = load_light(s, li);
          float lu = pt.U(), lv = pt.U();
          if (lu + lv > 1.0f) { lu = 1.0f - lu; lv = 1.0f - lv; }
          float lw = 1.0f - lu - lv;
          float qx = lw * t.v0.x + (lu * t.v1.x + lv * t.v2.x);
          float qy = lw * t.v0.y + (lu * t.v1.y + lv * t.v2.y);
          float qz = lw * t.v0.z + (lu * t.v1.z + lv * t.v2.z);
          float ldx = qx - px, ldy = qy - py, ldz = qz - pz;
          float dist = sqrtf(ldx * ldx + ldy * ldy + ldz * ldz);
          float wu = 0, ws = 0, ph = 0;
          if (dist > 0.003f) {
            float inv = 1.0f / dist;
            float dxn = ldx * inv, dyn = ldy * inv, dzn = ldz * inv;
            float lcos = -(t.nn.x * dxn + (t.nn.y * dyn + t.nn.z * dzn));
            float scos = pnx * dxn + (pny * dyn + pnz * dzn);
            if (lcos > 1e-8f && scos > 1e-8f) {
              float ll = lum3(t.er, t.eg, t.eb); if (ll < 1e-6f) ll = 1e-6f;
              float q = dist * dist * ll / (lcos * p.light_total);
              if (q > 1e-12f) {
                Bsdf e = Tracer::eval_bsdf_prep(bp, dxn, dyn, dzn, wox, woy, woz, pnx, pny, pnz, alpha2, spec_prob);
                float Fr = t.er * e.r * scos * t.alpha, Fg = t.eg * e.g * scos * t.alpha,
                      Fb = t.eb * e.b * scos * t.alpha;
                ph = lum3(Fr, Fg, Fb);
                if (ph > 0.0f) {
                  wu = ph / q;
                  bool occ = pt.occluded(sox, soy, soz, dxn, dyn, dzn, dist - 0.003f);
                  if (!occ) ws = wu;
                }
              }
            }
          }
          sumWu += wu; sumWs += ws;
          float r = pt.U();
          if (ws > 0.0f && r * sumWs < ws) {
            have = true;
            sel_lx = qx; sel_ly = qy; sel_lz = qz;
            sel_nx = t.nn.x; sel_ny = t.nn.y; sel_nz = t.nn.z;
            sel_er = t.er; sel_eg = t.eg; sel_eb = t.eb; sel_alpha = t.alpha; sel_ph = ph;
            sel_li = li;
          }
        }
        if (have && sumWs > 0.0f && sumWu > 0.0f && sel_ph > 0.0f) {
          ri.lp_alpha[id] = make_float4(sel_lx, sel_ly, sel_lz, sel_alpha);
          ri.ln_phat[id] = make_float4(sel_nx, sel_ny, sel_nz, sel_ph);
          ri.le_sumws[id] = make_float4(sel_er, sel_eg, sel_eb, sumWs);
          ri.sumwu_m_valid[id] = make_float4(sumWu, __int_as_float(Mc), __int_as_float(1), __int_as_float(sel_li));
        }
      }
    }
    rays = pt.rays; nodes = pt.nodes; tests = pt.tests;
  }
  __syncwarp();
  flush_counts(ctr, taken, rays, nodes, tests);
}

// Reprojection into the previous camera (pathtrace.metal:957-966).
__device__ __forceinline__ bool reproject(const Params& p, float cx, float cy, float cz, uint32_t& hidx) {
  const rm_camera& pc = p.prevCamera;
  float pdx = cx - pc.x, pdy = cy - pc.y, pdz = cz - pc.z;
  float ccx = pc.m0 * pdx + pc.m3 * pdy + pc.m6 * pdz;
  float ccy = pc.m1 * pdx + pc.m4 * pdy + pc.m7 * pdz;
  float ccz = pc.m2 * pdx + pc.m5 * pdy + pc.m8 * pdz;
  if (!(ccz > 1e-6f)) return false;
  float ppx = pc.focal * ccx / ccz + float(p.width) * 0.5f;
  float ppy = float(p.height) * 0.5f - pc.focal * ccy / ccz;
  if (!(ppx >= 0.0f && ppx < float(p.width) && ppy >= 0.0f && ppy < float(p.height))) return false;
  hidx = uint32_t(int(floorf(ppy))) * uint32_t(p.width) + uint32_t(int(floorf(ppx)));
  return true;
}

// K4 restir_spatial (pathtrace.metal:919-1054).  Three 256-thread blocks per
// SM (80 registers, ~1 KB of spills, against two at 128): the neighbours'
// visibility rays are latency-bound, and the pass took 1.76 against 2.13 ms
// on the 720p frame (four blocks at 64 registers: 2.28 ms).
__global__ void __launch_bounds__(256, 3) k_restir_spatial(Scene s, Params p, uint64_t seed, GBufSoA gb, ResSoA ri,
                                                        ResSoA ro, GBufSoA hg, ResSoA hr, unsigned long long* ctr,
                                                        uint32_t* err) {
  const uint32_t id = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t npix = uint32_t(p.width) * uint32_t(p.height);
  uint32_t taken = 0, rays = 0, nodes = 0, tests = 0;
  if (id < npix) {
    const uint32_t x = id % uint32_t(p.width), y = id / uint32_t(p.width);
    const float4 R0 = ri.lp_alpha[id], R1 = ri.ln_phat[id], R2 = ri.le_sumws[id], R3 = ri.sumwu_m_valid[id];
    ro.lp_alpha[id] = R0; ro.ln_phat[id] = R1; ro.le_sumws[id] = R2; ro.sumwu_m_valid[id] = R3;
    const float4 PK = gb.pos_kind[id];
    int S = p.restir_spatial; if (S < 0) S = 0; if (S > 8) S = 8;
    if (__float_as_int(PK.w) == 1 && __float_as_int(R3.z) != 0 && S != 0) {
      float radius = p.restir_radius; if (!(radius > 0.0f)) radius = 16.0f;
      int mcap = p.restir_mcap; if (mcap < 1) mcap = 1;
      Tracer pt(s, p, err);
      pt.rng.seed(seed ^ (uint64_t(id + 1) * 0x9E3779B97F4A7C15ull) ^ kSpatialSeedXor);
      const float4 NR = gb.nor_rough[id], AM = gb.alb_met[id], WO = gb.wo_ior[id];
      const float cpx = PK.x, cpy = PK.y, cpz = PK.z, cnx = NR.x, cny = NR.y, cnz = NR.z;
      float rough = NR.w; if (rough < 0.0f) rough = 0.0f; if (rough > 1.0f) rough = 1.0f;
      float metallic = AM.w; if (metallic < 0.0f) metallic = 0.0f; if (metallic > 1.0f) metallic = 1.0f;
      float r2 = rough; if (r2 < 0.02f) r2 = 0.02f;
      float alpha2 = (r2 * r2) * (r2 * r2);
      float spec_prob = 0.05f + 0.95f * metallic; if (spec_prob > 0.98f) spec_prob = 0.98f;
      if (metallic >= 0.999f) spec_prob = 1.0f;
      float cur_sumWs = R2.w, cur_sumWu = R3.x;
      uint32_t cur_M = uint32_t(__float_as_int(R3.y));
      float4 cur0 = R0, cur1 = R1, cur2 = R2;  // lp|alpha, ln|p_hat, le|(sumWs)
      float cur_li = R3.w;                     // the sample's light index (bits)
      const float sox = cpx + cnx * 0.002f, soy = cpy + cny * 0.002f, soz = cpz + cnz * 0.002f;
      // target p_hat of a light sample at this pixel; false if it fails a test
      auto eval_at = [&](const float4& lpa, const float4& ln, const float4& le, float& ph, float& dist, float& dxn,
                         float& dyn, float& dzn) -> bool {
        float ldx = lpa.x - cpx, ldy = lpa.y - cpy, ldz = lpa.z - cpz;
        dist = sqrtf(ldx * ldx + ldy * ldy + ldz * ldz);
        if (!(dist > 0.003f)) return false;
        float inv = 1.0f / dist;
        dxn = ldx * inv; dyn = ldy * inv; dzn = ldz * inv;
        float lcos = -(ln.x * dxn + (ln.y * dyn + ln.z * dzn));
        float scos = cnx * dxn + (cny * dyn + cnz * dzn);
        if (!(lcos > 1e-8f && scos > 1e-8f)) return false;
        Bsdf e = Tracer::eval_bsdf(dxn, dyn, dzn, WO.x, WO.y, WO.z, cnx, cny, cnz, alpha2, metallic, spec_prob, AM.x,
                                   AM.y, AM.z);
        float Fr = le.x * e.r * scos * lpa.w, Fg = le.y * e.g * scos * lpa.w, Fb = le.z * e.b * scos * lpa.w;
        ph = lum3(Fr, Fg, Fb);
        return true;
      };
      uint32_t hidx;
      if (p.hasHistory != 0 && reproject(p, cpx, cpy, cpz, hidx)) {
        const float4 HK = hg.pos_kind[hidx];
        const float4 H3 = hr.sumwu_m_valid[hidx];
        if (__float_as_int(HK.w) == 1 && __float_as_int(H3.z) != 0) {
          const float4 HN = hg.nor_rough[hidx];
          float ddx = cpx - HK.x, ddy = cpy - HK.y, ddz = cpz - HK.z;
          float dd = sqrtf(ddx * ddx + ddy * ddy + ddz * ddz);
          float dcx = cpx - p.camera.x, dcy = cpy - p.camera.y, dcz = cpz - p.camera.z;
          float dc = sqrtf(dcx * dcx + dcy * dcy + dcz * dcz);
          const float hsumWu = H3.x;
          const uint32_t hM = uint32_t(__float_as_int(H3.y));
          const float4 H0 = hr.lp_alpha[hidx], H1 = hr.ln_phat[hidx], H2 = hr.le_sumws[hidx];
          const float hph = H1.w, hsumWs = H2.w;
          if (dd < 0.02f * dc + 1e-3f && (cnx * HN.x + (cny * HN.y + cnz * HN.z)) > 0.9f && hsumWu > 0.0f && hM > 0 &&
              hph > 0.0f) {
            float ph, dist, dxn, dyn, dzn;
            if (eval_at(H0, H1, H2, ph, dist, dxn, dyn, dzn) && ph > 0.0f) {
              float wu = ph * hsumWu / hph;
              bool occ = pt.occluded(sox, soy, soz, dxn, dyn, dzn, dist - 0.003f);
              float ws = occ ? 0.0f : ph * hsumWs / hph;
              float sum_s = cur_sumWs + ws, sum_u = cur_sumWu + wu;
              uint32_t newM = cur_M + hM; if (newM > uint32_t(mcap)) newM = uint32_t(mcap);
              float r = pt.U();
              if (sum_s > 0.0f && r * sum_s < ws) {
                cur0 = H0; cur1 = make_float4(H1.x, H1.y, H1.z, ph); cur2 = H2; cur_li = H3.w;
              }
              cur_sumWs = sum_s; cur_sumWu = sum_u; cur_M = newM;
            }
          }
        }
      }
      for (int si = 0; si < S; ++si) {
        float rx = pt.U() * 2.0f - 1.0f, ry = pt.U() * 2.0f - 1.0f;
        float fx = float(x) + rx * radius + 0.5f, fy = float(y) + ry * radius + 0.5f;
        if (!(fx > -1073741824.0f && fx < 1073741824.0f && fy > -1073741824.0f && fy < 1073741824.0f)) continue;
        int nx = int(fx), ny = int(fy);
        if (nx < 0 || ny < 0 || nx >= p.width || ny >= p.height) continue;
        if (nx == int(x) && ny == int(y)) continue;
        const uint32_t nidx = uint32_t(ny) * uint32_t(p.width) + uint32_t(nx);
        const float4 N3 = ri.sumwu_m_valid[nidx];
        if (__float_as_int(gb.pos_kind[nidx].w) != 1 || __float_as_int(N3.z) == 0) continue;
        const float4 NN = gb.nor_rough[nidx];
        if (cnx * NN.x + (cny * NN.y + cnz * NN.z) < 0.9f) continue;
        const float4 N0 = ri.lp_alpha[nidx], N1 = ri.ln_phat[nidx], N2 = ri.le_sumws[nidx];
        const float nbr_sumWu = N3.x, nbr_ph = N1.w, nbr_sumWs = N2.w;
        const uint32_t nbr_M = uint32_t(__float_as_int(N3.y));
        if (!(nbr_sumWu > 0.0f) || nbr_M == 0 || !(nbr_ph > 0.0f)) continue;
        float ph_cur, dist, dxn, dyn, dzn;
        if (!eval_at(N0, N1, N2, ph_cur, dist, dxn, dyn, dzn)) continue;
        if (!(ph_cur > 0.0f)) continue;
        float w_nbr_u = ph_cur * nbr_sumWu / nbr_ph;
        if (!(w_nbr_u > 0.0f)) continue;
        bool occ = pt.occluded(sox, soy, soz, dxn, dyn, dzn, dist - 0.003f);
        float w_nbr_s = occ ? 0.0f : ph_cur * nbr_sumWs / nbr_ph;
        float sum_s = cur_sumWs + w_nbr_s, sum_u = cur_sumWu + w_nbr_u;
        if (!(sum_u > 0.0f) || !(sum_s >= 0.0f)) continue;
        float r = pt.U();
        uint32_t newM = cur_M + nbr_M; if (newM > uint32_t(mcap)) newM = uint32_t(mcap);
        if (sum_s > 0.0f && r * sum_s < w_nbr_s) {
          cur0 = N0; cur1 = make_float4(N1.x, N1.y, N1.z, ph_cur); cur2 = N2; cur_li = N3.w;
        }
        cur_sumWs = sum_s; cur_sumWu = sum_u; cur_M = newM;
      }
      ro.lp_alpha[id] = cur0;
      ro.ln_phat[id] = cur1;
      ro.le_sumws[id] = make_float4(cur2.x, cur2.y, cur2.z, cur_sumWs);
      ro.sumwu_m_valid[id] = make_float4(cur_sumWu, __int_as_float(int(cur_M)), __int_as_float(1), cur_li);
      rays = pt.rays; nodes = pt.nodes; tests = pt.tests;
    }
  }
  __syncwarp();
  flush_counts(ctr, taken, rays, nodes, tests);
}

// K5 restir_shade (pathtrace.metal:1056-1258)
__global__ void __launch_bounds__(256) k_restir_shade(Scene s, Params p, uint64_t seed, GBufSoA gb, ResSoA rm,
                                                      float* __restrict__ hdr, uint32_t* __restrict__ dbg,
                                                      unsigned long long* ctr, uint32_t* err) {
  const uint32_t id = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t npix = uint32_t(p.width) * uint32_t(p.height);
  uint32_t taken = 0, rays = 0, nodes = 0, tests = 0;
  if (id < npix) {
    const uint32_t x = id % uint32_t(p.width), y = id / uint32_t(p.width);
    const float4 PK = gb.pos_kind[id];
    const int kind = __float_as_int(PK.w);
    float outr = 0, outg = 0, outb = 0;
    uint32_t st = 0;
    int nout = 0;
    if (kind != 0) {
      Tracer pt(s, p, err);
      pt.rng.seed(seed ^ (uint64_t(id + 1) * 0xBF58476D1CE4E5B9ull) ^ 0x94D049BB133111EBull);
      if (kind == 3) {
        float sr = 0, sg = 0, sb = 0;
        int n = 0;
        for (int si = 0; si < p.spp; ++si) {
          float sx, sy, cr, cg, cb;
          pt.jitter(x, y, sx, sy);
          pt.sample_sensor(sx, sy, p.bounces, cr, cg, cb);
          clamp3(p, cr, cg, cb);
          sr += cr; sg += cg; sb += cb;
          ++n;
        }
        float fn = float(max(n, 1));
        outr = sr / fn; outg = sg / fn; outb = sb / fn;
        clamp3(p, outr, outg, outb);
        nout = n;
      } else {
        const float4 NR = gb.nor_rough[id], AM = gb.alb_met[id], WO = gb.wo_ior[id], EM = gb.emi[id];
        const float gpx = PK.x, gpy = PK.y, gpz = PK.z, gnx = NR.x, gny = NR.y, gnz = NR.z;
        float rough = NR.w; if (rough < 0.0f) rough = 0.0f; if (rough > 1.0f) rough = 1.0f;
        float metallic = AM.w; if (metallic < 0.0f) metallic = 0.0f; if (metallic > 1.0f) metallic = 1.0f;
        float r2 = rough; if (r2 < 0.02f) r2 = 0.02f;
        float alpha2 = (r2 * r2) * (r2 * r2);
        float spec_prob = 0.05f + 0.95f * metallic; if (spec_prob > 0.98f) spec_prob = 0.98f;
        if (metallic >= 0.999f) spec_prob = 1.0f;
        const bool nomis = p.nomis;
        float pdr = 0, pdg = 0, pdb = 0;
        float m_sumWu = 0;
        uint32_t m_M = 0;
        const float4 R3 = rm.sumwu_m_valid[id];
        const float4 R0 = rm.lp_alpha[id], R1 = rm.ln_phat[id], R2 = rm.le_sumws[id];
        if (__float_as_int(R3.z) != 0 && __float_as_int(R3.y) != 0 && R3.x > 0.0f && R2.w > 0.0f && R1.w > 0.0f) {
          m_sumWu = R3.x; m_M = uint32_t(__float_as_int(R3.y));
          float m_sumWs = R2.w;
          float ldx = R0.x - gpx, ldy = R0.y - gpy, ldz = R0.z - gpz;
          float dist = sqrtf(ldx * ldx + ldy * ldy + ldz * ldz);
          if (dist > 0.003f) {
            float inv = 1.0f / dist;
            float dxn = ldx * inv, dyn = ldy * inv, dzn = ldz * inv;
            float lcos = -(R1.x * dxn + (R1.y * dyn + R1.z * dzn));
            float scos = gnx * dxn + (gny * dyn + gnz * dzn);
            if (lcos > 1e-8f && scos > 1e-8f) {
              Bsdf e = Tracer::eval_bsdf(dxn, dyn, dzn, WO.x, WO.y, WO.z, gnx, gny, gnz, alpha2, metallic, spec_prob,
                                         AM.x, AM.y, AM.z);
              float Fr = R2.x * e.r * scos * R0.w, Fg = R2.y * e.g * scos * R0.w, Fb = R2.z * e.b * scos * R0.w;
              float ph = lum3(Fr, Fg, Fb);
              if (ph > 0.0f) {
                float pdf_ris = float(m_M) * ph / m_sumWu;
                float wnee = 1.0f;
                if (!nomis && e.pdf > 1e-20f) wnee = pdf_ris / (pdf_ris + e.pdf);
                float Wt = m_sumWs / (float(m_M) * ph);
                pdr = Fr * Wt * wnee; pdg = Fg * Wt * wnee; pdb = Fb * Wt * wnee;
              }
            }
          }
        }
        const float bsr = EM.x + pdr, bsg = EM.y + pdg, bsb = EM.z + pdb;
        if (p.bounces <= 1 || p.spp <= 0) {
          outr = bsr; outg = bsg; outb = bsb;
          clamp3(p, outr, outg, outb);
        } else {
          float sr = 0, sg = 0, sb = 0;
          int n = 0;
          for (int si = 0; si < p.spp; ++si) {
            float nx2 = 0, ny2 = 0, nz2 = 0;
            int pdelta = 0;
            bool early = false;
            if (pt.U() < spec_prob) {
              float hx, hy, hz;
              pt.sample_ggx_half(alpha2, gnx, gny, gnz, hx, hy, hz);
              float md = WO.x * hx + (WO.y * hy + WO.z * hz);
              if (!(md > 1e-8f)) early = true;
              else {
                nx2 = 2.0f * md * hx - WO.x; ny2 = 2.0f * md * hy - WO.y; nz2 = 2.0f * md * hz - WO.z;
                pdelta = (rough <= 0.0201f) ? 1 : 0;
              }
            } else {
              pt.sample_cosine(gnx, gny, gnz, nx2, ny2, nz2);
              pdelta = 0;
            }
            Bsdf e0{0.f, 0.f, 0.f, 0.f};
            if (!early) {
              float ncos = nx2 * gnx + (ny2 * gny + nz2 * gnz);
              if (!(ncos > 1e-8f)) early = true;
              else {
                float d = 1.0f / sqrtf(nx2 * nx2 + ny2 * ny2 + nz2 * nz2);
                nx2 *= d; ny2 *= d; nz2 *= d;
                e0 = Tracer::eval_bsdf(nx2, ny2, nz2, WO.x, WO.y, WO.z, gnx, gny, gnz, alpha2, metallic, spec_prob,
                                       AM.x, AM.y, AM.z);
                if (!(e0.pdf > 1e-12f)) early = true;
              }
            }
            if (early) {
              float fr = bsr, fg = bsg, fb = bsb;
              clamp3(p, fr, fg, fb);
              sr += fr; sg += fg; sb += fb;
              ++n;
              continue;
            }
            float cos0 = nx2 * gnx + (ny2 * gny + nz2 * gnz);
            float thx = e0.r * cos0 / e0.pdf, thy = e0.g * cos0 / e0.pdf, thz = e0.b * cos0 / e0.pdf;
            float ox = gpx + gnx * 0.001f, oy = gpy + gny * 0.001f, oz = gpz + gnz * 0.001f;
            float dx = nx2, dy = ny2, dz = nz2;
            float last_pdf = e0.pdf;
            float pb_r = e0.r, pb_g = e0.g, pb_b = e0.b, pb_cos = cos0;
            float psumW = m_sumWu;
            uint32_t pM = m_M;
            int pdel = pdelta;
            float acx = 0, acy = 0, acz = 0;
            for (int b = 1; b < p.bounces; ++b) {
              Hit hit = pt.cast_alpha_ray(ox, oy, oz, dx, dy, dz, kFar);
              if (hit.tri < 0) break;
              float pnx = hit.nix, pny = hit.niy, pnz = hit.niz;
              float gg = hit.ngx * pnx + (hit.ngy * pny + hit.ngz * pnz);
              if (gg < 0.0f) { pnx = -pnx; pny = -pny; pnz = -pnz; }
              float nd = dx * pnx + (dy * pny + dz * pnz);
              bool front = true;
              if (nd > 0.0f) { pnx = -pnx; pny = -pny; pnz = -pnz; front = false; }
              float wox = -dx, woy = -dy, woz = -dz;
              float rh = hit.rough; if (rh < 0.0f) rh = 0.0f; if (rh > 1.0f) rh = 1.0f; if (rh < 0.02f) rh = 0.02f;
              float al = rh * rh;
              float a2 = al * al;
              const rm_triangle& lt = s.tris[hit.tri];
              float met = lt.metallic; if (met < 0.0f) met = 0.0f; if (met > 1.0f) met = 1.0f;
              if (pdel == 1) {
                acx += hit.er * thx; acy += hit.eg * thy; acz += hit.eb * thz;
              } else {
                float lx = hit.px - ox, ly = hit.py - oy, lz = hit.pz - oz;
                float d2 = lx * lx + ly * ly + lz * lz;
                float dd = sqrtf(d2);
                float pl = 1e30f;
                const float lta = lt.alpha;
                if (dd > 1e-20f && last_pdf > 1e-20f && pM > 0 && psumW > 1e-20f) {
                  float ph = lum3(hit.er * pb_r * pb_cos * lta, hit.eg * pb_g * pb_cos * lta, hit.eb * pb_b * pb_cos * lta);
                  if (ph > 1e-20f) pl = float(pM) * ph / psumW;
                  else {
                    float inv = 1.0f / dd;
                    float xn = lx * inv, yn = ly * inv, zn = lz * inv;
                    float cl = -(lt.nn.x * xn + (lt.nn.y * yn + lt.nn.z * zn));
                    if (cl > 1e-8f) {
                      float lum = lum3(lt.er, lt.eg, lt.eb); if (lum < 1e-6f) lum = 1e-6f;
                      pl = d2 * lum / (cl * p.light_total);
                    }
                  }
                } else if (dd > 1e-20f && last_pdf > 1e-20f) {
                  float inv = 1.0f / dd;
                  lx *= inv; ly *= inv; lz *= inv;
                  float cl = -(lt.nn.x * lx + (lt.nn.y * ly + lt.nn.z * lz));
                  if (cl > 1e-8f) {
                    float lum = lum3(lt.er, lt.eg, lt.eb); if (lum < 1e-6f) lum = 1e-6f;
                    pl = d2 * lum / (cl * p.light_total);
                  }
                }
                float w = nomis ? 0.0f : ((last_pdf + pl > 1e-20f) ? last_pdf / (last_pdf + pl) : 0.0f);
                acx += hit.er * thx * w; acy += hit.eg * thy * w; acz += hit.eb * thz * w;
              }
              if (hit.ior > 1.0001f) {
                float qx, qy, qz, es;
                bool valid = pt.sample_dielectric(wox, woy, woz, pnx, pny, pnz, dx, dy, dz, hit.ior, front, rh, a2, qx,
                                                  qy, qz, es);
                if (!valid) break;
                thx *= es; thy *= es; thz *= es;
                float sgn = 1.0f;
                if (qx * pnx + (qy * pny + qz * pnz) < 0.0f) sgn = -1.0f;
                ox = hit.px + pnx * 0.001f * sgn; oy = hit.py + pny * 0.001f * sgn; oz = hit.pz + pnz * 0.001f * sgn;
                dx = qx; dy = qy; dz = qz;
                pdel = 1; psumW = 0; pM = 0;
              } else {
                float sp2 = 0.05f + 0.95f * met; if (sp2 > 0.98f) sp2 = 0.98f; if (met >= 0.999f) sp2 = 1.0f;
                float dlr = 0, dlg = 0, dlb = 0, csum = 0;
                uint32_t cM = 0;
                pt.direct_lighting(hit.px, hit.py, hit.pz, pnx, pny, pnz, wox, woy, woz, rh, met, sp2, hit.ar, hit.ag,
                                   hit.ab, dlr, dlg, dlb, csum, cM);
                acx += dlr * thx; acy += dlg * thy; acz += dlb * thz;
                float qx2, qy2, qz2;
                if (pt.U() < sp2) {
                  float hx, hy, hz;
                  pt.sample_ggx_half(a2, pnx, pny, pnz, hx, hy, hz);
                  float md = wox * hx + (woy * hy + woz * hz);
                  if (!(md > 1e-8f)) break;
                  qx2 = 2.0f * md * hx - wox; qy2 = 2.0f * md * hy - woy; qz2 = 2.0f * md * hz - woz;
                  pdel = (rh <= 0.0201f) ? 1 : 0;
                } else {
                  pt.sample_cosine(pnx, pny, pnz, qx2, qy2, qz2);
                  pdel = 0;
                }
                float nc = qx2 * pnx + (qy2 * pny + qz2 * pnz);
                if (!(nc > 1e-8f)) break;
                {
                  float d = 1.0f / sqrtf(qx2 * qx2 + qy2 * qy2 + qz2 * qz2);
                  qx2 *= d; qy2 *= d; qz2 *= d;
                }
                Bsdf ee = Tracer::eval_bsdf(qx2, qy2, qz2, wox, woy, woz, pnx, pny, pnz, a2, met, sp2, hit.ar, hit.ag,
                                            hit.ab);
                if (!(ee.pdf > 1e-12f)) break;
                last_pdf = ee.pdf;
                float ci = qx2 * pnx + (qy2 * pny + qz2 * pnz);
                thx *= ee.r * ci / ee.pdf; thy *= ee.g * ci / ee.pdf; thz *= ee.b * ci / ee.pdf;
                psumW = csum; pM = cM;
                pb_r = ee.r; pb_g = ee.g; pb_b = ee.b; pb_cos = ci;
                ox = hit.px + pnx * 0.001f; oy = hit.py + pny * 0.001f; oz = hit.pz + pnz * 0.001f;
                dx = qx2; dy = qy2; dz = qz2;
              }
              float mx = fmaxf(thx, thy);
              mx = fmaxf(mx, thz);
              if (!(mx >= 1e-12f)) break;
              if (p.rr && b >= 2) {
                float rr = mx; if (rr < 0.05f) rr = 0.05f; if (rr > 0.9f) rr = 0.9f;
                if (!(pt.U() <= rr)) break;
                float ir = 1.0f / rr;
                thx *= ir; thy *= ir; thz *= ir;
              }
            }
            float fr = bsr + acx, fg = bsg + acy, fb = bsb + acz;
            clamp3(p, fr, fg, fb);
            sr += fr; sg += fg; sb += fb;
            ++n;
          }
          float fn = float(max(n, 1));
          outr = sr / fn; outg = sg / fn; outb = sb / fn;
          nout = n;
        }
      }
      st = pt.rng.state;
      rays = pt.rays; nodes = pt.nodes; tests = pt.tests;
    }
    taken = uint32_t(nout);
    hdr[size_t(id) * 3] = outr; hdr[size_t(id) * 3 + 1] = outg; hdr[size_t(id) * 3 + 2] = outb;
    if (dbg) { dbg[size_t(id) * 2] = st; dbg[size_t(id) * 2 + 1] = uint32_t(nout); }
  }
  __syncwarp();
  flush_counts(ctr, taken, rays, nodes, tests);
}

// Closest-hit / any-hit query kernel behind rmcuda_trace.
__global__ void __launch_bounds__(256) k_trace(Scene s, const float* __restrict__ rays, int n, int any_hit,
                                               int32_t* __restrict__ tri, float* t, float* u, float* v, uint32_t* err) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float* r = rays + size_t(i) * 7;
  uint32_t nodes = 0, tests = 0;
  TraceResult h = any_hit ? traverse_any<true>(s, r[0], r[1], r[2], r[3], r[4], r[5], r[6], err, nodes, tests)
                          : traverse_any<false>(s, r[0], r[1], r[2], r[3], r[4], r[5], r[6], err, nodes, tests);
  tri[i] = h.tri;
  if (t) t[i] = h.tri >= 0 ? h.t : r[6];
  if (u) u[i] = h.u;
  if (v) v[i] = h.v;
}

// ---------------------------------------------------------------- launchers

static inline unsigned blocks_for(uint64_t threads, unsigned tpb) { return unsigned((threads + tpb - 1) / tpb); }

cudaError_t launch_render_paths(int lanes, const Scene& s, const Params& p, uint64_t seed, float* hdr, uint8_t* rgb,
                                uint32_t* dbg, unsigned long long* ctr, uint32_t* err, cudaStream_t st) {
  const uint64_t threads = uint64_t(p.width) * uint64_t(p.height) * uint64_t(lanes);
  const unsigned g = blocks_for(threads, 256);
  if (lanes == 32) k_render_paths<32><<<g, 256, 0, st>>>(s, p, seed, hdr, rgb, dbg, ctr, err);
  else if (lanes == 8) k_render_paths<8><<<g, 256, 0, st>>>(s, p, seed, hdr, rgb, dbg, ctr, err);
  else k_render_paths<1><<<g, 256, 0, st>>>(s, p, seed, hdr, rgb, dbg, ctr, err);
  return cudaGetLastError();
}

cudaError_t launch_restir_stage(int stage, const Scene& s, const Params& p, uint64_t seed, const GBufSoA& gb,
                                const ResSoA& ri, const ResSoA& rm, const GBufSoA& hg, const ResSoA& hr, float* hdr,
                                uint32_t* dbg, unsigned long long* ctr, uint32_t* err, cudaStream_t st) {
  const uint64_t npix = uint64_t(p.width) * uint64_t(p.height);
  const unsigned g = blocks_for(npix, 256);
  if (stage == 0) k_restir_generate<<<blocks_for(npix, 128), 128, 0, st>>>(s, p, seed, gb, ri, ctr, err);
  else if (stage == 1) k_restir_spatial<<<g, 256, 0, st>>>(s, p, seed, gb, ri, rm, hg, hr, ctr, err);
  else k_restir_shade<<<g, 256, 0, st>>>(s, p, seed, gb, rm, hdr, dbg, ctr, err);
  return cudaGetLastError();
}

cudaError_t launch_trace(const Scene& s, const float* rays, int n, int any_hit, int32_t* tri, float* t, float* u,
                         float* v, uint32_t* err, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  k_trace<<<blocks_for(uint64_t(n), 256), 256, 0, st>>>(s, rays, n, any_hit, tri, t, u, v, err);
  return cudaGetLastError();
}

}  // namespace rmd
