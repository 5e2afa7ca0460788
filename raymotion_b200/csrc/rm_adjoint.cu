// rm_adjoint.cu - path-replay adjoint of the plain single-frame chain:
// gradients of an image loss with respect to per-material albedo, roughness,
// emission and index of refraction.
//
// The differentiated estimator is the frame of render_paths (K1) or the lane
// kernel (K2) (pathtrace.metal:739-815) with its sampling held fixed: every
// random decision, sampled direction, pdf, MIS weight, light-sample
// resampling weight (RIS NEE) and Russian-roulette probability keeps its
// value at the current parameters, and only the
// factors of the path integrand that depend on the materials are
// differentiated - the opaque BSDF value (albedo, roughness), the emission of
// hit and sampled lights, and for a dielectric the Fresnel and (eta_i/eta_t)^2
// factors (index of refraction) and the microfacet D and G terms (roughness),
// each as a ratio to its value at the current parameters (path replay
// backpropagation with detached sampling, Vicini, Speierer and Jakob,
// SIGGRAPH 2021).  With the sample's radiance C and the radiance S_k that the
// path gathers after vertex k, the derivative of a sample is
//     sum_k thr_k * d(E_k + N_k) + sum_k (dB_k / B_k) * S_k
// (E_k emission at vertex k, N_k its light sample, B_k the throughput factor
// of its scattering).  Each thread owns a pixel lane, as the forward kernels
// do, and replays each of its samples from the sample's RNG state, in one
// walk: the terms independent of C at once, the C-proportional halves of
// g . dlogB_k . (C - acc_k) kept per vertex until the path ends (see
// adjoint_path); paths longer than the kept list walk twice (first for C).
// The refracted direction
// is held fixed when the index of refraction changes; its motion would need a
// reparameterised sampler and is not part of the estimator.
#include <cuda_runtime.h>

#include "rm_device.cuh"
#include "rm_launch.h"

namespace rmd {

namespace {

constexpr int kMatParams = 8;  // albedo rgb, rough, emission rgb, ior

struct GradSink {
  float* sh;  // per-block accumulators, or null
  float* gl;  // the caller's gradient
  __device__ __forceinline__ void add(int m, int k, float v) const {
    if (m < 0 || v == 0.0f) return;
    atomicAdd((sh ? sh : gl) + m * kMatParams + k, v);
  }
};

struct Dual {
  float v, d;
};
__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return Dual{a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return Dual{a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return Dual{a.v * b.v, a.d * b.v + a.v * b.d}; }
__device__ __forceinline__ Dual operator/(Dual a, Dual b) {
  return Dual{a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v)};
}
__device__ __forceinline__ Dual dsqrt(Dual a) {
  const float r = sqrtf(a.v);
  return Dual{r, r > 0.0f ? a.d / (2.0f * r) : 0.0f};
}
__device__ __forceinline__ Dual dc(float v) { return Dual{v, 0.0f}; }

// Fresnel (pathtrace.metal:80-91) and its derivative along the dual parts of
// the two indices.
__device__ Dual fresnel_dual(float ci, Dual eta_in, Dual eta_out) {
  if (ci < 0.0f) ci = 0.0f;
  if (ci > 1.0f) ci = 1.0f;
  const Dual eta = eta_in / eta_out;
  const Dual s2 = eta * eta * dc(1.0f - ci * ci);
  if (s2.v >= 1.0f) return dc(1.0f);
  const Dual ct = dsqrt(dc(1.0f) - s2);
  const Dual c = dc(ci);
  const Dual rp = (eta_out * c - eta_in * ct) / (eta_out * c + eta_in * ct);
  const Dual rs = (eta_in * c - eta_out * ct) / (eta_in * c + eta_out * ct);
  return dc(0.5f) * (rp * rp + rs * rs);
}

// |h x n|^2: the squared sine between two unit vectors, accurate near 0.
__device__ __forceinline__ float sin2(float hx, float hy, float hz, float nx, float ny, float nz) {
  const float cx = hy * nz - hz * ny, cy = hz * nx - hx * nz, cz = hx * ny - hy * nx;
  return cx * cx + cy * cy + cz * cz;
}

// d/dalpha2 of log G1 for one direction (Smith G1 of pathtrace.metal:270-276).
__device__ __forceinline__ float dlog_g1(float c, float alpha2) {
  const float sq = sqrtf(c * c + alpha2 * (1.0f - c * c));
  return -(1.0f - c * c) / (2.0f * sq * (c + sq));
}

// The opaque BSDF value (pathtrace.metal:243-295) with its derivatives with
// respect to each albedo channel and alpha2.
struct BsdfGrad {
  float f[3], da[3], dal2[3];
};

__device__ BsdfGrad bsdf_grad(float wix, float wiy, float wiz, float wox, float woy, float woz, float nx, float ny,
                              float nz, float alpha2, float metallic, float ar, float ag, float ab) {
  BsdfGrad out;
#pragma unroll
  for (int c = 0; c < 3; ++c) out.f[c] = out.da[c] = out.dal2[c] = 0.0f;
  const float cos_i = wix * nx + (wiy * ny + wiz * nz);
  const float cos_o = wox * nx + (woy * ny + woz * nz);
  if (!(cos_i > 1e-8f && cos_o > 1e-8f)) return out;
  float hx = wix + wox, hy = wiy + woy, hz = wiz + woz;
  const float hl = sqrtf(hx * hx + hy * hy + hz * hz);
  if (!(hl > 1e-8f)) return out;
  const float inv = 1.0f / hl;
  hx *= inv; hy *= inv; hz *= inv;
  float cos_h = hx * nx + (hy * ny + hz * nz);
  float vo_h = wox * hx + (woy * hy + woz * hz);
  if (cos_h < 0.0f) { cos_h = -cos_h; vo_h = -vo_h; }
  if (!(vo_h > 1e-8f)) return out;
  // cos_h^2 (alpha2 - 1) + 1 = |h x n|^2 + alpha2 cos_h^2, without the
  // cancellation near the lobe's peak (alpha2 can be 6e-6)
  const float dd = sin2(hx, hy, hz, nx, ny, nz) + alpha2 * cos_h * cos_h;
  const float D = alpha2 / (kPi * dd * dd);
  const float g1 = 2.0f * cos_o / (cos_o + sqrtf(cos_o * cos_o + alpha2 * (1.0f - cos_o * cos_o)));
  const float g2 = 2.0f * cos_i / (cos_i + sqrtf(cos_i * cos_i + alpha2 * (1.0f - cos_i * cos_i)));
  const float G = g1 * g2;
  float om = 1.0f - vo_h;
  om *= om; om *= om; om *= 1.0f - vo_h;
  const float di = 1.0f - metallic;
  const float base = D * G / (4.0f * cos_i * cos_o);
  const float dlog = 1.0f / alpha2 - 2.0f * cos_h * cos_h / dd + dlog_g1(cos_o, alpha2) + dlog_g1(cos_i, alpha2);
  const float alb[3] = {ar, ag, ab};
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const float f0 = 0.04f * di + alb[c] * metallic;
    const float F = f0 + (1.0f - f0) * om;
    out.f[c] = alb[c] * di * (1.0f - F) / kPi + base * F;
    out.da[c] = (di * (1.0f - F) - alb[c] * di * metallic * (1.0f - om)) / kPi + base * metallic * (1.0f - om);
    out.dal2[c] = base * dlog * F;
  }
  return out;
}

// d alpha2 / d rough for alpha2 = r^4, r = max(clamp(rough, 0, 1), 0.02).
__device__ __forceinline__ float dalpha2(float rough) {
  if (!(rough > 0.02f && rough < 1.0f)) return 0.0f;
  return 4.0f * rough * rough * rough;
}

// The terms of a sample's derivative that multiply its radiance C, one per
// scattering vertex, kept until C is known (single-pass adjoint).
struct Deferred {
  static constexpr int kMax = 24;
  int n;
  int m[kMax];
  int kind[kMax];    // 0 opaque surface, 1 dielectric
  float v[kMax][6];  // opaque: albedo r, g, b; rough per channel.  dielectric: ior, rough
};

// One sample's path again (pathtrace.metal:552-728, the same arithmetic and
// random draws as Tracer::pathtrace), accumulating g . dC/dparams.  With
// `dfr` null the sample's radiance C is given (a second walk after one that
// computed it); with `dfr` the walk computes C itself, adds at once every
// term that does not depend on it - the emission and light-sample terms and
// the -(g . acc) halves of the scattering terms g . dlogB_k . (C - acc_k) -
// and the g . dlogB_k . C halves when the path ends, returning C in C_out.
// kRis: the frame's NEE takes several candidates (RIS); a separate
// instantiation keeps the single-candidate walk's registers as they were.
// `from` (null: a camera ray) continues a path from a vertex already shaded
// (the ReSTIR shade's primary vertex, pathtrace.metal:1135-1255): its
// throughput, the BSDF sample that left it and its light-sample sums, so that
// the first vertex's emission takes its MIS weight.
struct WalkFrom {
  float thr[3], last_pdf, prev_b[3], prev_cos, prev_sumW;
  uint32_t prev_M;
  int prev_delta;
};

template <bool kRis>
__device__ __noinline__ void adjoint_path(Tracer& pt, const int32_t* __restrict__ tri_mat, float ox, float oy,
                                          float oz, float dx, float dy, float dz, int max_bounces, float Cr, float Cg,
                                          float Cb, float gr, float gg, float gb, const GradSink& sink,
                                          Deferred* dfr, float* C_out, const WalkFrom* from = nullptr) {
  if (dfr) dfr->n = 0;
  const Scene& s = pt.s;
  const Params& p = pt.p;
  float accr = 0, accg = 0, accb = 0, thr_r = 1, thr_g = 1, thr_b = 1;
  int bounce = 0, prev_delta = 1;
  float last_pdf = 0, prev_sumW = 0;
  uint32_t prev_M = 0;
  float prev_br = 0, prev_bg = 0, prev_bb = 0, prev_cos = 0;
  const bool camera = from == nullptr;
  if (from) {
    thr_r = from->thr[0]; thr_g = from->thr[1]; thr_b = from->thr[2];
    last_pdf = from->last_pdf;
    prev_br = from->prev_b[0]; prev_bg = from->prev_b[1]; prev_bb = from->prev_b[2]; prev_cos = from->prev_cos;
    prev_sumW = from->prev_sumW; prev_M = from->prev_M; prev_delta = from->prev_delta;
  }
  const float LT = p.light_total;
  for (int b = 0; b < max_bounces; ++b) {
    Hit hit = pt.cast_alpha_ray(ox, oy, oz, dx, dy, dz, kFar);
    if (hit.tri < 0) break;
    const int m = tri_mat[hit.tri];
    float pnx = hit.nix, pny = hit.niy, pnz = hit.niz;
    float geom = hit.ngx * pnx + (hit.ngy * pny + hit.ngz * pnz);
    if (geom < 0.0f) { pnx = -pnx; pny = -pny; pnz = -pnz; }
    float ndot = dx * pnx + (dy * pny + dz * pnz);
    bool front = true;
    if (ndot > 0.0f) { pnx = -pnx; pny = -pny; pnz = -pnz; front = false; }
    float wox = -dx, woy = -dy, woz = -dz;
    float rough = hit.rough;
    if (rough < 0.0f) rough = 0.0f;
    if (rough > 1.0f) rough = 1.0f;
    if (rough < 0.02f) rough = 0.02f;
    float alpha = rough * rough;
    float alpha2 = alpha * alpha;
    const float dal2 = dalpha2(hit.rough);
    const rm_triangle& lt = s.tris[hit.tri];
    float metallic = lt.metallic;
    if (metallic < 0.0f) metallic = 0.0f;
    if (metallic > 1.0f) metallic = 1.0f;
    float we = 1.0f;  // MIS weight of the emission term (held fixed)
    if ((camera && bounce == 0) || prev_delta == 1) {
      accr += hit.er * thr_r; accg += hit.eg * thr_g; accb += hit.eb * thr_b;
    } else {
      float lx = hit.px - ox, ly = hit.py - oy, lz = hit.pz - oz;
      float dist2 = lx * lx + ly * ly + lz * lz;
      float dist = sqrtf(dist2);
      float pl = 1e30f;
      float lta = lt.alpha;
      if (dist > 1e-20f && last_pdf > 1e-20f && prev_M > 0 && prev_sumW > 1e-20f) {
        float ph = lum3(hit.er * prev_br * prev_cos * lta, hit.eg * prev_bg * prev_cos * lta,
                        hit.eb * prev_bb * prev_cos * lta);
        if (ph > 1e-20f) pl = float(prev_M) * ph / prev_sumW;
        else {
          float inv = 1.0f / dist;
          float lxn = lx * inv, lyn = ly * inv, lzn = lz * inv;
          float cos_l = -(lt.nn.x * lxn + (lt.nn.y * lyn + lt.nn.z * lzn));
          if (cos_l > 1e-8f) {
            float lum = lum3(lt.er, lt.eg, lt.eb);
            if (lum < 1e-6f) lum = 1e-6f;
            pl = dist2 * lum / (cos_l * LT);
          }
        }
      } else if (dist > 1e-20f && last_pdf > 1e-20f) {
        float inv = 1.0f / dist;
        lx *= inv; ly *= inv; lz *= inv;
        float cos_l = -(lt.nn.x * lx + (lt.nn.y * ly + lt.nn.z * lz));
        if (cos_l > 1e-8f) {
          float lum = lum3(lt.er, lt.eg, lt.eb);
          if (lum < 1e-6f) lum = 1e-6f;
          pl = dist2 * lum / (cos_l * LT);
        }
      }
      we = p.nomis ? 0.0f : ((last_pdf + pl > 1e-20f) ? last_pdf / (last_pdf + pl) : 0.0f);
      accr += hit.er * thr_r * we; accg += hit.eg * thr_g * we; accb += hit.eb * thr_b * we;
    }
    sink.add(m, 4, gr * thr_r * we);
    sink.add(m, 5, gg * thr_g * we);
    sink.add(m, 6, gb * thr_b * we);
    if (hit.ior > 1.0001f) {
      float nx2, ny2, nz2, es;
      float dp[7];
      bool valid = pt.sample_dielectric(wox, woy, woz, pnx, pny, pnz, dx, dy, dz, hit.ior, front, rough, alpha2, nx2,
                                        ny2, nz2, es, dp);
      if (!valid) break;
      // B_k = es: d log B_k (ior, rough), times g . S_k
      float dlog_ior = 0.0f, dlog_r = 0.0f;
      const int event = int(dp[0]);
      if (event != 2) {
        const Dual ior{hit.ior, 1.0f};
        const Dual ei = front ? dc(1.0f) : ior, et = front ? ior : dc(1.0f);
        const Dual F = fresnel_dual(dp[1], ei, et);
        if (event == 0) dlog_ior = F.v > 0.0f ? F.d / F.v : 0.0f;
        else {
          dlog_ior = F.v < 1.0f ? -F.d / (1.0f - F.v) : 0.0f;
          dlog_ior += front ? -2.0f / hit.ior : 2.0f / hit.ior;  // (eta_i / eta_t)^2
        }
      }
      if (rough > 0.0201f && dal2 != 0.0f) {
        const float ch = dp[4];
        const float dd = dp[6] + alpha2 * ch * ch;
        dlog_r = 1.0f / alpha2 - 2.0f * ch * ch / dd;  // D
        if (dp[5] == 0.0f) dlog_r += dlog_g1(dp[3], alpha2) + dlog_g1(dp[2], alpha2);  // G, unless clamped
        dlog_r *= dal2;
      }
      if (dfr) {
        const float gA = gr * accr + gg * accg + gb * accb;
        sink.add(m, 7, -gA * dlog_ior);
        sink.add(m, 3, -gA * dlog_r);
        const int k = dfr->n++;
        dfr->m[k] = m; dfr->kind[k] = 1; dfr->v[k][0] = dlog_ior; dfr->v[k][1] = dlog_r;
      } else {
        const float gS = gr * (Cr - accr) + gg * (Cg - accg) + gb * (Cb - accb);
        sink.add(m, 7, gS * dlog_ior);
        sink.add(m, 3, gS * dlog_r);
      }
      thr_r *= es; thr_g *= es; thr_b *= es;
      float sg = 1.0f;
      if (nx2 * pnx + (ny2 * pny + nz2 * pnz) < 0.0f) sg = -1.0f;
      ox = hit.px + pnx * 0.001f * sg;
      oy = hit.py + pny * 0.001f * sg;
      oz = hit.pz + pnz * 0.001f * sg;
      dx = nx2; dy = ny2; dz = nz2;
      prev_delta = 1;
      prev_sumW = 0; prev_M = 0;
    } else {
      float spec_prob = 0.05f + 0.95f * metallic;
      if (spec_prob > 0.98f) spec_prob = 0.98f;
      if (metallic >= 0.999f) spec_prob = 1.0f;
      const bool alb_grad = hit.shader != 1;
      const float tx[3] = {hit.txr, hit.txg, hit.txb};
      const float gv[3] = {gr, gg, gb};
      float cur_sumW = 0;
      uint32_t cur_M = 0;
      {
        float dlr, dlg, dlb, sdist, sox, soy, soz, sdx, sdy, sdz;
        bool has_ray;
        float parts[2];
        // single-candidate NEE (pathtrace.metal:319-384) or RIS over the
        // candidates (:385-469), with the same draws; the selection, its
        // resampling weight W and the MIS weight are held, so the light sample
        // N_k = Le f k moves only with the light's emission and this BSDF
        if (kRis)
          pt.direct_lighting_deferred(hit.px, hit.py, hit.pz, pnx, pny, pnz, wox, woy, woz, rough, metallic,
                                      spec_prob, hit.ar, hit.ag, hit.ab, dlr, dlg, dlb, cur_sumW, cur_M, has_ray, sox,
                                      soy, soz, sdx, sdy, sdz, sdist, parts);
        else
          pt.nee_single_deferred(hit.px, hit.py, hit.pz, pnx, pny, pnz, wox, woy, woz, rough, metallic, spec_prob,
                                 hit.ar, hit.ag, hit.ab, dlr, dlg, dlb, cur_sumW, cur_M, has_ray, sox, soy, soz, sdx,
                                 sdy, sdz, sdist, parts);
        if (has_ray && !pt.occluded(sox, soy, soz, sdx, sdy, sdz, sdist)) {
          accr += dlr * thr_r; accg += dlg * thr_g; accb += dlb * thr_b;
          // N_k = Le * f * k: derivative in the light's emission and this surface's BSDF
          const int li = __float_as_int(parts[0]);
          const float k = parts[1];
          const LightRec L = load_light(s, li);
          const int ml = tri_mat[s.lights[li]];
          const BsdfGrad bg = bsdf_grad(sdx, sdy, sdz, wox, woy, woz, pnx, pny, pnz, alpha2, metallic, hit.ar, hit.ag,
                                        hit.ab);
          const float thr[3] = {thr_r, thr_g, thr_b};
          const float le[3] = {L.er, L.eg, L.eb};
          float drough = 0.0f;
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const float gt = gv[c] * thr[c] * k;
            sink.add(ml, 4 + c, gt * bg.f[c]);
            if (alb_grad) sink.add(m, c, gt * le[c] * bg.da[c] * tx[c]);
            drough += gt * le[c] * bg.dal2[c];
          }
          sink.add(m, 3, drough * dal2);
        }
      }
      float nx2, ny2, nz2;
      if (pt.U() < spec_prob) {
        float hx, hy, hz;
        pt.sample_ggx_half(alpha2, pnx, pny, pnz, hx, hy, hz);
        float md = wox * hx + (woy * hy + woz * hz);
        if (!(md > 1e-8f)) break;
        nx2 = 2.0f * md * hx - wox;
        ny2 = 2.0f * md * hy - woy;
        nz2 = 2.0f * md * hz - woz;
        prev_delta = (rough <= 0.0201f) ? 1 : 0;
      } else {
        pt.sample_cosine(pnx, pny, pnz, nx2, ny2, nz2);
        prev_delta = 0;
      }
      float ncos = nx2 * pnx + (ny2 * pny + nz2 * pnz);
      if (!(ncos > 1e-8f)) break;
      {
        float d = 1.0f / sqrtf(nx2 * nx2 + ny2 * ny2 + nz2 * nz2);
        nx2 *= d; ny2 *= d; nz2 *= d;
      }
      Bsdf e = Tracer::eval_bsdf(nx2, ny2, nz2, wox, woy, woz, pnx, pny, pnz, alpha2, metallic, spec_prob, hit.ar,
                                 hit.ag, hit.ab);
      if (!(e.pdf > 1e-12f)) break;
      {
        // B_k = f * cos / pdf: d log B_k = df / f, times g . S_k per channel
        const BsdfGrad bg = bsdf_grad(nx2, ny2, nz2, wox, woy, woz, pnx, pny, pnz, alpha2, metallic, hit.ar, hit.ag,
                                      hit.ab);
        float qa[3], qr[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const bool ok = bg.f[c] > 0.0f;
          qa[c] = (ok && alb_grad) ? gv[c] * bg.da[c] * tx[c] / bg.f[c] : 0.0f;
          qr[c] = ok ? gv[c] * bg.dal2[c] * dal2 / bg.f[c] : 0.0f;
        }
        const float acc[3] = {accr, accg, accb};
        const float S[3] = {Cr - accr, Cg - accg, Cb - accb};
        float drough = 0.0f;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const float w = dfr ? -acc[c] : S[c];
          if (alb_grad) sink.add(m, c, qa[c] * w);
          drough += qr[c] * w;
        }
        sink.add(m, 3, drough);
        if (dfr) {
          const int k = dfr->n++;
          dfr->m[k] = m; dfr->kind[k] = 0;
#pragma unroll
          for (int c = 0; c < 3; ++c) { dfr->v[k][c] = qa[c]; dfr->v[k][3 + c] = qr[c]; }
        }
      }
      last_pdf = e.pdf;
      float cos_i = nx2 * pnx + (ny2 * pny + nz2 * pnz);
      thr_r *= e.r * cos_i / e.pdf;
      thr_g *= e.g * cos_i / e.pdf;
      thr_b *= e.b * cos_i / e.pdf;
      prev_sumW = cur_sumW; prev_M = cur_M;
      prev_br = e.r; prev_bg = e.g; prev_bb = e.b; prev_cos = cos_i;
      ox = hit.px + pnx * 0.001f;
      oy = hit.py + pny * 0.001f;
      oz = hit.pz + pnz * 0.001f;
      dx = nx2; dy = ny2; dz = nz2;
    }
    if (thr_r < 0.0f) thr_r = 0.0f;
    if (thr_g < 0.0f) thr_g = 0.0f;
    if (thr_b < 0.0f) thr_b = 0.0f;
    float mx = fmaxf(thr_r, thr_g);
    mx = fmaxf(mx, thr_b);
    if (!(mx >= 1e-12f)) break;
    if (p.rr && bounce >= 1) {
      float rr = mx;
      if (rr < 0.05f) rr = 0.05f;
      if (rr > 0.9f) rr = 0.9f;
      if (!(pt.U() <= rr)) break;
      float ir = 1.0f / rr;
      thr_r *= ir; thr_g *= ir; thr_b *= ir;
    }
    bounce++;
  }
  if (dfr) {
    // the path is complete: acc is its radiance C
    const float C[3] = {accr, accg, accb};
    const float gC = gr * accr + gg * accg + gb * accb;
    for (int k = 0; k < dfr->n; ++k) {
      const int m = dfr->m[k];
      if (dfr->kind[k] == 0) {
        float dr = 0.0f;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          sink.add(m, c, dfr->v[k][c] * C[c]);
          dr += dfr->v[k][3 + c] * C[c];
        }
        sink.add(m, 3, dr);
      } else {
        sink.add(m, 7, dfr->v[k][0] * gC);
        sink.add(m, 3, dfr->v[k][1] * gC);
      }
    }
    C_out[0] = accr; C_out[1] = accg; C_out[2] = accb;
  }
}

// One sample of a camera path (pathtrace.metal:749-758, the samples of K1, K2
// and of K5's kind-3 pixels :1070-1084): the jitter draws, then the path's
// adjoint for the loss gradient (d0, d1, d2) of the sample's clamped value.
// One walk when the path's vertices fit the deferred list, else a first walk
// for C (Tracer::sample_sensor) and a second for the derivative.
template <bool kRis>
__device__ __forceinline__ void camera_sample_adjoint(Tracer& pt, const int32_t* __restrict__ tri_mat, uint32_t x,
                                                      uint32_t y, float d0, float d1, float d2,
                                                      const GradSink& sink) {
  const Params& p = pt.p;
  const bool one_walk = p.bounces <= Deferred::kMax;
  const bool cl = p.clamp_value > 0.0f;
  float sx, sy;
  pt.jitter(x, y, sx, sy);
  const uint32_t st0 = pt.rng.state;
  const rm_camera& cam = p.camera;
  const float focal2 = cam.focal * cam.focal;
  const float dist = 1.0f / sqrtf(sx * sx + (sy * sy + focal2));
  const float tx = sx * dist, ty = sy * dist, tz = cam.focal * dist;
  const float dx = tx * cam.m0 + (ty * cam.m1 + tz * cam.m2);
  const float dy = tx * cam.m3 + (ty * cam.m4 + tz * cam.m5);
  const float dz = tx * cam.m6 + (ty * cam.m7 + tz * cam.m8);
  float C[3];
  if (one_walk) {
    // derivative as if no channel were clamped; a clamped channel (rare)
    // is taken back out by a second walk with -g on that channel
    Deferred dfr;
    adjoint_path<kRis>(pt, tri_mat, cam.x, cam.y, cam.z, dx, dy, dz, p.bounces, 0.f, 0.f, 0.f, d0, d1, d2, sink, &dfr,
                 C);
    if (cl && !(C[0] < p.clamp_value && C[1] < p.clamp_value && C[2] < p.clamp_value)) {
      const uint32_t st1 = pt.rng.state;
      pt.rng.state = st0;
      adjoint_path<kRis>(pt, tri_mat, cam.x, cam.y, cam.z, dx, dy, dz, p.bounces, C[0], C[1], C[2],
                   C[0] < p.clamp_value ? 0.f : -d0, C[1] < p.clamp_value ? 0.f : -d1,
                   C[2] < p.clamp_value ? 0.f : -d2, sink, nullptr, nullptr);
      pt.rng.state = st1;
    }
  } else {
    pt.sample_sensor(sx, sy, p.bounces, C[0], C[1], C[2]);
    pt.rng.state = st0;
    // the sample enters the pixel mean clamped (pathtrace.metal:757)
    const float gr = (cl && !(C[0] < p.clamp_value)) ? 0.0f : d0;
    const float gg = (cl && !(C[1] < p.clamp_value)) ? 0.0f : d1;
    const float gb = (cl && !(C[2] < p.clamp_value)) ? 0.0f : d2;
    adjoint_path<kRis>(pt, tri_mat, cam.x, cam.y, cam.z, dx, dy, dz, p.bounces, C[0], C[1], C[2], gr, gg, gb, sink,
                 nullptr, nullptr);
  }
}

// One pixel lane per thread, the samples of K1 (LANES 1) or of one lane of K2,
// in the forward kernels' order (pathtrace.metal:749-758, :787-796).
template <int LANES, bool kRis>
__global__ void __launch_bounds__(256) k_adjoint(Scene s, Params p, uint64_t seed, const int32_t* __restrict__ tri_mat,
                                                 int n_mat, const float* __restrict__ dLdI, float* __restrict__ grad,
                                                 int use_shared, unsigned long long* ctr, uint32_t* err) {
  extern __shared__ float sh[];
  if (use_shared) {
    for (int i = threadIdx.x; i < n_mat * kMatParams; i += blockDim.x) sh[i] = 0.0f;
    __syncthreads();
  }
  const GradSink sink{use_shared ? sh : nullptr, grad};
  const uint64_t gid = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const uint32_t npix = uint32_t(p.width) * uint32_t(p.height);
  const uint32_t pixel = uint32_t(gid / LANES), lane = uint32_t(gid % LANES);
  uint32_t samples = 0;
  if (pixel < npix) {
    const uint32_t x = pixel % uint32_t(p.width), y = pixel / uint32_t(p.width);
    Tracer pt(s, p, err);
    uint64_t sd = seed_pixel(seed, x, y);
    if (LANES > 1) sd ^= uint64_t(lane) * 0x94D049BB133111EBull;
    pt.rng.seed(sd);
    const float inv_n = 1.0f / float(p.spp);
    const float d0 = dLdI[size_t(pixel) * 3] * inv_n, d1 = dLdI[size_t(pixel) * 3 + 1] * inv_n,
                d2 = dLdI[size_t(pixel) * 3 + 2] * inv_n;
    for (uint32_t si = lane; si < uint32_t(p.spp); si += LANES) {
      camera_sample_adjoint<kRis>(pt, tri_mat, x, y, d0, d1, d2, sink);
      ++samples;
    }
  }
  const unsigned long long tot = __reduce_add_sync(0xffffffffu, samples);
  if ((threadIdx.x & 31) == 0 && tot) atomicAdd(ctr, tot);
  if (use_shared) {
    __syncthreads();
    for (int i = threadIdx.x; i < n_mat * kMatParams; i += blockDim.x)
      if (sh[i] != 0.0f) atomicAdd(grad + i, sh[i]);
  }
}

// The adjoint of K5, the ReSTIR shade (pathtrace.metal:1056-1258), from the
// frame's checkpoint: its G-buffer and merged reservoirs (the light sample
// each kind-1 pixel shades, with its light index) stay as the forward pass
// left them, and the pixel's K5 draws are replayed.  Kind-3 pixels (a
// dielectric first hit) are camera paths, as in K1.  A kind-1 pixel's value
// is the mean over samples of clamp(base + C_s): base = the first hit's
// emission + the reservoir sample's Le f cos alpha W w_MIS (sample, W and MIS
// weight held), C_s an indirect path that leaves the first hit with the BSDF
// sample B_0 = f cos / pdf and goes on as a camera path's vertices do
// (adjoint_path from the first hit; Russian roulette from its second vertex).
// d(base) moves with the first hit's emission, albedo and roughness and the
// sampled light's emission; C_s with its vertices (the walk) and with B_0
// (dlog B_0 * C_s).  The first hit's material is found by tracing K3's
// primary ray again (pathtrace.metal:829-840).
template <bool kRis>
__global__ void __launch_bounds__(256) k_adjoint_restir(Scene s, Params p, uint64_t seed, GBufSoA gb, ResSoA rm,
                                                        const int32_t* __restrict__ tri_mat, int n_mat,
                                                        const float* __restrict__ dLdI,
                                                        const float* __restrict__ dLdalb, float* __restrict__ grad,
                                                        int use_shared, unsigned long long* ctr, uint32_t* err) {
  extern __shared__ float sh[];
  if (use_shared) {
    for (int i = threadIdx.x; i < n_mat * kMatParams; i += blockDim.x) sh[i] = 0.0f;
    __syncthreads();
  }
  const GradSink sink{use_shared ? sh : nullptr, grad};
  const uint32_t id = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t npix = uint32_t(p.width) * uint32_t(p.height);
  uint32_t samples = 0;
  const float4 PK = id < npix ? gb.pos_kind[id] : make_float4(0.f, 0.f, 0.f, 0.f);
  const int kind = __float_as_int(PK.w);
  if (id < npix && kind != 0) {
    const uint32_t x = id % uint32_t(p.width), y = id / uint32_t(p.width);
    Tracer pt(s, p, err);
    pt.rng.seed(seed ^ (uint64_t(id + 1) * 0xBF58476D1CE4E5B9ull) ^ 0x94D049BB133111EBull);
    const bool cl = p.clamp_value > 0.0f;
    const float D[3] = {dLdI[size_t(id) * 3], dLdI[size_t(id) * 3 + 1], dLdI[size_t(id) * 3 + 2]};
    // the first hit's triangle: K3's primary ray (its own random stream)
    int m0 = -1;
    float tx0[3] = {1.f, 1.f, 1.f};
    bool alb0 = false;
    float dal0 = 0.0f;
    if (kind == 1 || dLdalb) {
      Tracer p3(s, p, err);
      p3.rng.seed(seed_pixel(seed, x, y));
      float sx = float(x) + 1e-12f + (p.resolution - 2e-12f) * p3.U() - float(p.width) * 0.5f;
      float sy = float(p.height) * 0.5f - (float(y) + 1e-12f + (p.resolution - 2e-12f) * p3.U());
      const rm_camera& c = p.camera;
      float f2 = c.focal * c.focal;
      float dinv = 1.0f / sqrtf(sx * sx + sy * sy + f2);
      float tx = sx * dinv, ty = sy * dinv, tz = c.focal * dinv;
      float rdx = tx * c.m0 + (ty * c.m1 + tz * c.m2);
      float rdy = tx * c.m3 + (ty * c.m4 + tz * c.m5);
      float rdz = tx * c.m6 + (ty * c.m7 + tz * c.m8);
      const Hit h0 = p3.cast_alpha_ray(c.x, c.y, c.z, rdx, rdy, rdz, kFar);
      if (h0.tri >= 0) {
        m0 = tri_mat[h0.tri];
        tx0[0] = h0.txr; tx0[1] = h0.txg; tx0[2] = h0.txb;
        alb0 = h0.shader != 1;
        dal0 = dalpha2(h0.rough);
      }
    }
    // the denoiser's weights through this pixel's G-buffer albedo (the first
    // hit's albedo times its texel)
    if (dLdalb && alb0)
      for (int k = 0; k < 3; ++k) sink.add(m0, k, dLdalb[size_t(id) * 3 + k] * tx0[k]);
    if (kind == 3) {
      const float inv_n = 1.0f / float(p.spp);
      for (int si = 0; si < p.spp; ++si) {
        camera_sample_adjoint<kRis>(pt, tri_mat, x, y, D[0] * inv_n, D[1] * inv_n, D[2] * inv_n, sink);
        ++samples;
      }
    } else {
      const float4 NR = gb.nor_rough[id], AM = gb.alb_met[id], WO = gb.wo_ior[id], EM = gb.emi[id];
      const float gpx = PK.x, gpy = PK.y, gpz = PK.z, gnx = NR.x, gny = NR.y, gnz = NR.z;
      float rough = NR.w; if (rough < 0.0f) rough = 0.0f; if (rough > 1.0f) rough = 1.0f;
      float metallic = AM.w; if (metallic < 0.0f) metallic = 0.0f; if (metallic > 1.0f) metallic = 1.0f;
      float r2 = rough; if (r2 < 0.02f) r2 = 0.02f;
      const float alpha2 = (r2 * r2) * (r2 * r2);
      float spec_prob = 0.05f + 0.95f * metallic; if (spec_prob > 0.98f) spec_prob = 0.98f;
      if (metallic >= 0.999f) spec_prob = 1.0f;
      // base: emission + the reservoir's light sample (pathtrace.metal:1100-1128)
      float pd[3] = {0.f, 0.f, 0.f};
      float pk = 0.0f, pdx = 0.f, pdy = 0.f, pdz = 0.f, ple[3] = {0.f, 0.f, 0.f};
      int pli = -1;
      float m_sumWu = 0.0f;
      uint32_t m_M = 0;
      const float4 R3 = rm.sumwu_m_valid[id];
      const float4 R0 = rm.lp_alpha[id], R1 = rm.ln_phat[id], R2 = rm.le_sumws[id];
      if (__float_as_int(R3.z) != 0 && __float_as_int(R3.y) != 0 && R3.x > 0.0f && R2.w > 0.0f && R1.w > 0.0f) {
        m_sumWu = R3.x; m_M = uint32_t(__float_as_int(R3.y));
        const float m_sumWs = R2.w;
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
              if (!p.nomis && e.pdf > 1e-20f) wnee = pdf_ris / (pdf_ris + e.pdf);
              float Wt = m_sumWs / (float(m_M) * ph);
              pd[0] = Fr * Wt * wnee; pd[1] = Fg * Wt * wnee; pd[2] = Fb * Wt * wnee;
              pk = scos * R0.w * Wt * wnee;
              pdx = dxn; pdy = dyn; pdz = dzn;
              ple[0] = R2.x; ple[1] = R2.y; ple[2] = R2.z;
              pli = __float_as_int(R3.w);
            }
          }
        }
      }
      const float base[3] = {EM.x + pd[0], EM.y + pd[1], EM.z + pd[2]};
      float gbase[3] = {0.f, 0.f, 0.f};  // sum over samples of the gradient reaching `base`
      if (p.bounces <= 1 || p.spp <= 0) {
        for (int c = 0; c < 3; ++c) gbase[c] = (cl && !(base[c] < p.clamp_value)) ? 0.0f : D[c];
      } else {
        const float inv_n = 1.0f / float(p.spp);
        const float g[3] = {D[0] * inv_n, D[1] * inv_n, D[2] * inv_n};
        for (int si = 0; si < p.spp; ++si) {
          ++samples;
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
            for (int c = 0; c < 3; ++c) gbase[c] += (cl && !(base[c] < p.clamp_value)) ? 0.0f : g[c];
            continue;
          }
          const float cos0 = nx2 * gnx + (ny2 * gny + nz2 * gnz);
          WalkFrom wf;
          wf.thr[0] = e0.r * cos0 / e0.pdf; wf.thr[1] = e0.g * cos0 / e0.pdf; wf.thr[2] = e0.b * cos0 / e0.pdf;
          wf.last_pdf = e0.pdf;
          wf.prev_b[0] = e0.r; wf.prev_b[1] = e0.g; wf.prev_b[2] = e0.b; wf.prev_cos = cos0;
          wf.prev_sumW = m_sumWu; wf.prev_M = m_M; wf.prev_delta = pdelta;
          const float ox = gpx + gnx * 0.001f, oy = gpy + gny * 0.001f, oz = gpz + gnz * 0.001f;
          const uint32_t st0 = pt.rng.state;
          Deferred dfr;
          float C[3];
          adjoint_path<kRis>(pt, tri_mat, ox, oy, oz, nx2, ny2, nz2, p.bounces - 1, 0.f, 0.f, 0.f, g[0], g[1], g[2],
                             sink, &dfr, C, &wf);
          bool clamped[3];
          float ge[3];
          for (int c = 0; c < 3; ++c) {
            clamped[c] = cl && !(base[c] + C[c] < p.clamp_value);
            ge[c] = clamped[c] ? 0.0f : g[c];
            gbase[c] += ge[c];
          }
          if (clamped[0] || clamped[1] || clamped[2]) {
            // the clamped channels' walk terms back out
            const uint32_t st1 = pt.rng.state;
            pt.rng.state = st0;
            adjoint_path<kRis>(pt, tri_mat, ox, oy, oz, nx2, ny2, nz2, p.bounces - 1, C[0], C[1], C[2],
                               clamped[0] ? -g[0] : 0.f, clamped[1] ? -g[1] : 0.f, clamped[2] ? -g[2] : 0.f, sink,
                               nullptr, nullptr, &wf);
            pt.rng.state = st1;
          }
          // B_0 = f cos / pdf: dlog B_0 = df / f, times the walk's radiance C
          const BsdfGrad bg = bsdf_grad(nx2, ny2, nz2, WO.x, WO.y, WO.z, gnx, gny, gnz, alpha2, metallic, AM.x, AM.y,
                                        AM.z);
          float drough = 0.0f;
          for (int c = 0; c < 3; ++c) {
            if (!(bg.f[c] > 0.0f)) continue;
            const float w = ge[c] * C[c] / bg.f[c];
            if (alb0) sink.add(m0, c, w * bg.da[c] * tx0[c]);
            drough += w * bg.dal2[c];
          }
          sink.add(m0, 3, drough * dal0);
        }
      }
      // base terms: the first hit's emission and the held light sample Le f k
      for (int c = 0; c < 3; ++c) sink.add(m0, 4 + c, gbase[c]);
      if (pli >= 0 && pk != 0.0f) {
        const int ml = tri_mat[s.lights[pli]];
        const BsdfGrad bg = bsdf_grad(pdx, pdy, pdz, WO.x, WO.y, WO.z, gnx, gny, gnz, alpha2, metallic, AM.x, AM.y,
                                      AM.z);
        float drough = 0.0f;
        for (int c = 0; c < 3; ++c) {
          const float gt = gbase[c] * pk;
          sink.add(ml, 4 + c, gt * bg.f[c]);
          if (alb0) sink.add(m0, c, gt * ple[c] * bg.da[c] * tx0[c]);
          drough += gt * ple[c] * bg.dal2[c];
        }
        sink.add(m0, 3, drough * dal0);
      }
    }
  }
  const unsigned long long tot = __reduce_add_sync(0xffffffffu, samples);
  if ((threadIdx.x & 31) == 0 && tot) atomicAdd(ctr, tot);
  if (use_shared) {
    __syncthreads();
    for (int i = threadIdx.x; i < n_mat * kMatParams; i += blockDim.x)
      if (sh[i] != 0.0f) atomicAdd(grad + i, sh[i]);
  }
}

// Copy per-material parameters into the triangles (albedo, rough, emission, ior).
__global__ void k_apply_materials(rm_triangle* tris, const int32_t* __restrict__ tri_mat,
                                  const float* __restrict__ mats, int n_tris) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_tris) return;
  const int m = tri_mat[i];
  if (m < 0) return;
  const float* q = mats + size_t(m) * kMatParams;
  rm_triangle& t = tris[i];
  t.ar = q[0]; t.ag = q[1]; t.ab = q[2];
  t.rough = q[3];
  t.er = q[4]; t.eg = q[5]; t.eb = q[6];
  t.ior = q[7];
}

}  // namespace

cudaError_t launch_adjoint(int lanes, const Scene& s, const Params& p, uint64_t seed, const int32_t* tri_mat,
                           int n_mat, const float* dLdI, float* grad, unsigned long long* ctr, uint32_t* err,
                           cudaStream_t st) {
  const size_t shmem = size_t(n_mat) * kMatParams * sizeof(float);
  const int use_shared = shmem <= 32 * 1024 ? 1 : 0;
  const size_t threads = size_t(p.width) * size_t(p.height) * size_t(lanes);
  const unsigned grid = unsigned((threads + 255) / 256);
  const size_t sm = use_shared ? shmem : 0;
#define RM_ADJ(L, R) k_adjoint<L, R><<<grid, 256, sm, st>>>(s, p, seed, tri_mat, n_mat, dLdI, grad, use_shared, ctr, err)
  const bool ris = p.restir_candidates > 1;
  if (lanes == 32) { if (ris) RM_ADJ(32, true); else RM_ADJ(32, false); }
  else if (lanes == 8) { if (ris) RM_ADJ(8, true); else RM_ADJ(8, false); }
  else { if (ris) RM_ADJ(1, true); else RM_ADJ(1, false); }
#undef RM_ADJ
  return cudaGetLastError();
}

cudaError_t apply_materials(rm_triangle* tris, const int32_t* tri_mat, const float* mats, int n_tris,
                            cudaStream_t st) {
  if (n_tris <= 0) return cudaSuccess;
  k_apply_materials<<<(n_tris + 255) / 256, 256, 0, st>>>(tris, tri_mat, mats, n_tris);
  return cudaGetLastError();
}

cudaError_t launch_adjoint_restir(const Scene& s, const Params& p, uint64_t seed, const GBufSoA& gb, const ResSoA& rm,
                                  const int32_t* tri_mat, int n_mat, const float* dLdI, const float* dLdalb,
                                  float* grad, unsigned long long* ctr, uint32_t* err, cudaStream_t st) {
  const size_t shmem = size_t(n_mat) * kMatParams * sizeof(float);
  const int use_shared = shmem <= 32 * 1024 ? 1 : 0;
  const unsigned grid = unsigned((size_t(p.width) * size_t(p.height) + 255) / 256);
  const size_t sm = use_shared ? shmem : 0;
  if (p.restir_candidates > 1)
    k_adjoint_restir<true><<<grid, 256, sm, st>>>(s, p, seed, gb, rm, tri_mat, n_mat, dLdI, dLdalb, grad, use_shared,
                                                  ctr, err);
  else
    k_adjoint_restir<false><<<grid, 256, sm, st>>>(s, p, seed, gb, rm, tri_mat, n_mat, dLdI, dLdalb, grad,
                                                   use_shared, ctr, err);
  return cudaGetLastError();
}

}  // namespace rmd
