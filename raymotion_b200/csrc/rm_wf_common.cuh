// rm_wf_common.cuh - pieces shared by the wavefront renderers (rm_wavefront.cu,
// ReSTIR shading; rm_batch.cu, batched plain-path rendering): the per-path
// registers between waves, warp-aggregated queue appends, and one vertex of the
// reference path loop (pathtrace.metal:564-726, :1175-1251) with NEE's shadow
// ray left to a separate traversal pass.
#pragma once

#include "rm_device.cuh"

namespace rmd {
namespace wf {

// meta bits of a path slot
constexpr uint32_t kInd = 1u;        // K5 indirect path (kind 1); else camera path (kind 3)
constexpr uint32_t kDelta = 2u;      // previous vertex was delta (pdel / prev_delta)
constexpr uint32_t kExt = 4u;        // an extension ray is queued
constexpr uint32_t kShadow = 8u;     // a shadow ray is queued
constexpr uint32_t kFinish = 16u;    // path ended; its last shadow ray is still queued

struct PathRegs {
  float ax, ay, az, tx, ty, tz;
  float ox, oy, oz, dx, dy, dz;
  float last_pdf, psumW, pbr, pbg, pbb, pbcos;
  uint32_t pM;
  int v;
  uint32_t meta;
};

// Append flagged threads to a queue; the threads of a warp that reach this
// together share one atomic.
__device__ __forceinline__ void append(int* q, int* count, bool flag, int value) {
  const unsigned m = __activemask();
  const unsigned b = __ballot_sync(m, flag);
  if (!b) return;
  const int lane = int(threadIdx.x & 31);
  const int leader = __ffs(m) - 1;
  int base = 0;
  if (lane == leader) base = atomicAdd(count, __popc(b));
  base = __shfl_sync(m, base, leader);
  if (flag) q[base + __popc(b & ((1u << lane) - 1u))] = value;
}

__device__ __forceinline__ void warp_add(unsigned long long* ctr, uint32_t v) {
  unsigned long long s = __reduce_add_sync(0xffffffffu, v);
  if ((threadIdx.x & 31) == 0 && s) atomicAdd(ctr, s);
}

__device__ __forceinline__ void clamp3(const Params& p, float& r, float& g, float& b) {
  if (p.clamp_value > 0.0f) {
    r = fminf(r, p.clamp_value); g = fminf(g, p.clamp_value); b = fminf(b, p.clamp_value);
  }
}

// One vertex of the path loop (pathtrace.metal:564-726 for camera paths,
// :1175-1251 for kind-1 indirect paths).  Returns true when the path goes on
// (a new extension ray is in r.o / r.d).  In an opaque scene NEE leaves its
// shadow ray and the contribution of a visible light in so / sd / c; otherwise
// it tests visibility itself and adds the light at once.
// MAT 0: opaque surface, 1: dielectric (hit.ior > 1.0001).  NEE 0: the scene
// is opaque and NEE takes one candidate (the single-candidate branch inlined);
// 1: any scene and candidate count; 2: an opaque scene, any candidate count
// (without the in-place shadow test of partially transparent scenes).
template <int MAT, int NEE = 1>
__device__ bool vertex(Tracer& pt, const Params& p, PathRegs& r, const Hit& hit, bool& has_shadow, float4& so,
                       float4& sd, float4& c) {
  // the checked build: a hit whose triangle failed its check ends the path
  if (kChecked && bad_index(hit.tri, pt.s.n_tris, pt.err, kSiteVertex)) return false;
  const bool ind = (r.meta & kInd) != 0;
  float pnx = hit.nix, pny = hit.niy, pnz = hit.niz;
  float geom = hit.ngx * pnx + (hit.ngy * pny + hit.ngz * pnz);
  if (geom < 0.0f) { pnx = -pnx; pny = -pny; pnz = -pnz; }
  float ndot = r.dx * pnx + (r.dy * pny + r.dz * pnz);
  bool front = true;
  if (ndot > 0.0f) { pnx = -pnx; pny = -pny; pnz = -pnz; front = false; }
  float wox = -r.dx, woy = -r.dy, woz = -r.dz;
  float rough = hit.rough;
  if (rough < 0.0f) rough = 0.0f;
  if (rough > 1.0f) rough = 1.0f;
  if (rough < 0.02f) rough = 0.02f;
  float alpha = rough * rough;
  float alpha2 = alpha * alpha;
  const rm_triangle& lt = pt.s.tris[hit.tri];
  float metallic = lt.metallic;
  if (metallic < 0.0f) metallic = 0.0f;
  if (metallic > 1.0f) metallic = 1.0f;
  if (r.v == 0 || (r.meta & kDelta)) {
    r.ax += hit.er * r.tx; r.ay += hit.eg * r.ty; r.az += hit.eb * r.tz;
  } else {
    float lx = hit.px - r.ox, ly = hit.py - r.oy, lz = hit.pz - r.oz;
    float dist2 = lx * lx + ly * ly + lz * lz;
    float dist = sqrtf(dist2);
    float pl = 1e30f;
    const float lta = lt.alpha;
    if (dist > 1e-20f && r.last_pdf > 1e-20f && r.pM > 0 && r.psumW > 1e-20f) {
      float ph = lum3(hit.er * r.pbr * r.pbcos * lta, hit.eg * r.pbg * r.pbcos * lta,
                      hit.eb * r.pbb * r.pbcos * lta);
      if (ph > 1e-20f) pl = float(r.pM) * ph / r.psumW;
      else {
        float inv = 1.0f / dist;
        float lxn = lx * inv, lyn = ly * inv, lzn = lz * inv;
        float cos_l = -(lt.nn.x * lxn + (lt.nn.y * lyn + lt.nn.z * lzn));
        if (cos_l > 1e-8f) {
          float lum = lum3(lt.er, lt.eg, lt.eb);
          if (lum < 1e-6f) lum = 1e-6f;
          pl = dist2 * lum / (cos_l * p.light_total);
        }
      }
    } else if (dist > 1e-20f && r.last_pdf > 1e-20f) {
      float inv = 1.0f / dist;
      lx *= inv; ly *= inv; lz *= inv;
      float cos_l = -(lt.nn.x * lx + (lt.nn.y * ly + lt.nn.z * lz));
      if (cos_l > 1e-8f) {
        float lum = lum3(lt.er, lt.eg, lt.eb);
        if (lum < 1e-6f) lum = 1e-6f;
        pl = dist2 * lum / (cos_l * p.light_total);
      }
    }
    float w = p.nomis ? 0.0f : ((r.last_pdf + pl > 1e-20f) ? r.last_pdf / (r.last_pdf + pl) : 0.0f);
    r.ax += hit.er * r.tx * w; r.ay += hit.eg * r.ty * w; r.az += hit.eb * r.tz * w;
  }
  if (MAT == 1) {
    float nx2, ny2, nz2, es;
    bool valid = pt.sample_dielectric(wox, woy, woz, pnx, pny, pnz, r.dx, r.dy, r.dz, hit.ior, front, rough, alpha2,
                                      nx2, ny2, nz2, es);
    if (!valid) return false;
    r.tx *= es; r.ty *= es; r.tz *= es;
    float sg = 1.0f;
    if (nx2 * pnx + (ny2 * pny + nz2 * pnz) < 0.0f) sg = -1.0f;
    r.ox = hit.px + pnx * 0.001f * sg;
    r.oy = hit.py + pny * 0.001f * sg;
    r.oz = hit.pz + pnz * 0.001f * sg;
    r.dx = nx2; r.dy = ny2; r.dz = nz2;
    r.meta |= kDelta;
    r.psumW = 0.0f; r.pM = 0;
  } else {
    float spec_prob = 0.05f + 0.95f * metallic;
    if (spec_prob > 0.98f) spec_prob = 0.98f;
    if (metallic >= 0.999f) spec_prob = 1.0f;
    float dlr, dlg, dlb, cur_sumW;
    uint32_t cur_M;
    if (NEE != 1 || p.opaque) {
      float sdist, sox, soy, soz, sdx, sdy, sdz;
      bool has_ray;
      if (NEE == 0)
        pt.nee_single_deferred(hit.px, hit.py, hit.pz, pnx, pny, pnz, wox, woy, woz, rough, metallic, spec_prob,
                               hit.ar, hit.ag, hit.ab, dlr, dlg, dlb, cur_sumW, cur_M, has_ray, sox, soy, soz, sdx,
                               sdy, sdz, sdist);
      else
        pt.direct_lighting_deferred(hit.px, hit.py, hit.pz, pnx, pny, pnz, wox, woy, woz, rough, metallic, spec_prob,
                                  hit.ar, hit.ag, hit.ab, dlr, dlg, dlb, cur_sumW, cur_M, has_ray, sox, soy, soz,
                                  sdx, sdy, sdz, sdist);
      if (has_ray) {
        has_shadow = true;
        so = make_float4(sox, soy, soz, sdist);
        sd = make_float4(sdx, sdy, sdz, 0.f);
        c = make_float4(dlr * r.tx, dlg * r.ty, dlb * r.tz, 0.f);
      }
    } else if (NEE == 1) {
      // partially transparent scene: the shadow test draws random numbers
      // (pathtrace.metal:536-550), so it runs here, in stream order
      pt.direct_lighting(hit.px, hit.py, hit.pz, pnx, pny, pnz, wox, woy, woz, rough, metallic, spec_prob, hit.ar,
                         hit.ag, hit.ab, dlr, dlg, dlb, cur_sumW, cur_M);
      r.ax += dlr * r.tx; r.ay += dlg * r.ty; r.az += dlb * r.tz;
    }
    float nx2, ny2, nz2;
    if (pt.U() < spec_prob) {
      float hx, hy, hz;
      pt.sample_ggx_half(alpha2, pnx, pny, pnz, hx, hy, hz);
      float md = wox * hx + (woy * hy + woz * hz);
      if (!(md > 1e-8f)) return false;
      nx2 = 2.0f * md * hx - wox;
      ny2 = 2.0f * md * hy - woy;
      nz2 = 2.0f * md * hz - woz;
      r.meta = (r.meta & ~kDelta) | ((rough <= 0.0201f) ? kDelta : 0u);
    } else {
      pt.sample_cosine(pnx, pny, pnz, nx2, ny2, nz2);
      r.meta &= ~kDelta;
    }
    float ncos = nx2 * pnx + (ny2 * pny + nz2 * pnz);
    if (!(ncos > 1e-8f)) return false;
    {
      float d = 1.0f / sqrtf(nx2 * nx2 + ny2 * ny2 + nz2 * nz2);
      nx2 *= d; ny2 *= d; nz2 *= d;
    }
    Bsdf e = Tracer::eval_bsdf(nx2, ny2, nz2, wox, woy, woz, pnx, pny, pnz, alpha2, metallic, spec_prob, hit.ar,
                               hit.ag, hit.ab);
    if (!(e.pdf > 1e-12f)) return false;
    r.last_pdf = e.pdf;
    float cos_i = nx2 * pnx + (ny2 * pny + nz2 * pnz);
    r.tx *= e.r * cos_i / e.pdf;
    r.ty *= e.g * cos_i / e.pdf;
    r.tz *= e.b * cos_i / e.pdf;
    r.psumW = cur_sumW; r.pM = cur_M;
    r.pbr = e.r; r.pbg = e.g; r.pbb = e.b; r.pbcos = cos_i;
    r.ox = hit.px + pnx * 0.001f;
    r.oy = hit.py + pny * 0.001f;
    r.oz = hit.pz + pnz * 0.001f;
    r.dx = nx2; r.dy = ny2; r.dz = nz2;
  }
  if (!ind) {
    if (r.tx < 0.0f) r.tx = 0.0f;
    if (r.ty < 0.0f) r.ty = 0.0f;
    if (r.tz < 0.0f) r.tz = 0.0f;
  }
  float mx = fmaxf(r.tx, r.ty);
  mx = fmaxf(mx, r.tz);
  if (!(mx >= 1e-12f)) return false;
  if (p.rr && r.v >= (ind ? 2 : 1)) {
    float rr = mx;
    if (rr < 0.05f) rr = 0.05f;
    if (rr > 0.9f) rr = 0.9f;
    if (!(pt.U() <= rr)) return false;
    float ir = 1.0f / rr;
    r.tx *= ir; r.ty *= ir; r.tz *= ir;
  }
  r.v += 1;
  return r.v < p.bounces;
}

}  // namespace wf
}  // namespace rmd
