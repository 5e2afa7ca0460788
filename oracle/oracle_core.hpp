// oracle_core.hpp - CPU oracle of raymotion's path-tracing hot path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker: the tests, the smoke
// check and the CPU-baseline leg of the benchmark call it; the product
// (librmcuda.so) never includes or links it.
//
// It restates, scalar and in IEEE fp32, what the reference's Metal shaders do
// for one frame (reference src/engine/pathtrace.metal) and how its host picks
// the passes (src/engine/metal.mm:95-414).  Each function cites the lines it
// follows.  Expression trees keep the reference's operand order, because the
// CUDA kernels are compared bit for bit on identical RNG streams; the build
// uses -ffp-contract=off so that no a*b+c is fused.
//
// Where the reference is ambiguous or order-dependent, the oracle and the CUDA
// backend share one documented rule:
//  * dot(a,b) = (a.x*b.x + a.y*b.y) + a.z*b.z where the reference calls Metal's
//    dot(); normalize(v) = v * (1/sqrt(x*x + (y*y + z*z)));
//  * closest hit: smallest t, ties broken by the smaller triangle index (the
//    reference keeps the first one its traversal order finds,
//    pathtrace.metal:158); box culling keeps a relative slack of 2^-16 so that
//    no BVH can cull a hit that another BVH keeps;
//  * sin/cos/atan/exp come from include/rm_detmath.h;
//  * transparent crossings are capped at kMaxAlphaCrossings per ray
//    (pathtrace.metal:539-548 has no cap);
//  * the 17-hex-digit constant of pathtrace.metal:937 is its low 64 bits.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "rm_detmath.h"
#include "rmcuda.h"

namespace orc {

constexpr int kMaxAlphaCrossings = 1024;
constexpr float kBoxSlack = 1.0000152587890625f;  // 1 + 2^-16
constexpr uint64_t kSpatialSeedXor = 0x1B54A35A6F31B458ull;

template <class F> struct V3 { F x, y, z; };
template <class F> inline V3<F> mk(F x, F y, F z) { return V3<F>{x, y, z}; }
template <class F> inline V3<F> vf(const rm_vec3& v) { return V3<F>{F(v.x), F(v.y), F(v.z)}; }

// pathtrace.metal:93-101.  seed(): splitmix64 finaliser of s + golden ratio,
// truncated to 32 bits; uniform01(): LCG step, PCG RXS-M-XS output, top 24 bits.
struct Rng {
  uint32_t state = 0;
  void seed(uint64_t s) {
    uint64_t z = s + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    state = uint32_t(z ^ (z >> 31));
  }
  float uniform01() {
    state = state * 747796405u + 2891336453u;
    uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
    return float(((word >> 22u) ^ word) >> 8u) * 0x1p-24f;
  }
};

template <class F> inline F lum3(F r, F g, F b) {
  return F(0.2126f) * r + F(0.7152f) * g + F(0.0722f) * b;
}

inline void sincos_any(float a, float* s, float* c) { rm_sincosf(a, s, c); }
inline void sincos_any(double a, double* s, double* c) { *s = std::sin(a); *c = std::cos(a); }
inline float atan_any(float x) { return rm_atanf(x); }
inline double atan_any(double x) { return std::atan(x); }

// Preorder node with an escape link (metal_types.h:16-20, built by
// metal.mm:129-144): `escape` is the index after the node's subtree.
struct PNode {
  float mn[3], mx[3];
  int escape, offset, count;
};

// metal_types.h:21-30 plus the switches this build adds (rr).
struct Params {
  rm_camera camera;
  int width, height, spp, bounces, nodes, lights, adapt_min, adapt_step, nomis, opaque;
  float light_total, resolution, clamp_value, adapt_rel, adapt_abs;
  int restir_candidates, restir_spatial, restir_mcap;
  float restir_radius;
  rm_camera prevCamera;
  int hasHistory;
  int rr;
};

// The reference's ReSTIR records (metal_types.h:32-56), same field order.
struct GBuf {
  rm_vec3 pos, normal, albedo, wo, emission;
  float rough, metallic, ior;
  int kind;
};
struct Reservoir {
  rm_vec3 lightPos, lightNormal, emission;
  float alpha, p_hat, sumWs, sumWu;
  uint32_t M, valid;
};
static_assert(sizeof(GBuf) == 76, "G-buffer record must match the reference ABI");
static_assert(sizeof(Reservoir) == 60, "reservoir record must match the reference ABI");

struct SceneRef {
  const rm_triangle* tris = nullptr;
  int n_tris = 0;
  std::vector<PNode> nodes;
  const int32_t* indices = nullptr;
  const int32_t* lights = nullptr;
  const float* cdf = nullptr;
  int n_lights = 0;
  float light_total = 0;
  const rm_vec3* texels = nullptr;
};

template <class F> struct Hit {
  bool hit = false;
  F t = F(1e30f);
  int tri = -1;
  F u = 0, v = 0;
  V3<F> p{0, 0, 0};
  V3<F> n_interp{0, 0, 0};
  F ar = 0, ag = 0, ab = 0, er = 0, eg = 0, eb = 0, ior = 0, rough = 0;
  int shader = 0;
  V3<F> n_geom{0, 0, 0};
  F txr = 1, txg = 1, txb = 1;  // texel colour the albedo was multiplied by
};

struct Counters {
  uint64_t rays = 0;
};

template <class F> struct Tracer {
  const SceneRef* s;
  const Params* p;
  Rng rng;
  Counters* ctr = nullptr;

  struct Bsdf { F r = 0, g = 0, b = 0, pdf = 0; };
  struct Diel { bool valid = true; F n_x = 0, n_y = 0, n_z = 0, eta_scale = 1; };

  F U() { return F(rng.uniform01()); }

  static V3<F> cross(V3<F> a, V3<F> b) {
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
  }
  static F dot(V3<F> a, V3<F> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

  // Stackless escape-link traversal, pathtrace.metal:137-161, with the
  // deterministic tie-break and slack described in the header.
  Hit<F> intersect(V3<F> ro, V3<F> rd, F dist, bool shadow) {
    if (ctr) ctr->rays++;
    Hit<F> h;
    h.t = dist;
    if (p->nodes == 0) return h;
    V3<F> safe = mk(rd.x == F(0) ? F(1e-30f) : rd.x, rd.y == F(0) ? F(1e-30f) : rd.y,
                    rd.z == F(0) ? F(1e-30f) : rd.z);
    V3<F> inv = mk(F(1) / safe.x, F(1) / safe.y, F(1) / safe.z);
    const int M = int(s->nodes.size());
    int ni = 0;
    while (ni < M) {
      const PNode& n = s->nodes[size_t(ni)];
      F ax = (F(n.mn[0]) - ro.x) * inv.x, ay = (F(n.mn[1]) - ro.y) * inv.y, az = (F(n.mn[2]) - ro.z) * inv.z;
      F bx = (F(n.mx[0]) - ro.x) * inv.x, by = (F(n.mx[1]) - ro.y) * inv.y, bz = (F(n.mx[2]) - ro.z) * inv.z;
      F lx = std::min(ax, bx), ly = std::min(ay, by), lz = std::min(az, bz);
      F hx = std::max(ax, bx), hy = std::max(ay, by), hz = std::max(az, bz);
      F near_t = std::max(F(0), std::max(lx, std::max(ly, lz)));
      F far_t = std::min(h.t, std::min(hx, std::min(hy, hz)));
      if (near_t > far_t * F(kBoxSlack)) { ni = n.escape; continue; }
      ++ni;
      if (n.count == 0) continue;
      for (int k = 0; k < n.count; ++k) {
        int j = s->indices[n.offset + k];
        const rm_triangle& t = s->tris[j];
        V3<F> v0 = vf<F>(t.v0);
        V3<F> e1 = mk(F(t.v1.x) - v0.x, F(t.v1.y) - v0.y, F(t.v1.z) - v0.z);
        V3<F> e2 = mk(F(t.v2.x) - v0.x, F(t.v2.y) - v0.y, F(t.v2.z) - v0.z);
        V3<F> pv = cross(rd, e2);
        F det = dot(e1, pv);
        if (std::fabs(det) < F(1e-12f)) continue;
        V3<F> tv = mk(ro.x - v0.x, ro.y - v0.y, ro.z - v0.z);
        F u = dot(tv, pv) / det;
        if (u < F(0) || u > F(1)) continue;
        V3<F> q = cross(tv, e1);
        F v = dot(rd, q) / det;
        if (v < F(0) || u + v > F(1)) continue;
        F d = dot(e2, q) / det;
        if (d > F(1e-8f) && (d < h.t || (d == h.t && h.tri >= 0 && j < h.tri))) {
          h.t = d; h.tri = j; h.u = u; h.v = v; h.hit = true;
          if (shadow) return h;
        }
      }
    }
    h.p = mk(ro.x + rd.x * h.t, ro.y + rd.y * h.t, ro.z + rd.z * h.t);
    return h;
  }
  bool cast_shadow_ray(V3<F> ro, V3<F> rd, F dist) { return intersect(ro, rd, dist, true).hit; }

  static void hsv2rgb(F h, F sat, F val, F& r, F& g, F& b) {  // pathtrace.metal:27-64
    F c = sat * val;
    F hm = h / F(60);
    F md = hm - std::floor(hm / F(2)) * F(2);
    F x = c * (F(1) - std::fabs(md - F(1)));
    F m = val - c;
    F cr = 0, cg = 0, cb = 0;
    if (h < F(60)) { cr = c; cg = x; }
    else if (h < F(120)) { cr = x; cg = c; }
    else if (h < F(180)) { cg = c; cb = x; }
    else if (h < F(240)) { cg = x; cb = c; }
    else if (h < F(300)) { cr = x; cb = c; }
    else if (h < F(360)) { cr = c; cb = x; }
    cr += m; cg += m; cb += m;
    r = cr * F(255); g = cg * F(255); b = cb * F(255);
  }

  // pathtrace.metal:165-204: closest hit plus its attributes.
  Hit<F> cast_ray(V3<F> ro, V3<F> rd, F dist) {
    Hit<F> h = intersect(ro, rd, dist, false);
    if (h.tri >= 0) {
      const rm_triangle& t = s->tris[h.tri];
      F w = F(1) - (h.u + h.v);
      F nx = w * F(t.n0.x) + (h.u * F(t.n1.x) + h.v * F(t.n2.x));
      F ny = w * F(t.n0.y) + (h.u * F(t.n1.y) + h.v * F(t.n2.y));
      F nz = w * F(t.n0.z) + (h.u * F(t.n1.z) + h.v * F(t.n2.z));
      F d = F(1) / std::sqrt(nx * nx + (ny * ny + nz * nz));
      h.n_interp = mk(nx * d, ny * d, nz * d);
      h.ar = F(t.ar); h.ag = F(t.ag); h.ab = F(t.ab);
      if (t.texture_offset >= 0) {
        F tu = w * F(t.tu0) + h.u * F(t.tu1) + h.v * F(t.tu2);
        F tv = w * F(t.tv0) + h.u * F(t.tv1) + h.v * F(t.tv2);
        tu = std::min(tu - std::floor(tu), F(0.99999994f));
        tv = std::min(tv - std::floor(tv), F(0.99999994f));
        int x = std::min(int(tu * F(t.texture_width)), t.texture_width - 1);
        int y = t.texture_height - 1 - std::min(int(tv * F(t.texture_height)), t.texture_height - 1);
        const rm_vec3& c = s->texels[size_t(t.texture_offset) + size_t(y) * size_t(t.texture_width) + size_t(x)];
        h.ar *= F(c.x); h.ag *= F(c.y); h.ab *= F(c.z);
        h.txr = F(c.x); h.txg = F(c.y); h.txb = F(c.z);
      }
      h.er = F(t.er); h.eg = F(t.eg); h.eb = F(t.eb);
      h.ior = F(t.ior); h.rough = F(t.rough); h.shader = t.shader;
      h.n_geom = vf<F>(t.n);
      if (h.shader == 1) {
        F az = atan_any(h.p.x / h.p.z) * F(180) / F(3.141592653589793f) + ((h.p.z > F(0)) ? F(0) : F(180));
        F hh = (az - std::floor(az / F(360)) * F(360)) / F(360);
        hsv2rgb(hh, F(0.8f), F(1), h.ar, h.ag, h.ab);
      }
    }
    return h;
  }

  // pathtrace.metal:65-78
  static void tangent(F nx, F ny, F nz, F& tx, F& ty, F& tz, F& bx, F& by, F& bz) {
    if (std::fabs(nx) > F(0.1f)) { tx = nz; ty = F(0); tz = -nx; }
    else { tx = F(0); ty = -nz; tz = ny; }
    F l = F(1) / std::sqrt(tx * tx + ty * ty + tz * tz);
    tx *= l; ty *= l; tz *= l;
    bx = ny * tz - nz * ty;
    by = nz * tx - nx * tz;
    bz = nx * ty - ny * tx;
  }
  // pathtrace.metal:205-220
  void sample_cosine(F nx, F ny, F nz, F& ox, F& oy, F& oz) {
    F ru = U();
    F phi = U() * F(2.0f * 3.141592653589793f);
    F sp, c;
    sincos_any(phi, &sp, &c);
    F rr = std::sqrt(ru);
    F lx = rr * c, ly = rr * sp, lz = std::sqrt(std::max(F(0), F(1) - ru));
    F tx, ty, tz, bx, by, bz;
    tangent(nx, ny, nz, tx, ty, tz, bx, by, bz);
    ox = tx * lx + (bx * ly + nx * lz);
    oy = ty * lx + (by * ly + ny * lz);
    oz = tz * lx + (bz * ly + nz * lz);
  }
  // pathtrace.metal:221-242 (the first draw is discarded, :224-225)
  void sample_ggx_half(F alpha2, F nx, F ny, F nz, F& hx, F& hy, F& hz) {
    (void)U();
    F rv = U();
    F phi = U() * F(2.0f * 3.141592653589793f);
    F sp, c;
    sincos_any(phi, &sp, &c);
    F cs = std::sqrt((F(1) - rv) / (F(1) + (alpha2 - F(1)) * rv));
    F sn = std::sqrt(std::max(F(0), F(1) - cs * cs));
    F lx = sn * c, ly = sn * sp, lz = cs;
    F tx, ty, tz, bx, by, bz;
    tangent(nx, ny, nz, tx, ty, tz, bx, by, bz);
    hx = tx * lx + (bx * ly + nx * lz);
    hy = ty * lx + (by * ly + ny * lz);
    hz = tz * lx + (bz * ly + nz * lz);
    F d = F(1) / std::sqrt(hx * hx + hy * hy + hz * hz);
    hx *= d; hy *= d; hz *= d;
  }
  // pathtrace.metal:243-295
  static Bsdf eval_bsdf(F wix, F wiy, F wiz, F wox, F woy, F woz, F nx, F ny, F nz, F alpha2,
                        F metallic, F spec_prob, F ar, F ag, F ab) {
    const F kPi = F(3.141592653589793f);
    Bsdf out;
    F cos_i = wix * nx + (wiy * ny + wiz * nz);
    F cos_o = wox * nx + (woy * ny + woz * nz);
    if (!(cos_i > F(1e-8f) && cos_o > F(1e-8f))) return out;
    F hx = wix + wox, hy = wiy + woy, hz = wiz + woz;
    F hl = std::sqrt(hx * hx + hy * hy + hz * hz);
    if (!(hl > F(1e-8f))) return out;
    F inv = F(1) / hl;
    hx *= inv; hy *= inv; hz *= inv;
    F cos_h = hx * nx + (hy * ny + hz * nz);
    F vo_h = wox * hx + (woy * hy + woz * hz);
    if (cos_h < F(0)) { hx = -hx; hy = -hy; hz = -hz; cos_h = -cos_h; vo_h = -vo_h; }
    if (!(vo_h > F(1e-8f))) return out;
    F dd = cos_h * cos_h * (alpha2 - F(1)) + F(1);
    F D = alpha2 / (kPi * dd * dd);
    F g1 = F(2) * cos_o / (cos_o + std::sqrt(cos_o * cos_o + alpha2 * (F(1) - cos_o * cos_o)));
    F g2 = F(2) * cos_i / (cos_i + std::sqrt(cos_i * cos_i + alpha2 * (F(1) - cos_i * cos_i)));
    F G = g1 * g2;
    F om = F(1) - vo_h;
    om *= om; om *= om; om *= F(1) - vo_h;
    F di = F(1) - metallic;
    F f0r = F(0.04f) * di + ar * metallic, f0g = F(0.04f) * di + ag * metallic, f0b = F(0.04f) * di + ab * metallic;
    F fr = f0r + (F(1) - f0r) * om, fg = f0g + (F(1) - f0g) * om, fb = f0b + (F(1) - f0b) * om;
    F kdr = ar * di * (F(1) - fr), kdg = ag * di * (F(1) - fg), kdb = ab * di * (F(1) - fb);
    F base = D * G / (F(4) * cos_i * cos_o);
    out.r = kdr / kPi + base * fr;
    out.g = kdg / kPi + base * fg;
    out.b = kdb / kPi + base * fb;
    F pdf_d = cos_i / kPi;
    F pdf_s = D * cos_h / (F(4) * vo_h);
    out.pdf = (F(1) - spec_prob) * pdf_d + spec_prob * pdf_s;
    return out;
  }

  int pick_light(F pick) {  // pathtrace.metal:323-331 (binary search over the CDF)
    int lo = 0, hi = p->lights - 1;
    while (lo < hi) {
      int mid = (lo + hi) / 2;
      if (F(s->cdf[mid]) >= pick) hi = mid; else lo = mid + 1;
    }
    return s->lights[lo];
  }

  bool occluded(V3<F> so, V3<F> d, F dist) {
    return p->opaque ? cast_shadow_ray(so, d, dist) : cast_alpha_ray(so, d, dist).tri >= 0;
  }

  // pathtrace.metal:299-469: NEE; legacy single sample for Mc <= 1, else RIS.
  void direct_lighting(F px, F py, F pz, F nx, F ny, F nz, F wox, F woy, F woz, F rough,
                       F metallic, F spec_prob, F ar, F ag, F ab, F& o_r, F& o_g, F& o_b,
                       F& out_sumW, uint32_t& out_M) {
    o_r = o_g = o_b = 0;
    out_sumW = 0;
    out_M = 0;
    if (p->lights == 0 || !(F(p->light_total) > F(1e-12f))) return;
    int Mc = p->restir_candidates;
    if (Mc < 1) Mc = 1;
    if (Mc > 32) Mc = 32;
    F r2 = rough;
    if (r2 < F(0)) r2 = F(0);
    if (r2 > F(1)) r2 = F(1);
    if (r2 < F(0.02f)) r2 = F(0.02f);
    F alpha2 = (r2 * r2) * (r2 * r2);
    const F LT = F(p->light_total);
    if (Mc <= 1) {
      F pick = U() * LT;
      const rm_triangle& t = s->tris[pick_light(pick)];
      F lu = U(), lv = U();
      if (lu + lv > F(1)) { lu = F(1) - lu; lv = F(1) - lv; }
      F lw = F(1) - lu - lv;
      F ldx = lw * F(t.v0.x) + (lu * F(t.v1.x) + lv * F(t.v2.x)) - px;
      F ldy = lw * F(t.v0.y) + (lu * F(t.v1.y) + lv * F(t.v2.y)) - py;
      F ldz = lw * F(t.v0.z) + (lu * F(t.v1.z) + lv * F(t.v2.z)) - pz;
      F dist = std::sqrt(ldx * ldx + ldy * ldy + ldz * ldz);
      if (!(dist > F(0.003f))) { out_M = 1; return; }
      F inv = F(1) / dist;
      ldx *= inv; ldy *= inv; ldz *= inv;
      F lcos = -(F(t.nn.x) * ldx + (F(t.nn.y) * ldy + F(t.nn.z) * ldz));
      F scos = nx * ldx + (ny * ldy + nz * ldz);
      if (!(lcos > F(1e-8f) && scos > F(1e-8f))) { out_M = 1; return; }
      F lt_lum = lum3(F(t.er), F(t.eg), F(t.eb));
      if (lt_lum < F(1e-6f)) lt_lum = F(1e-6f);
      F pdf = dist * dist * lt_lum / (lcos * LT);
      V3<F> so = mk(px + nx * F(0.002f), py + ny * F(0.002f), pz + nz * F(0.002f));
      if (occluded(so, mk(ldx, ldy, ldz), dist - F(0.003f))) {
        Bsdf eo = eval_bsdf(ldx, ldy, ldz, wox, woy, woz, nx, ny, nz, alpha2, metallic, spec_prob, ar, ag, ab);
        F Fr0 = F(t.er) * eo.r * scos * F(t.alpha);
        F Fg0 = F(t.eg) * eo.g * scos * F(t.alpha);
        F Fb0 = F(t.eb) * eo.b * scos * F(t.alpha);
        F ph0 = lum3(Fr0, Fg0, Fb0);
        out_sumW = (ph0 > F(0) && pdf > F(1e-12f)) ? ph0 / pdf : F(0);
        out_M = 1;
        return;
      }
      Bsdf e = eval_bsdf(ldx, ldy, ldz, wox, woy, woz, nx, ny, nz, alpha2, metallic, spec_prob, ar, ag, ab);
      if (!(pdf > F(1e-12f))) { out_M = 1; return; }
      F Fr = F(t.er) * e.r * scos * F(t.alpha);
      F Fg = F(t.eg) * e.g * scos * F(t.alpha);
      F Fb = F(t.eb) * e.b * scos * F(t.alpha);
      F ph = lum3(Fr, Fg, Fb);
      out_sumW = (ph > F(0)) ? ph / pdf : F(0);
      out_M = 1;
      F wnee = F(1);
      if (!p->nomis && e.pdf > F(1e-20f)) wnee = pdf / (pdf + e.pdf);
      F k = scos * wnee * F(t.alpha) / pdf;
      o_r = F(t.er) * e.r * k;
      o_g = F(t.eg) * e.g * k;
      o_b = F(t.eb) * e.b * k;
      return;
    }
    F sumW = 0;
    F sel_lx = 0, sel_ly = 0, sel_lz = 0;
    F sel_Fr = 0, sel_Fg = 0, sel_Fb = 0, sel_phat = 0, sel_epdf = 0;
    bool have = false;
    for (int j = 0; j < Mc; ++j) {
      F pick = U() * LT;
      const rm_triangle& t = s->tris[pick_light(pick)];
      F lu = U(), lv = U();
      if (lu + lv > F(1)) { lu = F(1) - lu; lv = F(1) - lv; }
      F lw = F(1) - lu - lv;
      F qx = lw * F(t.v0.x) + (lu * F(t.v1.x) + lv * F(t.v2.x));
      F qy = lw * F(t.v0.y) + (lu * F(t.v1.y) + lv * F(t.v2.y));
      F qz = lw * F(t.v0.z) + (lu * F(t.v1.z) + lv * F(t.v2.z));
      F ldx = qx - px, ldy = qy - py, ldz = qz - pz;
      F dist = std::sqrt(ldx * ldx + ldy * ldy + ldz * ldz);
      F w = 0, ph = 0, epdf = 0, Fr = 0, Fg = 0, Fb = 0;
      if (dist > F(0.003f)) {
        F inv = F(1) / dist;
        F dxn = ldx * inv, dyn = ldy * inv, dzn = ldz * inv;
        F lcos = -(F(t.nn.x) * dxn + (F(t.nn.y) * dyn + F(t.nn.z) * dzn));
        F scos = nx * dxn + (ny * dyn + nz * dzn);
        if (lcos > F(1e-8f) && scos > F(1e-8f)) {
          F lt_lum = lum3(F(t.er), F(t.eg), F(t.eb));
          if (lt_lum < F(1e-6f)) lt_lum = F(1e-6f);
          F q = dist * dist * lt_lum / (lcos * LT);
          if (q > F(1e-12f)) {
            Bsdf e = eval_bsdf(dxn, dyn, dzn, wox, woy, woz, nx, ny, nz, alpha2, metallic, spec_prob, ar, ag, ab);
            epdf = e.pdf;
            Fr = F(t.er) * e.r * scos * F(t.alpha);
            Fg = F(t.eg) * e.g * scos * F(t.alpha);
            Fb = F(t.eb) * e.b * scos * F(t.alpha);
            ph = lum3(Fr, Fg, Fb);
            if (ph > F(0)) w = ph / q;
          }
        }
      }
      sumW += w;
      F r = U();
      if (w > F(0) && r * sumW < w) {
        have = true;
        sel_lx = qx; sel_ly = qy; sel_lz = qz;
        sel_Fr = Fr; sel_Fg = Fg; sel_Fb = Fb;
        sel_phat = ph; sel_epdf = epdf;
      }
    }
    out_sumW = sumW;
    out_M = uint32_t(Mc);
    if (!have || !(sumW > F(0)) || !(sel_phat > F(0))) return;
    F pdf_ris = F(float(Mc)) * sel_phat / sumW;
    F wnee = F(1);
    if (!p->nomis && sel_epdf > F(1e-20f)) wnee = pdf_ris / (pdf_ris + sel_epdf);
    F vdx = sel_lx - px, vdy = sel_ly - py, vdz = sel_lz - pz;
    F vdist = std::sqrt(vdx * vdx + vdy * vdy + vdz * vdz);
    if (!(vdist > F(0.003f))) return;
    F vinv = F(1) / vdist;
    vdx *= vinv; vdy *= vinv; vdz *= vinv;
    V3<F> so = mk(px + nx * F(0.002f), py + ny * F(0.002f), pz + nz * F(0.002f));
    if (occluded(so, mk(vdx, vdy, vdz), vdist - F(0.003f))) return;
    F W = sumW / (F(float(Mc)) * sel_phat);
    o_r = sel_Fr * W * wnee;
    o_g = sel_Fg * W * wnee;
    o_b = sel_Fb * W * wnee;
  }

  static F fresnel(F ci_in, F eta_in, F eta_out) {  // pathtrace.metal:80-91
    F ci = ci_in;
    if (ci < F(0)) ci = F(0);
    if (ci > F(1)) ci = F(1);
    F eta = eta_in / eta_out;
    F s2 = eta * eta * (F(1) - ci * ci);
    if (s2 >= F(1)) return F(1);
    F ct = std::sqrt(F(1) - s2);
    F rp = (eta_out * ci - eta_in * ct) / (eta_out * ci + eta_in * ct);
    F rs = (eta_in * ci - eta_out * ct) / (eta_in * ci + eta_out * ct);
    return F(0.5f) * (rp * rp + rs * rs);
  }

  // pathtrace.metal:470-534
  Diel sample_dielectric(F wox, F woy, F woz, F nx, F ny, F nz, F cdx, F cdy, F cdz, F ior,
                         bool front, F rough, F alpha2) {
    Diel out;
    out.valid = true;
    F eta_i = F(1), eta_t = ior;
    if (!front) { eta_i = ior; eta_t = F(1); }
    F hx, hy, hz;
    if (rough <= F(0.0201f)) { hx = nx; hy = ny; hz = nz; }
    else {
      sample_ggx_half(alpha2, nx, ny, nz, hx, hy, hz);
      F md = wox * hx + (woy * hy + woz * hz);
      if (!(md > F(1e-8f))) out.valid = false;
    }
    F cos_m = wox * hx + (woy * hy + woz * hz);
    if (cos_m < F(0)) { hx = -hx; hy = -hy; hz = -hz; cos_m = -cos_m; }
    if (cos_m > F(1)) cos_m = F(1);
    F fres = fresnel(cos_m, eta_i, eta_t);
    F eta = eta_i / eta_t;
    F s2 = eta * eta * (F(1) - cos_m * cos_m);
    if (s2 >= F(1) || U() < fres) {
      out.n_x = F(2) * cos_m * hx - wox;
      out.n_y = F(2) * cos_m * hy - woy;
      out.n_z = F(2) * cos_m * hz - woz;
      out.eta_scale = F(1);
    } else {
      F cos_t = std::sqrt(F(1) - s2);
      out.n_x = eta * cdx + hx * (eta * cos_m - cos_t);
      out.n_y = eta * cdy + hy * (eta * cos_m - cos_t);
      out.n_z = eta * cdz + hz * (eta * cos_m - cos_t);
      out.eta_scale = eta * eta;
    }
    {
      F d = F(1) / std::sqrt(out.n_x * out.n_x + out.n_y * out.n_y + out.n_z * out.n_z);
      out.n_x *= d; out.n_y *= d; out.n_z *= d;
    }
    if (rough > F(0.0201f)) {
      F cos_i = std::fabs(out.n_x * nx + (out.n_y * ny + out.n_z * nz));
      F cos_o = std::fabs(wox * nx + (woy * ny + woz * nz));
      F cos_h = std::fabs(hx * nx + (hy * ny + hz * nz));
      F vo_h = std::fabs(wox * hx + (woy * hy + woz * hz));
      if (cos_i > F(1e-8f) && cos_o > F(1e-8f) && cos_h > F(1e-8f) && vo_h > F(1e-8f)) {
        F g1 = F(2) * cos_o / (cos_o + std::sqrt(cos_o * cos_o + alpha2 * (F(1) - cos_o * cos_o)));
        F g2 = F(2) * cos_i / (cos_i + std::sqrt(cos_i * cos_i + alpha2 * (F(1) - cos_i * cos_i)));
        F w = g1 * g2 * vo_h / (cos_o * cos_h);
        if (w > F(10)) w = F(10);
        out.eta_scale *= w;
      } else {
        out.valid = false;
      }
    }
    return out;
  }

  // pathtrace.metal:536-550 (stochastic coverage; crossings capped).
  Hit<F> cast_alpha_ray(V3<F> ro, V3<F> rd, F dist) {
    if (p->opaque) return cast_ray(ro, rd, dist);
    F traveled = 0;
    for (int it = 0; it < kMaxAlphaCrossings && traveled < dist; ++it) {
      Hit<F> h = cast_ray(mk(ro.x + rd.x * traveled, ro.y + rd.y * traveled, ro.z + rd.z * traveled), rd,
                          dist - traveled);
      if (h.tri < 0) return h;
      F opacity = F(s->tris[h.tri].alpha);
      if (opacity >= F(1) || (opacity > F(0) && U() < opacity)) {
        h.t += traveled;
        return h;
      }
      traveled += h.t + F(0.0001f);
    }
    return Hit<F>{};
  }

  // pathtrace.metal:552-728: one path sample from (ro, rd).
  V3<F> pathtrace(V3<F> ro, V3<F> rd, int max_bounces) {
    F ox = ro.x, oy = ro.y, oz = ro.z, dx = rd.x, dy = rd.y, dz = rd.z;
    F accr = 0, accg = 0, accb = 0, thr_r = 1, thr_g = 1, thr_b = 1;
    int bounce = 0, prev_delta = 1;
    F last_pdf = 0, prev_sumW = 0;
    uint32_t prev_M = 0;
    F prev_br = 0, prev_bg = 0, prev_bb = 0, prev_cos = 0;
    const F LT = F(p->light_total);
    for (int b = 0; b < max_bounces; ++b) {
      Hit<F> hit = cast_alpha_ray(mk(ox, oy, oz), mk(dx, dy, dz), F(1e30f));
      if (hit.tri < 0) break;
      F pnx = hit.n_interp.x, pny = hit.n_interp.y, pnz = hit.n_interp.z;
      F geom = hit.n_geom.x * pnx + (hit.n_geom.y * pny + hit.n_geom.z * pnz);
      if (geom < F(0)) { pnx = -pnx; pny = -pny; pnz = -pnz; }
      F ndot = dx * pnx + (dy * pny + dz * pnz);
      bool front = true;
      if (ndot > F(0)) { pnx = -pnx; pny = -pny; pnz = -pnz; front = false; }
      F wox = -dx, woy = -dy, woz = -dz;
      F rough = hit.rough;
      if (rough < F(0)) rough = F(0);
      if (rough > F(1)) rough = F(1);
      if (rough < F(0.02f)) rough = F(0.02f);
      F alpha = rough * rough;
      F alpha2 = alpha * alpha;
      const rm_triangle& lt = s->tris[hit.tri];
      F metallic = F(lt.metallic);
      if (metallic < F(0)) metallic = F(0);
      if (metallic > F(1)) metallic = F(1);
      if (bounce == 0 || prev_delta == 1) {
        accr += hit.er * thr_r; accg += hit.eg * thr_g; accb += hit.eb * thr_b;
      } else {
        F lx = hit.p.x - ox, ly = hit.p.y - oy, lz = hit.p.z - oz;
        F dist2 = lx * lx + ly * ly + lz * lz;
        F dist = std::sqrt(dist2);
        F pl = F(1e30f);
        if (dist > F(1e-20f) && last_pdf > F(1e-20f) && prev_M > 0 && prev_sumW > F(1e-20f)) {
          F ph = lum3(hit.er * prev_br * prev_cos * F(lt.alpha), hit.eg * prev_bg * prev_cos * F(lt.alpha),
                      hit.eb * prev_bb * prev_cos * F(lt.alpha));
          if (ph > F(1e-20f)) pl = F(float(prev_M)) * ph / prev_sumW;
          else {
            F inv = F(1) / dist;
            F lxn = lx * inv, lyn = ly * inv, lzn = lz * inv;
            F cos_l = -(F(lt.nn.x) * lxn + (F(lt.nn.y) * lyn + F(lt.nn.z) * lzn));
            if (cos_l > F(1e-8f)) {
              F lum = lum3(F(lt.er), F(lt.eg), F(lt.eb));
              if (lum < F(1e-6f)) lum = F(1e-6f);
              pl = dist2 * lum / (cos_l * LT);
            }
          }
        } else if (dist > F(1e-20f) && last_pdf > F(1e-20f)) {
          F inv = F(1) / dist;
          lx *= inv; ly *= inv; lz *= inv;
          F cos_l = -(F(lt.nn.x) * lx + (F(lt.nn.y) * ly + F(lt.nn.z) * lz));
          if (cos_l > F(1e-8f)) {
            F lum = lum3(F(lt.er), F(lt.eg), F(lt.eb));
            if (lum < F(1e-6f)) lum = F(1e-6f);
            pl = dist2 * lum / (cos_l * LT);
          }
        }
        F w = p->nomis ? F(0) : ((last_pdf + pl > F(1e-20f)) ? last_pdf / (last_pdf + pl) : F(0));
        accr += hit.er * thr_r * w; accg += hit.eg * thr_g * w; accb += hit.eb * thr_b * w;
      }
      if (hit.ior > F(1.0001f)) {
        Diel ds = sample_dielectric(wox, woy, woz, pnx, pny, pnz, dx, dy, dz, hit.ior, front, rough, alpha2);
        if (!ds.valid) break;
        thr_r *= ds.eta_scale; thr_g *= ds.eta_scale; thr_b *= ds.eta_scale;
        F sg = F(1);
        if (ds.n_x * pnx + (ds.n_y * pny + ds.n_z * pnz) < F(0)) sg = F(-1);
        ox = hit.p.x + pnx * F(0.001f) * sg;
        oy = hit.p.y + pny * F(0.001f) * sg;
        oz = hit.p.z + pnz * F(0.001f) * sg;
        dx = ds.n_x; dy = ds.n_y; dz = ds.n_z;
        prev_delta = 1;
        prev_sumW = 0; prev_M = 0;
      } else {
        F spec_prob = F(0.05f) + F(0.95f) * metallic;
        if (spec_prob > F(0.98f)) spec_prob = F(0.98f);
        if (metallic >= F(0.999f)) spec_prob = F(1);
        F cur_sumW = 0;
        uint32_t cur_M = 0;
        {
          F dlr, dlg, dlb;
          direct_lighting(hit.p.x, hit.p.y, hit.p.z, pnx, pny, pnz, wox, woy, woz, rough, metallic,
                          spec_prob, hit.ar, hit.ag, hit.ab, dlr, dlg, dlb, cur_sumW, cur_M);
          accr += dlr * thr_r; accg += dlg * thr_g; accb += dlb * thr_b;
        }
        F nx2, ny2, nz2;
        if (U() < spec_prob) {
          F hx, hy, hz;
          sample_ggx_half(alpha2, pnx, pny, pnz, hx, hy, hz);
          F md = wox * hx + (woy * hy + woz * hz);
          if (!(md > F(1e-8f))) break;
          nx2 = F(2) * md * hx - wox;
          ny2 = F(2) * md * hy - woy;
          nz2 = F(2) * md * hz - woz;
          prev_delta = (rough <= F(0.0201f)) ? 1 : 0;
        } else {
          sample_cosine(pnx, pny, pnz, nx2, ny2, nz2);
          prev_delta = 0;
        }
        F ncos = nx2 * pnx + (ny2 * pny + nz2 * pnz);
        if (!(ncos > F(1e-8f))) break;
        {
          F d = F(1) / std::sqrt(nx2 * nx2 + ny2 * ny2 + nz2 * nz2);
          nx2 *= d; ny2 *= d; nz2 *= d;
        }
        Bsdf e = eval_bsdf(nx2, ny2, nz2, wox, woy, woz, pnx, pny, pnz, alpha2, metallic, spec_prob,
                           hit.ar, hit.ag, hit.ab);
        if (!(e.pdf > F(1e-12f))) break;
        last_pdf = e.pdf;
        F cos_i = nx2 * pnx + (ny2 * pny + nz2 * pnz);
        thr_r *= e.r * cos_i / e.pdf;
        thr_g *= e.g * cos_i / e.pdf;
        thr_b *= e.b * cos_i / e.pdf;
        prev_sumW = cur_sumW; prev_M = cur_M;
        prev_br = e.r; prev_bg = e.g; prev_bb = e.b; prev_cos = cos_i;
        ox = hit.p.x + pnx * F(0.001f);
        oy = hit.p.y + pny * F(0.001f);
        oz = hit.p.z + pnz * F(0.001f);
        dx = nx2; dy = ny2; dz = nz2;
      }
      if (thr_r < F(0)) thr_r = F(0);
      if (thr_g < F(0)) thr_g = F(0);
      if (thr_b < F(0)) thr_b = F(0);
      F mx = std::max(thr_r, thr_g);
      mx = std::max(mx, thr_b);
      if (!(mx >= F(1e-12f))) break;
      if (p->rr && bounce >= 1) {
        F rr = mx;
        if (rr < F(0.05f)) rr = F(0.05f);
        if (rr > F(0.9f)) rr = F(0.9f);
        if (!(U() <= rr)) break;
        F ir = F(1) / rr;
        thr_r *= ir; thr_g *= ir; thr_b *= ir;
      }
      bounce++;
    }
    return mk(accr, accg, accb);
  }

  // pathtrace.metal:729-737
  V3<F> sample_sensor(F sx, F sy, const rm_camera& cam, F focal2, int max_bounces) {
    F dist = F(1) / std::sqrt(sx * sx + (sy * sy + focal2));
    F tx = sx * dist, ty = sy * dist, tz = F(cam.focal) * dist;
    V3<F> rd = mk(tx * F(cam.m0) + (ty * F(cam.m1) + tz * F(cam.m2)),
                  tx * F(cam.m3) + (ty * F(cam.m4) + tz * F(cam.m5)),
                  tx * F(cam.m6) + (ty * F(cam.m7) + tz * F(cam.m8)));
    return pathtrace(mk(F(cam.x), F(cam.y), F(cam.z)), rd, max_bounces);
  }

  // Jittered sensor coordinates, pathtrace.metal:754-755.
  void jitter(uint32_t x, uint32_t y, F& sx, F& sy) {
    const F res = F(p->resolution);
    sx = F(float(x)) + F(1e-12f) + (res - F(2e-12f)) * U() - F(float(p->width)) * F(0.5f);
    sy = F(float(p->height)) * F(0.5f) - (F(float(y)) + F(1e-12f) + (res - F(2e-12f)) * U());
  }
};

// Seeds of the kernels (pathtrace.metal:751, :787, :829, :937, :1069).
inline uint64_t seed_pixel(uint64_t seed, uint32_t x, uint32_t y) {
  return seed ^ (uint64_t(y + 1) * 0x9E3779B97F4A7C15ull) ^ (uint64_t(x + 1) * 0xBF58476D1CE4E5B9ull);
}
inline uint64_t seed_lane(uint64_t seed, uint32_t x, uint32_t y, uint32_t lane) {
  return seed_pixel(seed, x, y) ^ (uint64_t(lane) * 0x94D049BB133111EBull);
}
inline uint64_t seed_spatial(uint64_t seed, uint32_t id) {
  return seed ^ (uint64_t(id + 1) * 0x9E3779B97F4A7C15ull) ^ kSpatialSeedXor;
}
inline uint64_t seed_shade(uint64_t seed, uint32_t id) {
  return seed ^ (uint64_t(id + 1) * 0xBF58476D1CE4E5B9ull) ^ 0x94D049BB133111EBull;
}

template <class F> inline uint8_t tonemap8(F c) {  // pathtrace.metal:767
  F v = std::floor(c / (c + F(1)) * F(255));
  v = std::fmin(std::fmax(v, F(0)), F(255));
  return uint8_t(v);
}

}  // namespace orc
