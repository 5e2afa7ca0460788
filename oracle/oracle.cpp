// oracle.cpp - frame-level CPU oracle and its C entry points (ctypes).
//
// TEST INFRASTRUCTURE ONLY: used by tests/, the smoke check and the benchmark's
// CPU-baseline leg as the checker.  Never linked into librmcuda.so.
//
// Restates, on the CPU:
//  * the reference's host policy for one frame, render_image_metal
//    (src/engine/metal.mm:95-414): validation, parameter resolution and the
//    environment switches, preorder escape-link BVH conversion, lane choice,
//    ReSTIR eligibility, scene hash and temporal history;
//  * the nine Metal kernels (src/engine/pathtrace.metal:739-1363);
//  * the reference CPU BVH builder and refit (src/engine/bvh.cpp:29-272) in
//    fp64, which produce the BVH the oracle traverses.
#include <atomic>
#include <limits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <queue>
#include <string>
#include <thread>

#include "oracle_core.hpp"

namespace orc {
namespace {

void set_err(char* err, size_t cap, const std::string& msg) {
  if (err && cap) { std::snprintf(err, cap, "%s", msg.c_str()); }
}

template <class Fn> void parallel_for(int n, int nthreads, Fn fn) {
  if (nthreads <= 1 || n <= 1) {
    for (int i = 0; i < n; ++i) fn(i);
    return;
  }
  std::atomic<int> next{0};
  std::vector<std::thread> pool;
  int T = std::min(nthreads, n);
  for (int t = 0; t < T; ++t)
    pool.emplace_back([&] {
      for (;;) {
        int i = next.fetch_add(1);
        if (i >= n) break;
        fn(i);
      }
    });
  for (auto& th : pool) th.join();
}

// metal.mm:129-144: DFS from the root; each node records the index following
// its subtree as the escape link.
std::vector<PNode> to_preorder(const rm_bvh_node* nodes, int n_nodes) {
  std::vector<PNode> out;
  if (!nodes || n_nodes <= 0) return out;
  out.reserve(size_t(n_nodes));
  std::vector<std::pair<int, bool>> todo;
  todo.emplace_back(0, false);
  while (!todo.empty()) {
    auto [index, leaving] = todo.back();
    todo.pop_back();
    if (leaving) { out[size_t(index)].escape = int(out.size()); continue; }
    const rm_bvh_node& s = nodes[index];
    int dest = int(out.size());
    PNode t{};
    t.mn[0] = s.mn.x; t.mn[1] = s.mn.y; t.mn[2] = s.mn.z;
    t.mx[0] = s.mx.x; t.mx[1] = s.mx.y; t.mx[2] = s.mx.z;
    t.offset = s.offset; t.count = s.count;
    out.push_back(t);
    todo.emplace_back(dest, true);
    if (s.count <= 0) { todo.emplace_back(s.right, false); todo.emplace_back(s.left, false); }
  }
  return out;
}

struct Env {
  bool noadapt = false, nomis = false, restir_off = false, denoise_off = false, temporal_off = false;
  bool have_cand = false, have_spatial = false;
  int cand = 0, spatial = 0;
};

Env read_env(uint32_t flags) {
  Env e;
  if (flags & RM_FLAG_NO_ENV) {
    e.noadapt = flags & RM_FLAG_NOADAPT;
    e.nomis = flags & RM_FLAG_NOMIS;
    e.restir_off = flags & RM_FLAG_RESTIR_OFF;
    e.denoise_off = flags & RM_FLAG_DENOISE_OFF;
    e.temporal_off = flags & RM_FLAG_TEMPORAL_OFF;
    return e;
  }
  e.noadapt = std::getenv("UOW2_NOADAPT") != nullptr;
  e.nomis = std::getenv("UOW2_NOMIS") != nullptr;
  const char* r = std::getenv("RAYMOTION_RESTIR");
  e.restir_off = r && std::string(r) == "0";
  const char* d = std::getenv("RAYMOTION_DENOISE");
  e.denoise_off = d && std::string(d) == "0";
  const char* tv = std::getenv("RAYMOTION_RESTIR_TEMPORAL");
  e.temporal_off = tv && std::string(tv) == "0";
  if (const char* v = std::getenv("RAYMOTION_RESTIR_CANDIDATES")) { e.have_cand = true; e.cand = std::atoi(v); }
  if (const char* v = std::getenv("RAYMOTION_RESTIR_SPATIAL")) { e.have_spatial = true; e.spatial = std::atoi(v); }
  return e;
}

// metal.mm:146-170
Params resolve(const rm_config& c, const rm_camera& cam, int n_nodes, int n_lights, float light_total,
               bool opaque, const Env& env) {
  Params p{};
  p.camera = cam;
  p.width = c.width; p.height = c.height; p.spp = c.spp; p.bounces = c.max_bounces;
  p.nodes = n_nodes; p.lights = n_lights; p.light_total = light_total;
  p.resolution = c.resolution; p.clamp_value = c.clamp; p.adapt_rel = c.adapt_rel; p.adapt_abs = c.adapt_abs;
  p.adapt_min = env.noadapt ? 0 : c.adapt_min;
  p.adapt_step = c.adapt_step > 0 ? c.adapt_step : 8;
  p.opaque = opaque ? 1 : 0;
  p.nomis = env.nomis ? 1 : 0;
  p.restir_candidates = env.restir_off ? 1 : (c.restir_candidates > 0 ? c.restir_candidates : 1);
  if (p.restir_candidates < 1) p.restir_candidates = 1;
  if (p.restir_candidates > 32) p.restir_candidates = 32;
  p.restir_spatial = env.restir_off ? 0 : (c.restir_spatial > 0 ? c.restir_spatial : 0);
  if (p.restir_spatial < 0) p.restir_spatial = 0;
  if (p.restir_spatial > 8) p.restir_spatial = 8;
  p.restir_mcap = c.restir_mcap > 0 ? c.restir_mcap : 128;
  if (p.restir_mcap < 1) p.restir_mcap = 1;
  p.restir_radius = c.restir_radius > 0 ? c.restir_radius : 16.0f;
  if (env.have_cand) p.restir_candidates = std::max(1, env.cand);
  if (env.have_spatial) p.restir_spatial = std::max(0, env.spatial);
  p.rr = (c.flags & RM_FLAG_NO_RR) ? 0 : 1;
  return p;
}

// Scene hash guarding temporal reuse (metal.mm:241-248): FNV-1a style over
// the packed triangle bytes, seeded with the counts and light_total bits.
uint64_t scene_hash(const rm_triangle* tris, int n, int n_lights, float light_total) {
  uint32_t lt_bits;
  std::memcpy(&lt_bits, &light_total, 4);
  uint64_t h = uint64_t(n) * 0x9E3779B97F4A7C15ull ^ uint64_t(n_lights) * 0xBF58476D1CE4E5B9ull ^
               (uint64_t(lt_bits) * 0x94D049BB133111EBull);
  const unsigned char* b = reinterpret_cast<const unsigned char*>(tris);
  for (size_t i = 0, m = size_t(n) * sizeof(rm_triangle); i < m; ++i) {
    h ^= uint64_t(b[i]);
    h *= 0x100000001B3ull;
  }
  return h;
}

struct Reproj { bool ok; uint32_t hidx; };
// Reprojection into the previous camera (pathtrace.metal:957-966, :1287-1297).
inline Reproj reproject(const Params& p, float cx, float cy, float cz) {
  const rm_camera& pc = p.prevCamera;
  float pdx = cx - pc.x, pdy = cy - pc.y, pdz = cz - pc.z;
  float ccx = pc.m0 * pdx + pc.m3 * pdy + pc.m6 * pdz;
  float ccy = pc.m1 * pdx + pc.m4 * pdy + pc.m7 * pdz;
  float ccz = pc.m2 * pdx + pc.m5 * pdy + pc.m8 * pdz;
  Reproj r{false, 0};
  if (!(ccz > 1e-6f)) return r;
  float ppx = pc.focal * ccx / ccz + float(p.width) * 0.5f;
  float ppy = float(p.height) * 0.5f - pc.focal * ccy / ccz;
  // int(floor(v)) in [0, n) <=> 0 <= v < n (also rejects NaN and huge values)
  if (!(ppx >= 0.0f && ppx < float(p.width) && ppy >= 0.0f && ppy < float(p.height))) return r;
  int hx = int(std::floor(ppx)), hy = int(std::floor(ppy));
  r.ok = true;
  r.hidx = uint32_t(hy) * uint32_t(p.width) + uint32_t(hx);
  return r;
}

inline float luma(float r, float g, float b) { return 0.2126f * r + 0.7152f * g + 0.0722f * b; }

}  // namespace

struct Ctx {
  // temporal history (metal.mm:35-40)
  std::vector<GBuf> hist_g;
  std::vector<Reservoir> hist_r;
  std::vector<float> hist_col;
  rm_camera hist_cam{};
  int hist_w = 0, hist_h = 0;
  uint64_t hist_seed = 0, hist_hash = 0;
  bool hist_valid = false, have_hist_bufs = false;
  // last frame (debug reads)
  std::vector<GBuf> g;
  std::vector<Reservoir> rinit, rmerged;
  std::vector<float> hdr;
  std::vector<uint32_t> dbg;  // per pixel: xor of final RNG states, samples taken
  uint64_t samples = 0, rays = 0;
  int chain = 0;
};

// ---------------------------------------------------------------- kernels

// K1 render_paths (pathtrace.metal:739-769) and K2 render_paths_simd
// (:773-815) for `lanes` in {1, 8, 32}; writes linear radiance to hdr.
static void k_render_paths(const SceneRef& s, const Params& p, uint64_t seed, int lanes, int row0, int row1,
                           float* hdr, uint32_t* dbg, int nthreads, std::atomic<uint64_t>& samples,
                           std::atomic<uint64_t>& rays) {
  const int W = p.width;
  parallel_for(row1 - row0, nthreads, [&](int ry) {
    uint32_t y = uint32_t(row0 + ry);
    Counters ctr;
    uint64_t taken = 0;
    for (uint32_t x = 0; x < uint32_t(W); ++x) {
      size_t id = size_t(y) * size_t(W) + x;
      float sum[3] = {0, 0, 0};
      float sum_l = 0, sum_l2 = 0;
      int n = 0;
      uint32_t rng_xor = 0;
      if (lanes == 1) {
        Tracer<float> pt{&s, &p, Rng{}, &ctr};
        pt.rng.seed(seed_pixel(seed, x, y));
        for (int si = 0; si < p.spp; ++si) {
          float sx, sy;
          pt.jitter(x, y, sx, sy);
          V3<float> c = pt.sample_sensor(sx, sy, p.camera, p.camera.focal * p.camera.focal, p.bounces);
          if (p.clamp_value > 0) {
            c.x = std::fmin(c.x, p.clamp_value); c.y = std::fmin(c.y, p.clamp_value); c.z = std::fmin(c.z, p.clamp_value);
          }
          sum[0] += c.x; sum[1] += c.y; sum[2] += c.z;
          ++n;
          if (p.adapt_min > 0) {
            float lum = c.x * 0.2126f + c.y * 0.7152f + c.z * 0.0722f;
            sum_l += lum; sum_l2 += lum * lum;
            if (n >= p.adapt_min && n > 1 && n % p.adapt_step == 0) {
              float mean = sum_l / float(n);
              float var = std::max(0.0f, (sum_l2 - sum_l * mean) / float(n - 1));
              float thr = p.adapt_rel * mean + p.adapt_abs;
              if (var < thr * thr) break;
            }
          }
        }
        taken += uint64_t(n);
        rng_xor = pt.rng.state;
      } else {
        std::vector<Tracer<float>> lt(size_t(lanes), Tracer<float>{&s, &p, Rng{}, &ctr});
        for (int l = 0; l < lanes; ++l) lt[size_t(l)].rng.seed(seed_lane(seed, x, y, uint32_t(l)));
        const size_t L = static_cast<size_t>(lanes);
        std::vector<float> cr(L), cg(L), cb(L), lm(L), lm2(L);
        for (uint32_t base = 0; base < uint32_t(p.spp); base += uint32_t(lanes)) {
          for (int l = 0; l < lanes; ++l) {
            float c3[3] = {0, 0, 0};
            if (base + uint32_t(l) < uint32_t(p.spp)) {
              Tracer<float>& pt = lt[size_t(l)];
              float sx, sy;
              pt.jitter(x, y, sx, sy);
              V3<float> c = pt.sample_sensor(sx, sy, p.camera, p.camera.focal * p.camera.focal, p.bounces);
              if (p.clamp_value > 0) {
                c.x = std::fmin(c.x, p.clamp_value); c.y = std::fmin(c.y, p.clamp_value); c.z = std::fmin(c.z, p.clamp_value);
              }
              c3[0] = c.x; c3[1] = c.y; c3[2] = c.z;
              taken++;
            }
            cr[size_t(l)] = c3[0]; cg[size_t(l)] = c3[1]; cb[size_t(l)] = c3[2];
            float lum = c3[0] * 0.2126f + c3[1] * 0.7152f + c3[2] * 0.0722f;
            lm[size_t(l)] = lum; lm2[size_t(l)] = lum * lum;
          }
          // butterfly (simd_shuffle_xor) sums, pathtrace.metal:799-803
          for (int mask = 1; mask < lanes; mask *= 2) {
            std::vector<float> a = cr, b = cg, c = cb, d = lm, e = lm2;
            for (int l = 0; l < lanes; ++l) {
              size_t o = size_t(l ^ mask), i = size_t(l);
              cr[i] = a[i] + a[o]; cg[i] = b[i] + b[o]; cb[i] = c[i] + c[o];
              lm[i] = d[i] + d[o]; lm2[i] = e[i] + e[o];
            }
          }
          sum[0] += cr[0]; sum[1] += cg[0]; sum[2] += cb[0];
          sum_l += lm[0]; sum_l2 += lm2[0];
          n = int(std::min(base + uint32_t(lanes), uint32_t(p.spp)));
          if (p.adapt_min > 0 && n >= p.adapt_min && n > 1 && n % p.adapt_step == 0) {
            float mean = sum_l / float(n);
            float var = std::max(0.0f, (sum_l2 - sum_l * mean) / float(n - 1));
            float thr = p.adapt_rel * mean + p.adapt_abs;
            if (var < thr * thr) break;
          }
        }
        for (int l = 0; l < lanes; ++l) rng_xor ^= lt[size_t(l)].rng.state;
      }
      hdr[id * 3 + 0] = sum[0] / float(n);
      hdr[id * 3 + 1] = sum[1] / float(n);
      hdr[id * 3 + 2] = sum[2] / float(n);
      if (dbg) { dbg[id * 2] = rng_xor; dbg[id * 2 + 1] = uint32_t(n); }
    }
    samples += taken;
    rays += ctr.rays;
  });
}

// K3 restir_generate (pathtrace.metal:817-917)
static void k_generate(const SceneRef& s, const Params& p, uint64_t seed, int row0, int row1, GBuf* gb,
                       Reservoir* ri, int nthreads, std::atomic<uint64_t>& rays, int32_t* rl = nullptr) {
  const int W = p.width;
  parallel_for(row1 - row0, nthreads, [&](int ry) {
    uint32_t y = uint32_t(row0 + ry);
    Counters ctr;
    for (uint32_t x = 0; x < uint32_t(W); ++x) {
      size_t id = size_t(y) * size_t(W) + x;
      Tracer<float> pt{&s, &p, Rng{}, &ctr};
      pt.rng.seed(seed_pixel(seed, x, y));
      GBuf& g = gb[id];
      Reservoir& r = ri[id];
      g.kind = 0;
      r.valid = 0;
      if (rl) rl[id] = -1;  // the selected light's triangle (the adjoint's check), or -1
      float sx = float(x) + 1e-12f + (p.resolution - 2e-12f) * pt.U() - float(p.width) * 0.5f;
      float sy = float(p.height) * 0.5f - (float(y) + 1e-12f + (p.resolution - 2e-12f) * pt.U());
      float f2 = p.camera.focal * p.camera.focal;
      float dinv = 1.0f / std::sqrt(sx * sx + sy * sy + f2);
      float tx = sx * dinv, ty = sy * dinv, tz = p.camera.focal * dinv;
      const rm_camera& c = p.camera;
      V3<float> rd = mk(tx * c.m0 + (ty * c.m1 + tz * c.m2), tx * c.m3 + (ty * c.m4 + tz * c.m5),
                        tx * c.m6 + (ty * c.m7 + tz * c.m8));
      V3<float> ro = mk(c.x, c.y, c.z);
      Hit<float> hit = pt.cast_alpha_ray(ro, rd, 1e30f);
      if (hit.tri < 0) continue;
      float pnx = hit.n_interp.x, pny = hit.n_interp.y, pnz = hit.n_interp.z;
      float geom = hit.n_geom.x * pnx + (hit.n_geom.y * pny + hit.n_geom.z * pnz);
      if (geom < 0) { pnx = -pnx; pny = -pny; pnz = -pnz; }
      float ndot = rd.x * pnx + (rd.y * pny + rd.z * pnz);
      if (ndot > 0) { pnx = -pnx; pny = -pny; pnz = -pnz; }
      float wox = -rd.x, woy = -rd.y, woz = -rd.z;
      float rough = hit.rough; if (rough < 0) rough = 0; if (rough > 1) rough = 1;
      float metallic = s.tris[hit.tri].metallic; if (metallic < 0) metallic = 0; if (metallic > 1) metallic = 1;
      g.pos = {hit.p.x, hit.p.y, hit.p.z};
      g.normal = {pnx, pny, pnz};
      g.albedo = {hit.ar, hit.ag, hit.ab};
      g.wo = {wox, woy, woz};
      g.emission = {hit.er, hit.eg, hit.eb};
      g.rough = rough; g.metallic = metallic;
      if (hit.ior > 1.0001f) { g.ior = hit.ior; g.kind = 3; continue; }
      g.ior = 1; g.kind = 1;
      if (p.lights == 0 || !(p.light_total > 1e-12f)) continue;
      int Mc = p.restir_candidates; if (Mc < 1) Mc = 1; if (Mc > 32) Mc = 32;
      float r2 = rough; if (r2 < 0.02f) r2 = 0.02f;
      float alpha2 = (r2 * r2) * (r2 * r2);
      float spec_prob = 0.05f + 0.95f * metallic; if (spec_prob > 0.98f) spec_prob = 0.98f;
      if (metallic >= 0.999f) spec_prob = 1.0f;
      float px = hit.p.x, py = hit.p.y, pz = hit.p.z;
      float sumWs = 0, sumWu = 0, sel_lx = 0, sel_ly = 0, sel_lz = 0, sel_nx = 0, sel_ny = 0, sel_nz = 0;
      float sel_er = 0, sel_eg = 0, sel_eb = 0, sel_alpha = 1, sel_ph = 0;
      int sel_tri = -1;
      bool have = false;
      V3<float> so = mk(px + pnx * 0.002f, py + pny * 0.002f, pz + pnz * 0.002f);
      for (int j = 0; j < Mc; ++j) {
        float pick = pt.U() * p.light_total;
        const int ltri = pt.pick_light(pick);
        const rm_triangle& t = s.tris[ltri];
        float lu = pt.U(), lv = pt.U();
        if (lu + lv > 1.0f) { lu = 1.0f - lu; lv = 1.0f - lv; }
        float lw = 1.0f - lu - lv;
        float qx = lw * t.v0.x + (lu * t.v1.x + lv * t.v2.x);
        float qy = lw * t.v0.y + (lu * t.v1.y + lv * t.v2.y);
        float qz = lw * t.v0.z + (lu * t.v1.z + lv * t.v2.z);
        float ldx = qx - px, ldy = qy - py, ldz = qz - pz;
        float dist = std::sqrt(ldx * ldx + ldy * ldy + ldz * ldz);
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
              auto e = Tracer<float>::eval_bsdf(dxn, dyn, dzn, wox, woy, woz, pnx, pny, pnz, alpha2, metallic,
                                                spec_prob, hit.ar, hit.ag, hit.ab);
              float Fr = t.er * e.r * scos * t.alpha, Fg = t.eg * e.g * scos * t.alpha, Fb = t.eb * e.b * scos * t.alpha;
              ph = lum3(Fr, Fg, Fb);
              if (ph > 0) {
                wu = ph / q;
                bool occ = pt.occluded(so, mk(dxn, dyn, dzn), dist - 0.003f);
                if (!occ) ws = wu;
              }
            }
          }
        }
        sumWu += wu; sumWs += ws;
        float r = pt.U();
        if (ws > 0 && r * sumWs < ws) {
          have = true;
          sel_lx = qx; sel_ly = qy; sel_lz = qz;
          sel_nx = t.nn.x; sel_ny = t.nn.y; sel_nz = t.nn.z;
          sel_er = t.er; sel_eg = t.eg; sel_eb = t.eb; sel_alpha = t.alpha; sel_ph = ph;
          sel_tri = ltri;
        }
      }
      if (!have || !(sumWs > 0) || !(sumWu > 0) || !(sel_ph > 0)) continue;
      r.lightPos = {sel_lx, sel_ly, sel_lz};
      r.lightNormal = {sel_nx, sel_ny, sel_nz};
      r.emission = {sel_er, sel_eg, sel_eb};
      r.alpha = sel_alpha; r.p_hat = sel_ph; r.sumWs = sumWs; r.sumWu = sumWu; r.M = uint32_t(Mc); r.valid = 1;
      if (rl) rl[id] = sel_tri;
    }
    rays += ctr.rays;
  });
}

// K4 restir_spatial (pathtrace.metal:919-1054)
static void k_spatial(const SceneRef& s, const Params& p, uint64_t seed, int row0, int row1, const GBuf* gb,
                      const Reservoir* ri, Reservoir* ro_, const GBuf* hg, const Reservoir* hr, int nthreads,
                      std::atomic<uint64_t>& rays, const int32_t* ril = nullptr, int32_t* rol = nullptr,
                      const int32_t* hrl = nullptr) {
  const int W = p.width, H = p.height;
  parallel_for(row1 - row0, nthreads, [&](int ry) {
    uint32_t y = uint32_t(row0 + ry);
    Counters ctr;
    for (uint32_t x = 0; x < uint32_t(W); ++x) {
      uint32_t id = y * uint32_t(W) + x;
      ro_[id] = ri[id];
      if (rol) rol[id] = ril ? ril[id] : -1;  // the selected light's triangle follows the sample
      if (gb[id].kind != 1 || ri[id].valid == 0) continue;
      int S = p.restir_spatial; if (S < 0) S = 0; if (S > 8) S = 8;
      if (S == 0) continue;
      float radius = p.restir_radius; if (!(radius > 0)) radius = 16;
      int mcap = p.restir_mcap; if (mcap < 1) mcap = 1;
      Tracer<float> pt{&s, &p, Rng{}, &ctr};
      pt.rng.seed(seed_spatial(seed, id));
      const GBuf& g = gb[id];
      V3<float> cpos = vf<float>(g.pos), cnor = vf<float>(g.normal), cwo = vf<float>(g.wo), calb = vf<float>(g.albedo);
      float rough = g.rough; if (rough < 0) rough = 0; if (rough > 1) rough = 1;
      float metallic = g.metallic; if (metallic < 0) metallic = 0; if (metallic > 1) metallic = 1;
      float r2 = rough; if (r2 < 0.02f) r2 = 0.02f;
      float alpha2 = (r2 * r2) * (r2 * r2);
      float spec_prob = 0.05f + 0.95f * metallic; if (spec_prob > 0.98f) spec_prob = 0.98f;
      if (metallic >= 0.999f) spec_prob = 1.0f;
      const Reservoir& R = ri[id];
      float cur_sumWs = R.sumWs, cur_sumWu = R.sumWu;
      uint32_t cur_M = R.M;
      float cur_ph = R.p_hat;
      rm_vec3 cur_lp = R.lightPos, cur_ln = R.lightNormal, cur_le = R.emission;
      float cur_alpha = R.alpha;
      int cur_l = ril ? ril[id] : -1;
      auto eval_at = [&](const rm_vec3& lp, const rm_vec3& ln, const rm_vec3& le, float la, float& ph_out,
                         float& dist_out, V3<float>& dn_out) -> bool {
        float ldx = lp.x - cpos.x, ldy = lp.y - cpos.y, ldz = lp.z - cpos.z;
        float dist = std::sqrt(ldx * ldx + ldy * ldy + ldz * ldz);
        dist_out = dist;
        if (!(dist > 0.003f)) return false;
        float inv = 1.0f / dist;
        float dxn = ldx * inv, dyn = ldy * inv, dzn = ldz * inv;
        float lcos = -(ln.x * dxn + (ln.y * dyn + ln.z * dzn));
        float scos = cnor.x * dxn + (cnor.y * dyn + cnor.z * dzn);
        if (!(lcos > 1e-8f && scos > 1e-8f)) return false;
        auto e = Tracer<float>::eval_bsdf(dxn, dyn, dzn, cwo.x, cwo.y, cwo.z, cnor.x, cnor.y, cnor.z, alpha2, metallic,
                                          spec_prob, calb.x, calb.y, calb.z);
        float Fr = le.x * e.r * scos * la, Fg = le.y * e.g * scos * la, Fb = le.z * e.b * scos * la;
        ph_out = lum3(Fr, Fg, Fb);
        dn_out = mk(dxn, dyn, dzn);
        return true;
      };
      if (p.hasHistory != 0) {
        Reproj rp = reproject(p, cpos.x, cpos.y, cpos.z);
        if (rp.ok) {
          const GBuf& hgb = hg[rp.hidx];
          const Reservoir& hrr = hr[rp.hidx];
          if (hgb.kind == 1 && hrr.valid != 0) {
            float ddx = cpos.x - hgb.pos.x, ddy = cpos.y - hgb.pos.y, ddz = cpos.z - hgb.pos.z;
            float dd = std::sqrt(ddx * ddx + ddy * ddy + ddz * ddz);
            float dcx = cpos.x - p.camera.x, dcy = cpos.y - p.camera.y, dcz = cpos.z - p.camera.z;
            float dc = std::sqrt(dcx * dcx + dcy * dcy + dcz * dcz);
            float hn_dot = cnor.x * hgb.normal.x + (cnor.y * hgb.normal.y + cnor.z * hgb.normal.z);
            if (dd < 0.02f * dc + 1e-3f && hn_dot > 0.9f && hrr.sumWu > 0 && hrr.M > 0 && hrr.p_hat > 0) {
              float ph, dist;
              V3<float> dn;
              if (eval_at(hrr.lightPos, hrr.lightNormal, hrr.emission, hrr.alpha, ph, dist, dn) && ph > 0) {
                float wu = ph * hrr.sumWu / hrr.p_hat;
                V3<float> so = mk(cpos.x + cnor.x * 0.002f, cpos.y + cnor.y * 0.002f, cpos.z + cnor.z * 0.002f);
                bool occ = pt.occluded(so, dn, dist - 0.003f);
                float ws = occ ? 0.0f : ph * hrr.sumWs / hrr.p_hat;
                float sum_s = cur_sumWs + ws, sum_u = cur_sumWu + wu;
                uint32_t newM = cur_M + hrr.M; if (newM > uint32_t(mcap)) newM = uint32_t(mcap);
                float r = pt.U();
                if (sum_s > 0 && r * sum_s < ws) {
                  cur_lp = hrr.lightPos; cur_ln = hrr.lightNormal; cur_le = hrr.emission; cur_alpha = hrr.alpha; cur_ph = ph;
                  cur_l = hrl ? hrl[rp.hidx] : -1;
                }
                cur_sumWs = sum_s; cur_sumWu = sum_u; cur_M = newM;
              }
            }
          }
        }
      }
      for (int si = 0; si < S; ++si) {
        float rx = pt.U() * 2.0f - 1.0f, ryy = pt.U() * 2.0f - 1.0f;
        float fx = float(x) + rx * radius + 0.5f, fy = float(y) + ryy * radius + 0.5f;
        if (!(fx > -1073741824.0f && fx < 1073741824.0f && fy > -1073741824.0f && fy < 1073741824.0f)) continue;
        int nx = int(fx), ny = int(fy);
        if (nx < 0 || ny < 0 || nx >= W || ny >= H) continue;
        if (nx == int(x) && ny == int(y)) continue;
        uint32_t nidx = uint32_t(ny) * uint32_t(W) + uint32_t(nx);
        if (gb[nidx].kind != 1 || ri[nidx].valid == 0) continue;
        const rm_vec3& nn = gb[nidx].normal;
        if (cnor.x * nn.x + (cnor.y * nn.y + cnor.z * nn.z) < 0.9f) continue;
        const Reservoir& N = ri[nidx];
        if (!(N.sumWu > 0) || N.M == 0 || !(N.p_hat > 0)) continue;
        float ph_cur, dist;
        V3<float> dn;
        if (!eval_at(N.lightPos, N.lightNormal, N.emission, N.alpha, ph_cur, dist, dn)) continue;
        if (!(ph_cur > 0)) continue;
        float w_nbr_u = ph_cur * N.sumWu / N.p_hat;
        if (!(w_nbr_u > 0)) continue;
        V3<float> so = mk(cpos.x + cnor.x * 0.002f, cpos.y + cnor.y * 0.002f, cpos.z + cnor.z * 0.002f);
        bool occ = pt.occluded(so, dn, dist - 0.003f);
        float w_nbr_s = occ ? 0.0f : ph_cur * N.sumWs / N.p_hat;
        float sum_s = cur_sumWs + w_nbr_s, sum_u = cur_sumWu + w_nbr_u;
        if (!(sum_u > 0) || !(sum_s >= 0)) continue;
        float r = pt.U();
        uint32_t newM = cur_M + N.M; if (newM > uint32_t(mcap)) newM = uint32_t(mcap);
        if (sum_s > 0 && r * sum_s < w_nbr_s) {
          cur_lp = N.lightPos; cur_ln = N.lightNormal; cur_le = N.emission; cur_alpha = N.alpha; cur_ph = ph_cur;
          cur_l = ril ? ril[nidx] : -1;
        }
        cur_sumWs = sum_s; cur_sumWu = sum_u; cur_M = newM;
      }
      Reservoir& O = ro_[id];
      O.lightPos = cur_lp; O.lightNormal = cur_ln; O.emission = cur_le; O.alpha = cur_alpha;
      O.p_hat = cur_ph; O.sumWs = cur_sumWs; O.sumWu = cur_sumWu; O.M = cur_M; O.valid = 1;
      if (rol) rol[id] = cur_l;
    }
    rays += ctr.rays;
  });
}

// K5 restir_shade (pathtrace.metal:1056-1258)
static void k_shade(const SceneRef& s, const Params& p, uint64_t seed, int row0, int row1, const GBuf* gb,
                    const Reservoir* rm, float* hdr, uint32_t* dbg, int nthreads, std::atomic<uint64_t>& samples,
                    std::atomic<uint64_t>& rays) {
  const int W = p.width;
  const float LT = p.light_total;
  parallel_for(row1 - row0, nthreads, [&](int ry) {
    uint32_t y = uint32_t(row0 + ry);
    Counters ctr;
    uint64_t taken = 0;
    for (uint32_t x = 0; x < uint32_t(W); ++x) {
      uint32_t id = y * uint32_t(W) + x;
      float* out = hdr + size_t(id) * 3;
      const GBuf& g = gb[id];
      if (g.kind == 0) {
        out[0] = out[1] = out[2] = 0;
        if (dbg) { dbg[id * 2] = 0; dbg[id * 2 + 1] = 0; }
        continue;
      }
      Tracer<float> pt{&s, &p, Rng{}, &ctr};
      pt.rng.seed(seed_shade(seed, id));
      auto clampv = [&](V3<float>& c) {
        if (p.clamp_value > 0) {
          c.x = std::fmin(c.x, p.clamp_value); c.y = std::fmin(c.y, p.clamp_value); c.z = std::fmin(c.z, p.clamp_value);
        }
      };
      if (g.kind == 3) {
        V3<float> sum = mk(0.f, 0.f, 0.f);
        int n = 0;
        for (int si = 0; si < p.spp; ++si) {
          float sx, sy;
          pt.jitter(x, y, sx, sy);
          V3<float> c = pt.sample_sensor(sx, sy, p.camera, p.camera.focal * p.camera.focal, p.bounces);
          clampv(c);
          sum.x += c.x; sum.y += c.y; sum.z += c.z;
          ++n;
        }
        float fn = float(std::max(n, 1));
        V3<float> c = mk(sum.x / fn, sum.y / fn, sum.z / fn);
        clampv(c);
        out[0] = c.x; out[1] = c.y; out[2] = c.z;
        taken += uint64_t(n);
        if (dbg) { dbg[id * 2] = pt.rng.state; dbg[id * 2 + 1] = uint32_t(n); }
        continue;
      }
      V3<float> gpos = vf<float>(g.pos), gnor = vf<float>(g.normal), galb = vf<float>(g.albedo),
                gwo = vf<float>(g.wo), gemi = vf<float>(g.emission);
      float rough = g.rough; if (rough < 0) rough = 0; if (rough > 1) rough = 1;
      float metallic = g.metallic; if (metallic < 0) metallic = 0; if (metallic > 1) metallic = 1;
      float r2 = rough; if (r2 < 0.02f) r2 = 0.02f;
      float alpha2 = (r2 * r2) * (r2 * r2);
      float spec_prob = 0.05f + 0.95f * metallic; if (spec_prob > 0.98f) spec_prob = 0.98f;
      if (metallic >= 0.999f) spec_prob = 1.0f;
      bool nomis = p.nomis;
      V3<float> prim = mk(0.f, 0.f, 0.f);
      float m_sumWu = 0;
      uint32_t m_M = 0;
      const Reservoir& R = rm[id];
      if (R.valid != 0 && R.M > 0 && R.sumWu > 0 && R.sumWs > 0 && R.p_hat > 0) {
        m_sumWu = R.sumWu; m_M = R.M;
        float m_sumWs = R.sumWs;
        float ldx = R.lightPos.x - gpos.x, ldy = R.lightPos.y - gpos.y, ldz = R.lightPos.z - gpos.z;
        float dist = std::sqrt(ldx * ldx + ldy * ldy + ldz * ldz);
        if (dist > 0.003f) {
          float inv = 1.0f / dist;
          float dxn = ldx * inv, dyn = ldy * inv, dzn = ldz * inv;
          float lcos = -(R.lightNormal.x * dxn + (R.lightNormal.y * dyn + R.lightNormal.z * dzn));
          float scos = gnor.x * dxn + (gnor.y * dyn + gnor.z * dzn);
          if (lcos > 1e-8f && scos > 1e-8f) {
            auto e = Tracer<float>::eval_bsdf(dxn, dyn, dzn, gwo.x, gwo.y, gwo.z, gnor.x, gnor.y, gnor.z, alpha2,
                                              metallic, spec_prob, galb.x, galb.y, galb.z);
            float Fr = R.emission.x * e.r * scos * R.alpha, Fg = R.emission.y * e.g * scos * R.alpha,
                  Fb = R.emission.z * e.b * scos * R.alpha;
            float ph = lum3(Fr, Fg, Fb);
            if (ph > 0) {
              float pdf_ris = float(m_M) * ph / m_sumWu;
              float wnee = 1.0f;
              if (!nomis && e.pdf > 1e-20f) wnee = pdf_ris / (pdf_ris + e.pdf);
              float Wt = m_sumWs / (float(m_M) * ph);
              prim = mk(Fr * Wt * wnee, Fg * Wt * wnee, Fb * Wt * wnee);
            }
          }
        }
      }
      V3<float> base = mk(gemi.x + prim.x, gemi.y + prim.y, gemi.z + prim.z);
      if (p.bounces <= 1 || p.spp <= 0) {
        V3<float> c = base;
        clampv(c);
        out[0] = c.x; out[1] = c.y; out[2] = c.z;
        if (dbg) { dbg[id * 2] = pt.rng.state; dbg[id * 2 + 1] = 0; }
        continue;
      }
      V3<float> sum = mk(0.f, 0.f, 0.f);
      int n = 0;
      for (int si = 0; si < p.spp; ++si) {
        float nx2, ny2, nz2;
        int pdelta = 0;
        bool early = false;
        if (pt.U() < spec_prob) {
          float hx, hy, hz;
          pt.sample_ggx_half(alpha2, gnor.x, gnor.y, gnor.z, hx, hy, hz);
          float md = gwo.x * hx + (gwo.y * hy + gwo.z * hz);
          if (!(md > 1e-8f)) early = true;
          else {
            nx2 = 2.0f * md * hx - gwo.x; ny2 = 2.0f * md * hy - gwo.y; nz2 = 2.0f * md * hz - gwo.z;
            pdelta = (rough <= 0.0201f) ? 1 : 0;
          }
        } else {
          pt.sample_cosine(gnor.x, gnor.y, gnor.z, nx2, ny2, nz2);
          pdelta = 0;
        }
        Tracer<float>::Bsdf e0;
        if (!early) {
          float ncos = nx2 * gnor.x + (ny2 * gnor.y + nz2 * gnor.z);
          if (!(ncos > 1e-8f)) early = true;
          else {
            float d = 1.0f / std::sqrt(nx2 * nx2 + ny2 * ny2 + nz2 * nz2);
            nx2 *= d; ny2 *= d; nz2 *= d;
            e0 = Tracer<float>::eval_bsdf(nx2, ny2, nz2, gwo.x, gwo.y, gwo.z, gnor.x, gnor.y, gnor.z, alpha2,
                                          metallic, spec_prob, galb.x, galb.y, galb.z);
            if (!(e0.pdf > 1e-12f)) early = true;
          }
        }
        if (early) {
          V3<float> full = base;
          clampv(full);
          sum.x += full.x; sum.y += full.y; sum.z += full.z;
          ++n;
          continue;
        }
        float cos0 = nx2 * gnor.x + (ny2 * gnor.y + nz2 * gnor.z);
        V3<float> thr = mk(e0.r * cos0 / e0.pdf, e0.g * cos0 / e0.pdf, e0.b * cos0 / e0.pdf);
        float ox = gpos.x + gnor.x * 0.001f, oy = gpos.y + gnor.y * 0.001f, oz = gpos.z + gnor.z * 0.001f;
        float dx = nx2, dy = ny2, dz = nz2;
        float last_pdf = e0.pdf;
        float pb_r = e0.r, pb_g = e0.g, pb_b = e0.b, pb_cos = cos0;
        float psumW = m_sumWu;
        uint32_t pM = m_M;
        int pdel = pdelta;
        V3<float> acc = mk(0.f, 0.f, 0.f);
        for (int b = 1; b < p.bounces; ++b) {
          Hit<float> hit = pt.cast_alpha_ray(mk(ox, oy, oz), mk(dx, dy, dz), 1e30f);
          if (hit.tri < 0) break;
          float pnx = hit.n_interp.x, pny = hit.n_interp.y, pnz = hit.n_interp.z;
          float gg = hit.n_geom.x * pnx + (hit.n_geom.y * pny + hit.n_geom.z * pnz);
          if (gg < 0) { pnx = -pnx; pny = -pny; pnz = -pnz; }
          float nd = dx * pnx + (dy * pny + dz * pnz);
          bool front = true;
          if (nd > 0) { pnx = -pnx; pny = -pny; pnz = -pnz; front = false; }
          float wox = -dx, woy = -dy, woz = -dz;
          float rh = hit.rough; if (rh < 0) rh = 0; if (rh > 1) rh = 1; if (rh < 0.02f) rh = 0.02f;
          float al = rh * rh;
          float a2 = al * al;
          const rm_triangle& lt = s.tris[hit.tri];
          float met = lt.metallic; if (met < 0) met = 0; if (met > 1) met = 1;
          if (pdel == 1) {
            acc.x += hit.er * thr.x; acc.y += hit.eg * thr.y; acc.z += hit.eb * thr.z;
          } else {
            float lx = hit.p.x - ox, ly = hit.p.y - oy, lz = hit.p.z - oz;
            float d2 = lx * lx + ly * ly + lz * lz;
            float dd = std::sqrt(d2);
            float pl = 1e30f;
            if (dd > 1e-20f && last_pdf > 1e-20f && pM > 0 && psumW > 1e-20f) {
              float ph = lum3(hit.er * pb_r * pb_cos * lt.alpha, hit.eg * pb_g * pb_cos * lt.alpha,
                              hit.eb * pb_b * pb_cos * lt.alpha);
              if (ph > 1e-20f) pl = float(pM) * ph / psumW;
              else {
                float inv = 1.0f / dd;
                float xn = lx * inv, yn = ly * inv, zn = lz * inv;
                float cl = -(lt.nn.x * xn + (lt.nn.y * yn + lt.nn.z * zn));
                if (cl > 1e-8f) {
                  float lum = lum3(lt.er, lt.eg, lt.eb); if (lum < 1e-6f) lum = 1e-6f;
                  pl = d2 * lum / (cl * LT);
                }
              }
            } else if (dd > 1e-20f && last_pdf > 1e-20f) {
              float inv = 1.0f / dd;
              lx *= inv; ly *= inv; lz *= inv;
              float cl = -(lt.nn.x * lx + (lt.nn.y * ly + lt.nn.z * lz));
              if (cl > 1e-8f) {
                float lum = lum3(lt.er, lt.eg, lt.eb); if (lum < 1e-6f) lum = 1e-6f;
                pl = d2 * lum / (cl * LT);
              }
            }
            float w = nomis ? 0.0f : ((last_pdf + pl > 1e-20f) ? last_pdf / (last_pdf + pl) : 0.0f);
            acc.x += hit.er * thr.x * w; acc.y += hit.eg * thr.y * w; acc.z += hit.eb * thr.z * w;
          }
          if (hit.ior > 1.0001f) {
            auto ds = pt.sample_dielectric(wox, woy, woz, pnx, pny, pnz, dx, dy, dz, hit.ior, front, rh, a2);
            if (!ds.valid) break;
            thr.x *= ds.eta_scale; thr.y *= ds.eta_scale; thr.z *= ds.eta_scale;
            float sgn = 1.0f;
            if (ds.n_x * pnx + (ds.n_y * pny + ds.n_z * pnz) < 0) sgn = -1.0f;
            ox = hit.p.x + pnx * 0.001f * sgn; oy = hit.p.y + pny * 0.001f * sgn; oz = hit.p.z + pnz * 0.001f * sgn;
            dx = ds.n_x; dy = ds.n_y; dz = ds.n_z;
            pdel = 1; psumW = 0; pM = 0;
          } else {
            float sp2 = 0.05f + 0.95f * met; if (sp2 > 0.98f) sp2 = 0.98f; if (met >= 0.999f) sp2 = 1.0f;
            float dlr = 0, dlg = 0, dlb = 0, csum = 0;
            uint32_t cM = 0;
            pt.direct_lighting(hit.p.x, hit.p.y, hit.p.z, pnx, pny, pnz, wox, woy, woz, rh, met, sp2, hit.ar, hit.ag,
                               hit.ab, dlr, dlg, dlb, csum, cM);
            acc.x += dlr * thr.x; acc.y += dlg * thr.y; acc.z += dlb * thr.z;
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
              float d = 1.0f / std::sqrt(qx2 * qx2 + qy2 * qy2 + qz2 * qz2);
              qx2 *= d; qy2 *= d; qz2 *= d;
            }
            auto ee = Tracer<float>::eval_bsdf(qx2, qy2, qz2, wox, woy, woz, pnx, pny, pnz, a2, met, sp2, hit.ar,
                                               hit.ag, hit.ab);
            if (!(ee.pdf > 1e-12f)) break;
            last_pdf = ee.pdf;
            float ci = qx2 * pnx + (qy2 * pny + qz2 * pnz);
            thr.x *= ee.r * ci / ee.pdf; thr.y *= ee.g * ci / ee.pdf; thr.z *= ee.b * ci / ee.pdf;
            psumW = csum; pM = cM;
            pb_r = ee.r; pb_g = ee.g; pb_b = ee.b; pb_cos = ci;
            ox = hit.p.x + pnx * 0.001f; oy = hit.p.y + pny * 0.001f; oz = hit.p.z + pnz * 0.001f;
            dx = qx2; dy = qy2; dz = qz2;
          }
          float mx = std::max(thr.x, thr.y);
          mx = std::max(mx, thr.z);
          if (!(mx >= 1e-12f)) break;
          if (p.rr && b >= 2) {
            float rr = mx; if (rr < 0.05f) rr = 0.05f; if (rr > 0.9f) rr = 0.9f;
            if (!(pt.U() <= rr)) break;
            float ir = 1.0f / rr;
            thr.x *= ir; thr.y *= ir; thr.z *= ir;
          }
        }
        V3<float> full = mk(base.x + acc.x, base.y + acc.y, base.z + acc.z);
        clampv(full);
        sum.x += full.x; sum.y += full.y; sum.z += full.z;
        ++n;
      }
      float fn = float(std::max(n, 1));
      out[0] = sum.x / fn; out[1] = sum.y / fn; out[2] = sum.z / fn;
      taken += uint64_t(n);
      if (dbg) { dbg[id * 2] = pt.rng.state; dbg[id * 2 + 1] = uint32_t(n); }
    }
    samples += taken;
    rays += ctr.rays;
  });
}

// K6 denoise_temporal (pathtrace.metal:1263-1314)
static void k_temporal(const Params& p, const GBuf* gb, const GBuf* hg, const float* cur, const float* hc,
                       float* out, int nthreads) {
  const int W = p.width, H = p.height;
  parallel_for(H, nthreads, [&](int yi) {
    uint32_t y = uint32_t(yi);
    for (uint32_t x = 0; x < uint32_t(W); ++x) {
      size_t id = size_t(y) * size_t(W) + x;
      float c[3] = {cur[id * 3], cur[id * 3 + 1], cur[id * 3 + 2]};
      float o[3] = {c[0], c[1], c[2]};
      if (p.hasHistory != 0 && gb[id].kind == 1) {
        float mn[3] = {c[0], c[1], c[2]}, mx[3] = {c[0], c[1], c[2]};
        for (int dy = -1; dy <= 1; ++dy)
          for (int dx = -1; dx <= 1; ++dx) {
            int nx = int(x) + dx, ny = int(y) + dy;
            if (nx < 0 || ny < 0 || nx >= W || ny >= H) continue;
            size_t n = size_t(ny) * size_t(W) + size_t(nx);
            for (int k = 0; k < 3; ++k) {
              mn[k] = std::fmin(mn[k], cur[n * 3 + size_t(k)]);
              mx[k] = std::fmax(mx[k], cur[n * 3 + size_t(k)]);
            }
          }
        const GBuf& g = gb[id];
        Reproj rp = reproject(p, g.pos.x, g.pos.y, g.pos.z);
        if (rp.ok && hg[rp.hidx].kind == 1) {
          const GBuf& h = hg[rp.hidx];
          float ddx = g.pos.x - h.pos.x, ddy = g.pos.y - h.pos.y, ddz = g.pos.z - h.pos.z;
          float dd = std::sqrt(ddx * ddx + ddy * ddy + ddz * ddz);
          float dcx = g.pos.x - p.camera.x, dcy = g.pos.y - p.camera.y, dcz = g.pos.z - p.camera.z;
          float dc = std::sqrt(dcx * dcx + dcy * dcy + dcz * dcz);
          if (dd < 0.02f * dc + 1e-3f &&
              (g.normal.x * h.normal.x + (g.normal.y * h.normal.y + g.normal.z * h.normal.z)) > 0.9f) {
            for (int k = 0; k < 3; ++k) {
              float hv = hc[size_t(rp.hidx) * 3 + size_t(k)];
              hv = std::fmin(std::fmax(hv, mn[k]), mx[k]);
              o[k] = hv + (c[k] - hv) * 0.2f;
            }
          }
        }
      }
      out[id * 3] = o[0]; out[id * 3 + 1] = o[1]; out[id * 3 + 2] = o[2];
    }
  });
}

// K7 denoise_atrous (pathtrace.metal:1315-1354)
static void k_atrous(const Params& p, const GBuf* gb, const float* in, float* out, int step, int nthreads) {
  const int W = p.width, H = p.height;
  const int stride = 1 << step;
  parallel_for(H, nthreads, [&](int yi) {
    uint32_t y = uint32_t(yi);
    for (uint32_t x = 0; x < uint32_t(W); ++x) {
      size_t id = size_t(y) * size_t(W) + x;
      const GBuf& g0 = gb[id];
      if (g0.kind == 0) { out[id * 3] = out[id * 3 + 1] = out[id * 3 + 2] = 0; continue; }
      float c0[3] = {in[id * 3], in[id * 3 + 1], in[id * 3 + 2]};
      float l0 = luma(c0[0], c0[1], c0[2]);
      float dcx = g0.pos.x - p.camera.x, dcy = g0.pos.y - p.camera.y, dcz = g0.pos.z - p.camera.z;
      float dc = std::sqrt(dcx * dcx + dcy * dcy + dcz * dcz);
      float sum[3] = {0, 0, 0}, wsum = 0;
      for (int dy = -2; dy <= 2; ++dy)
        for (int dx = -2; dx <= 2; ++dx) {
          int nx = int(x) + dx * stride, ny = int(y) + dy * stride;
          if (nx < 0 || ny < 0 || nx >= W || ny >= H) continue;
          size_t n = size_t(ny) * size_t(W) + size_t(nx);
          const GBuf& g = gb[n];
          if (g.kind == 0) continue;
          float c[3] = {in[n * 3], in[n * 3 + 1], in[n * 3 + 2]};
          float nd = g.normal.x * g0.normal.x + (g.normal.y * g0.normal.y + g.normal.z * g0.normal.z);
          float wn = rm_pow16f(std::max(nd, 0.0f));
          float ex = g.pos.x - g0.pos.x, ey = g.pos.y - g0.pos.y, ez = g.pos.z - g0.pos.z;
          float wz = rm_expf(-std::sqrt(ex * ex + ey * ey + ez * ez) / (0.1f * dc + 1e-4f));
          float wl = rm_expf(-std::fabs(luma(c[0], c[1], c[2]) - l0) / (0.3f * std::max(l0, 0.5f) + 1e-3f));
          float ax = g.albedo.x - g0.albedo.x, ay = g.albedo.y - g0.albedo.y, az = g.albedo.z - g0.albedo.z;
          float wa = rm_expf(-std::sqrt(ax * ax + ay * ay + az * az) / 0.25f);
          float w = wn * wz * wl * wa;
          sum[0] += w * c[0]; sum[1] += w * c[1]; sum[2] += w * c[2];
          wsum += w;
        }
      if (wsum > 1e-12f) {
        out[id * 3] = sum[0] / wsum; out[id * 3 + 1] = sum[1] / wsum; out[id * 3 + 2] = sum[2] / wsum;
      } else {
        out[id * 3] = c0[0]; out[id * 3 + 1] = c0[1]; out[id * 3 + 2] = c0[2];
      }
    }
  });
}

}  // namespace orc

// ---------------------------------------------------------------- C API
using namespace orc;

namespace orc {
namespace {

// ---- frozen-path evaluation: the finite-difference side of the adjoint check
//
// The adjoint (raymotion_b200/csrc/rm_adjoint.cu) differentiates the plain
// frame with its sampling held at the current parameters: every random
// decision, direction, pdf, MIS weight and Russian-roulette probability stays
// as the fp32 path made it, and only the material-dependent factors of the
// path integrand move.  frozen_path() walks the fp32 path exactly as
// Tracer<float>::pathtrace does (pathtrace.metal:552-728, single-candidate
// NEE :319-384 or RIS NEE :385-469 with the selection and its resampling
// weight held, dielectric :470-534), taking every decision from it, and
// evaluates alongside in double the sample's value with the material factors
// at parameters `prm`: the opaque BSDF value (albedo x texel, alpha2 from the
// roughness), the emission of hit and sampled lights, and for a dielectric
// the Fresnel / (eta_i/eta_t)^2 and microfacet D, G factors relative to their
// value at the scene's own (fp32) parameters.  At the scene's parameters it is
// the fp32 sample in double; its central differences are what the adjoint's
// gradient must match.
struct MatTable {
  const int32_t* tri_mat = nullptr;  // per triangle, -1: the triangle's own values
  const double* prm = nullptr;       // n x 8: albedo rgb, rough, emission rgb, ior
  double get(const rm_triangle* tris, int tri, int k) const {
    const int m = tri_mat ? tri_mat[tri] : -1;
    if (m >= 0) return prm[size_t(m) * 8 + size_t(k)];
    const rm_triangle& t = tris[tri];
    switch (k) {
      case 0: return t.ar;
      case 1: return t.ag;
      case 2: return t.ab;
      case 3: return t.rough;
      case 4: return t.er;
      case 5: return t.eg;
      case 6: return t.eb;
      default: return t.ior;
    }
  }
};

double alpha2_of(double rough) {
  double r = rough;
  if (r < 0) r = 0;
  if (r > 1) r = 1;
  if (r < 0.02) r = 0.02;
  return (r * r) * (r * r);
}

V3<double> bsdf64(const MatTable& mt, const SceneRef& s, const Hit<float>& hit, double wix, double wiy, double wiz,
                  double wox, double woy, double woz, double nx, double ny, double nz, double metallic,
                  double spec_prob) {
  double a[3];
  const double tx[3] = {double(hit.txr), double(hit.txg), double(hit.txb)};
  const double own[3] = {double(hit.ar), double(hit.ag), double(hit.ab)};
  for (int c = 0; c < 3; ++c) a[c] = hit.shader == 1 ? own[c] : mt.get(s.tris, hit.tri, c) * tx[c];
  const auto e = Tracer<double>::eval_bsdf(wix, wiy, wiz, wox, woy, woz, nx, ny, nz,
                                           alpha2_of(mt.get(s.tris, hit.tri, 3)), metallic, spec_prob, a[0], a[1],
                                           a[2]);
  return mk(e.r, e.g, e.b);
}

// The dielectric factor that depends on the material: event 0 reflection
// (Fresnel), 1 refraction ((1 - Fresnel) (eta_i/eta_t)^2), 2 total internal
// reflection (1); for a rough surface, whatever the event, times D and the
// clamped G weight (pathtrace.metal:520-532 weights every rough event).
double diel_value(double ior, bool front, int event, double cos_m, bool rough_branch, double alpha2, double cos_i,
                  double cos_o, double cos_h, double vo_h) {
  double v = 1.0;
  if (event != 2) {
    const double ei = front ? 1.0 : ior, et = front ? ior : 1.0;
    const double F = Tracer<double>::fresnel(cos_m, ei, et);
    v = event == 0 ? F : (1.0 - F) * (ei / et) * (ei / et);
  }
  if (rough_branch) {
    const double dd = cos_h * cos_h * (alpha2 - 1.0) + 1.0;
    const double D = alpha2 / (3.141592653589793 * dd * dd);
    const double g1 = 2.0 * cos_o / (cos_o + std::sqrt(cos_o * cos_o + alpha2 * (1.0 - cos_o * cos_o)));
    const double g2 = 2.0 * cos_i / (cos_i + std::sqrt(cos_i * cos_i + alpha2 * (1.0 - cos_i * cos_i)));
    double w = g1 * g2 * vo_h / (cos_o * cos_h);
    if (w > 10.0) w = 10.0;
    v *= D * w;
  }
  return v;
}

// A path continued from a vertex already shaded (the ReSTIR shade's first
// hit, pathtrace.metal:1135-1255): its throughput (fp32, and in double at the
// parameters), the BSDF sample that left it and its light-sample sums.
struct FrozenFrom {
  float thr[3];
  double t64[3];
  float last_pdf, prev_b[3], prev_cos, prev_sumW;
  uint32_t prev_M;
  int prev_delta;
};

V3<double> frozen_path(Tracer<float>& pt, const MatTable& mt, V3<float> ro, V3<float> rd, int max_bounces,
                       const FrozenFrom* from = nullptr) {
  const SceneRef& S = *pt.s;
  const Params& P = *pt.p;
  float ox = ro.x, oy = ro.y, oz = ro.z, dx = rd.x, dy = rd.y, dz = rd.z;
  float thr_r = 1, thr_g = 1, thr_b = 1;
  double t64[3] = {1, 1, 1}, a64[3] = {0, 0, 0};
  int bounce = 0, prev_delta = 1;
  float last_pdf = 0, prev_sumW = 0;
  uint32_t prev_M = 0;
  float prev_br = 0, prev_bg = 0, prev_bb = 0, prev_cos = 0;
  const bool camera = from == nullptr;
  if (from) {
    thr_r = from->thr[0]; thr_g = from->thr[1]; thr_b = from->thr[2];
    for (int c = 0; c < 3; ++c) t64[c] = from->t64[c];
    last_pdf = from->last_pdf;
    prev_br = from->prev_b[0]; prev_bg = from->prev_b[1]; prev_bb = from->prev_b[2]; prev_cos = from->prev_cos;
    prev_sumW = from->prev_sumW; prev_M = from->prev_M; prev_delta = from->prev_delta;
  }
  const float LT = float(P.light_total);
  for (int b = 0; b < max_bounces; ++b) {
    Hit<float> hit = pt.cast_alpha_ray(mk(ox, oy, oz), mk(dx, dy, dz), 1e30f);
    if (hit.tri < 0) break;
    float pnx = hit.n_interp.x, pny = hit.n_interp.y, pnz = hit.n_interp.z;
    float geom = hit.n_geom.x * pnx + (hit.n_geom.y * pny + hit.n_geom.z * pnz);
    if (geom < 0) { pnx = -pnx; pny = -pny; pnz = -pnz; }
    float ndot = dx * pnx + (dy * pny + dz * pnz);
    bool front = true;
    if (ndot > 0) { pnx = -pnx; pny = -pny; pnz = -pnz; front = false; }
    float wox = -dx, woy = -dy, woz = -dz;
    float rough = hit.rough;
    if (rough < 0) rough = 0;
    if (rough > 1) rough = 1;
    if (rough < 0.02f) rough = 0.02f;
    float alpha = rough * rough;
    float alpha2 = alpha * alpha;
    const rm_triangle& lt = S.tris[hit.tri];
    float metallic = lt.metallic;
    if (metallic < 0) metallic = 0;
    if (metallic > 1) metallic = 1;
    float we = 1.0f;
    if (!((camera && bounce == 0) || prev_delta == 1)) {
      float lx = hit.p.x - ox, ly = hit.p.y - oy, lz = hit.p.z - oz;
      float dist2 = lx * lx + ly * ly + lz * lz;
      float dist = std::sqrt(dist2);
      float pl = 1e30f;
      if (dist > 1e-20f && last_pdf > 1e-20f && prev_M > 0 && prev_sumW > 1e-20f) {
        float ph = lum3(hit.er * prev_br * prev_cos * lt.alpha, hit.eg * prev_bg * prev_cos * lt.alpha,
                        hit.eb * prev_bb * prev_cos * lt.alpha);
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
      we = P.nomis ? 0.0f : ((last_pdf + pl > 1e-20f) ? last_pdf / (last_pdf + pl) : 0.0f);
    }
    for (int c = 0; c < 3; ++c) a64[c] += mt.get(S.tris, hit.tri, 4 + c) * t64[c] * double(we);
    if (hit.ior > 1.0001f) {
      // sample_dielectric (pathtrace.metal:470-534) with its pieces kept
      float eta_i = 1.0f, eta_t = hit.ior;
      if (!front) { eta_i = hit.ior; eta_t = 1.0f; }
      float hx, hy, hz;
      bool valid = true;
      if (rough <= 0.0201f) { hx = pnx; hy = pny; hz = pnz; }
      else {
        pt.sample_ggx_half(alpha2, pnx, pny, pnz, hx, hy, hz);
        float md = wox * hx + (woy * hy + woz * hz);
        if (!(md > 1e-8f)) valid = false;
      }
      float cos_m = wox * hx + (woy * hy + woz * hz);
      if (cos_m < 0) { hx = -hx; hy = -hy; hz = -hz; cos_m = -cos_m; }
      if (cos_m > 1) cos_m = 1;
      float fres = Tracer<float>::fresnel(cos_m, eta_i, eta_t);
      float eta = eta_i / eta_t;
      float s2 = eta * eta * (1.0f - cos_m * cos_m);
      float n_x, n_y, n_z, es;
      int event;
      if (s2 >= 1.0f || pt.U() < fres) {
        n_x = 2.0f * cos_m * hx - wox;
        n_y = 2.0f * cos_m * hy - woy;
        n_z = 2.0f * cos_m * hz - woz;
        es = 1.0f;
        event = s2 >= 1.0f ? 2 : 0;
      } else {
        float cos_t = std::sqrt(1.0f - s2);
        n_x = eta * dx + hx * (eta * cos_m - cos_t);
        n_y = eta * dy + hy * (eta * cos_m - cos_t);
        n_z = eta * dz + hz * (eta * cos_m - cos_t);
        es = eta * eta;
        event = 1;
      }
      {
        float d = 1.0f / std::sqrt(n_x * n_x + n_y * n_y + n_z * n_z);
        n_x *= d; n_y *= d; n_z *= d;
      }
      float ci = 0, co = 0, chh = 0, voh = 0;
      const bool rb = rough > 0.0201f;
      if (rb) {
        ci = std::fabs(n_x * pnx + (n_y * pny + n_z * pnz));
        co = std::fabs(wox * pnx + (woy * pny + woz * pnz));
        chh = std::fabs(hx * pnx + (hy * pny + hz * pnz));
        voh = std::fabs(wox * hx + (woy * hy + woz * hz));
        if (ci > 1e-8f && co > 1e-8f && chh > 1e-8f && voh > 1e-8f) {
          float g1 = 2.0f * co / (co + std::sqrt(co * co + alpha2 * (1.0f - co * co)));
          float g2 = 2.0f * ci / (ci + std::sqrt(ci * ci + alpha2 * (1.0f - ci * ci)));
          float w = g1 * g2 * voh / (co * chh);
          if (w > 10.0f) w = 10.0f;
          es *= w;
        } else {
          valid = false;
        }
      }
      if (!valid) break;
      const double v0 = diel_value(lt.ior, front, event, cos_m, rb, alpha2_of(lt.rough), ci, co, chh, voh);
      const double v1 = diel_value(mt.get(S.tris, hit.tri, 7), front, event, cos_m, rb,
                                   alpha2_of(mt.get(S.tris, hit.tri, 3)), ci, co, chh, voh);
      const double ratio = v0 > 0 ? v1 / v0 : 1.0;
      for (int c = 0; c < 3; ++c) t64[c] *= double(es) * ratio;
      thr_r *= es; thr_g *= es; thr_b *= es;
      float sg = 1.0f;
      if (n_x * pnx + (n_y * pny + n_z * pnz) < 0.0f) sg = -1.0f;
      ox = hit.p.x + pnx * 0.001f * sg;
      oy = hit.p.y + pny * 0.001f * sg;
      oz = hit.p.z + pnz * 0.001f * sg;
      dx = n_x; dy = n_y; dz = n_z;
      prev_delta = 1;
      prev_sumW = 0; prev_M = 0;
    } else {
      float spec_prob = 0.05f + 0.95f * metallic;
      if (spec_prob > 0.98f) spec_prob = 0.98f;
      if (metallic >= 0.999f) spec_prob = 1.0f;
      float cur_sumW = 0;
      uint32_t cur_M = 0;
      int Mc = P.restir_candidates;
      if (Mc < 1) Mc = 1;
      if (Mc > 32) Mc = 32;
      // direct_lighting with RIS over Mc candidates (pathtrace.metal:385-469):
      // the selection, its resampling weight W and the MIS weight are held;
      // the selected light's emission and this surface's BSDF move
      if (Mc > 1 && P.lights != 0 && LT > 1e-12f) {
        float r2 = rough;
        if (r2 < 0.02f) r2 = 0.02f;
        float al2 = (r2 * r2) * (r2 * r2);
        float sumW = 0;
        float sel_lx = 0, sel_ly = 0, sel_lz = 0, sel_phat = 0, sel_epdf = 0, sel_sa = 0;
        float sel_dx = 0, sel_dy = 0, sel_dz = 0;
        int sel_tri = -1;
        bool have = false;
        for (int j = 0; j < Mc; ++j) {
          float pick = pt.U() * LT;
          const int ltri = pt.pick_light(pick);
          const rm_triangle& t = S.tris[ltri];
          float lu = pt.U(), lv = pt.U();
          if (lu + lv > 1.0f) { lu = 1.0f - lu; lv = 1.0f - lv; }
          float lw = 1.0f - lu - lv;
          float qx = lw * t.v0.x + (lu * t.v1.x + lv * t.v2.x);
          float qy = lw * t.v0.y + (lu * t.v1.y + lv * t.v2.y);
          float qz = lw * t.v0.z + (lu * t.v1.z + lv * t.v2.z);
          float ldx = qx - hit.p.x, ldy = qy - hit.p.y, ldz = qz - hit.p.z;
          float dist = std::sqrt(ldx * ldx + ldy * ldy + ldz * ldz);
          float w = 0, ph = 0, epdf = 0, sa = 0, dxn = 0, dyn = 0, dzn = 0;
          if (dist > 0.003f) {
            float inv = 1.0f / dist;
            dxn = ldx * inv; dyn = ldy * inv; dzn = ldz * inv;
            float lcos = -(t.nn.x * dxn + (t.nn.y * dyn + t.nn.z * dzn));
            float scos = pnx * dxn + (pny * dyn + pnz * dzn);
            if (lcos > 1e-8f && scos > 1e-8f) {
              float lt_lum = lum3(t.er, t.eg, t.eb);
              if (lt_lum < 1e-6f) lt_lum = 1e-6f;
              float q = dist * dist * lt_lum / (lcos * LT);
              if (q > 1e-12f) {
                auto e = Tracer<float>::eval_bsdf(dxn, dyn, dzn, wox, woy, woz, pnx, pny, pnz, al2, metallic,
                                                  spec_prob, hit.ar, hit.ag, hit.ab);
                epdf = e.pdf;
                float Fr = t.er * e.r * scos * t.alpha;
                float Fg = t.eg * e.g * scos * t.alpha;
                float Fb = t.eb * e.b * scos * t.alpha;
                ph = lum3(Fr, Fg, Fb);
                if (ph > 0.0f) w = ph / q;
                sa = scos * t.alpha;
              }
            }
          }
          sumW += w;
          float r = pt.U();
          if (w > 0.0f && r * sumW < w) {
            have = true;
            sel_lx = qx; sel_ly = qy; sel_lz = qz;
            sel_phat = ph; sel_epdf = epdf; sel_sa = sa;
            sel_dx = dxn; sel_dy = dyn; sel_dz = dzn;
            sel_tri = ltri;
          }
        }
        cur_sumW = sumW;
        cur_M = uint32_t(Mc);
        if (have && sumW > 0.0f && sel_phat > 0.0f) {
          float pdf_ris = float(Mc) * sel_phat / sumW;
          float wnee = 1.0f;
          if (!P.nomis && sel_epdf > 1e-20f) wnee = pdf_ris / (pdf_ris + sel_epdf);
          float vdx = sel_lx - hit.p.x, vdy = sel_ly - hit.p.y, vdz = sel_lz - hit.p.z;
          float vdist = std::sqrt(vdx * vdx + vdy * vdy + vdz * vdz);
          if (vdist > 0.003f) {
            float vinv = 1.0f / vdist;
            vdx *= vinv; vdy *= vinv; vdz *= vinv;
            V3<float> so = mk(hit.p.x + pnx * 0.002f, hit.p.y + pny * 0.002f, hit.p.z + pnz * 0.002f);
            if (!pt.occluded(so, mk(vdx, vdy, vdz), vdist - 0.003f)) {
              const float W = sumW / (float(Mc) * sel_phat);
              const double k = double(sel_sa) * double(W) * double(wnee);
              const V3<double> f = bsdf64(mt, S, hit, sel_dx, sel_dy, sel_dz, wox, woy, woz, pnx, pny, pnz, metallic,
                                          spec_prob);
              const double fv[3] = {f.x, f.y, f.z};
              for (int c = 0; c < 3; ++c) a64[c] += t64[c] * mt.get(S.tris, sel_tri, 4 + c) * fv[c] * k;
            }
          }
        }
      }
      // direct_lighting, single candidate (pathtrace.metal:319-384)
      if (Mc <= 1 && P.lights != 0 && LT > 1e-12f) {
        float r2 = rough;
        if (r2 < 0.02f) r2 = 0.02f;
        float al2 = (r2 * r2) * (r2 * r2);
        float pick = pt.U() * LT;
        const int ltri = pt.pick_light(pick);
        const rm_triangle& t = S.tris[ltri];
        float lu = pt.U(), lv = pt.U();
        if (lu + lv > 1.0f) { lu = 1.0f - lu; lv = 1.0f - lv; }
        float lw = 1.0f - lu - lv;
        float ldx = lw * t.v0.x + (lu * t.v1.x + lv * t.v2.x) - hit.p.x;
        float ldy = lw * t.v0.y + (lu * t.v1.y + lv * t.v2.y) - hit.p.y;
        float ldz = lw * t.v0.z + (lu * t.v1.z + lv * t.v2.z) - hit.p.z;
        float dist = std::sqrt(ldx * ldx + ldy * ldy + ldz * ldz);
        cur_M = 1;
        if (dist > 0.003f) {
          float inv = 1.0f / dist;
          ldx *= inv; ldy *= inv; ldz *= inv;
          float lcos = -(t.nn.x * ldx + (t.nn.y * ldy + t.nn.z * ldz));
          float scos = pnx * ldx + (pny * ldy + pnz * ldz);
          if (lcos > 1e-8f && scos > 1e-8f) {
            float lt_lum = lum3(t.er, t.eg, t.eb);
            if (lt_lum < 1e-6f) lt_lum = 1e-6f;
            float pdf = dist * dist * lt_lum / (lcos * LT);
            V3<float> so = mk(hit.p.x + pnx * 0.002f, hit.p.y + pny * 0.002f, hit.p.z + pnz * 0.002f);
            const bool occ = pt.occluded(so, mk(ldx, ldy, ldz), dist - 0.003f);
            auto e = Tracer<float>::eval_bsdf(ldx, ldy, ldz, wox, woy, woz, pnx, pny, pnz, al2, metallic, spec_prob,
                                              hit.ar, hit.ag, hit.ab);
            if (pdf > 1e-12f) {
              float Fr = t.er * e.r * scos * t.alpha;
              float Fg = t.eg * e.g * scos * t.alpha;
              float Fb = t.eb * e.b * scos * t.alpha;
              float ph = lum3(Fr, Fg, Fb);
              cur_sumW = ph > 0 ? ph / pdf : 0.0f;
              if (!occ) {
                float wnee = 1.0f;
                if (!P.nomis && e.pdf > 1e-20f) wnee = pdf / (pdf + e.pdf);
                const float k = scos * wnee * t.alpha / pdf;
                const V3<double> f = bsdf64(mt, S, hit, ldx, ldy, ldz, wox, woy, woz, pnx, pny, pnz, metallic,
                                            spec_prob);
                const double fv[3] = {f.x, f.y, f.z};
                for (int c = 0; c < 3; ++c) a64[c] += t64[c] * mt.get(S.tris, ltri, 4 + c) * fv[c] * double(k);
              }
            }
          }
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
        float d = 1.0f / std::sqrt(nx2 * nx2 + ny2 * ny2 + nz2 * nz2);
        nx2 *= d; ny2 *= d; nz2 *= d;
      }
      auto e = Tracer<float>::eval_bsdf(nx2, ny2, nz2, wox, woy, woz, pnx, pny, pnz, alpha2, metallic, spec_prob,
                                        hit.ar, hit.ag, hit.ab);
      if (!(e.pdf > 1e-12f)) break;
      last_pdf = e.pdf;
      float cos_i = nx2 * pnx + (ny2 * pny + nz2 * pnz);
      const V3<double> f = bsdf64(mt, S, hit, nx2, ny2, nz2, wox, woy, woz, pnx, pny, pnz, metallic, spec_prob);
      t64[0] *= f.x * double(cos_i) / double(e.pdf);
      t64[1] *= f.y * double(cos_i) / double(e.pdf);
      t64[2] *= f.z * double(cos_i) / double(e.pdf);
      thr_r *= e.r * cos_i / e.pdf;
      thr_g *= e.g * cos_i / e.pdf;
      thr_b *= e.b * cos_i / e.pdf;
      prev_sumW = cur_sumW; prev_M = cur_M;
      prev_br = e.r; prev_bg = e.g; prev_bb = e.b; prev_cos = cos_i;
      ox = hit.p.x + pnx * 0.001f;
      oy = hit.p.y + pny * 0.001f;
      oz = hit.p.z + pnz * 0.001f;
      dx = nx2; dy = ny2; dz = nz2;
    }
    if (thr_r < 0) thr_r = 0;
    if (thr_g < 0) thr_g = 0;
    if (thr_b < 0) thr_b = 0;
    for (int c = 0; c < 3; ++c)
      if (t64[c] < 0) t64[c] = 0;
    float mx = std::max(thr_r, thr_g);
    mx = std::max(mx, thr_b);
    if (!(mx >= 1e-12f)) break;
    if (P.rr && bounce >= 1) {
      float rr = mx;
      if (rr < 0.05f) rr = 0.05f;
      if (rr > 0.9f) rr = 0.9f;
      if (!(pt.U() <= rr)) break;
      float ir = 1.0f / rr;
      thr_r *= ir; thr_g *= ir; thr_b *= ir;
      for (int c = 0; c < 3; ++c) t64[c] *= double(ir);
    }
    bounce++;
  }
  return mk(a64[0], a64[1], a64[2]);
}

}  // namespace
}  // namespace orc

extern "C" {

orc::Ctx* orc_create(void) { return new orc::Ctx(); }
void orc_destroy(orc::Ctx* c) { delete c; }
void orc_reset_history(orc::Ctx* c) { c->hist_valid = false; }

// The reference frame (metal.mm:95-414).  rgb: W*H*3 bytes; hdr: W*H*3 floats
// (the tonemap input), either may be NULL.  row0/row1 restrict the rendered
// rows (row1 <= 0 means all rows); restricting rows is only meaningful for the
// plain path and for timing.  stats (may be NULL): [samples, rays, chain].
int orc_render(orc::Ctx* ctx, const rm_scene_view* sv, const rm_camera* cam, const rm_config* cfg, uint64_t seed,
               uint8_t* rgb, float* hdr, int nthreads, int row0, int row1, uint64_t* stats, char* err,
               size_t errcap) {
  const rm_config& c = *cfg;
  if (c.width <= 0 || c.height <= 0 || c.spp <= 0 || c.max_bounces < 0 ||
      size_t(c.width) * size_t(c.height) > 100000000) {
    set_err(err, errcap, "Invalid Metal render dimensions or sample count");
    return RM_ERR_INVALID;
  }
  if (row1 <= 0 || row1 > c.height) row1 = c.height;
  if (row0 < 0) row0 = 0;
  if (row0 > row1) row0 = row1;
  SceneRef s;
  s.tris = sv->tris; s.n_tris = sv->n_tris;
  s.nodes = to_preorder(sv->nodes, sv->n_nodes);
  s.indices = sv->bvh_tri; s.lights = sv->light_tri; s.cdf = sv->light_cdf;
  s.n_lights = sv->n_lights; s.light_total = sv->light_total; s.texels = sv->texels;
  bool opaque = true;
  for (int i = 0; i < sv->n_tris; ++i)
    if (!(sv->tris[i].alpha >= 1)) { opaque = false; break; }
  Env env = read_env(c.flags);
  Params p = resolve(c, *cam, int(s.nodes.size()), sv->n_lights, sv->light_total, opaque, env);
  const size_t pixels = size_t(c.width) * size_t(c.height);
  const size_t restir_bytes = pixels * (sizeof(GBuf) + 2 * sizeof(Reservoir));
  bool use_spatial = p.restir_spatial > 0 && p.lights > 0 && p.bounces > 0 && p.opaque &&
                     restir_bytes <= size_t(512) * 1024 * 1024;
  uint64_t hash = scene_hash(sv->tris, sv->n_tris, sv->n_lights, sv->light_total);
  bool animated = (c.flags & RM_FLAG_ANIMATED_HISTORY) != 0;
  bool have_hist = use_spatial && ctx->hist_valid && ctx->hist_w == c.width && ctx->hist_h == c.height &&
                   ctx->have_hist_bufs && seed != ctx->hist_seed && (animated || hash == ctx->hist_hash);
  if (env.temporal_off) have_hist = false;
  p.hasHistory = have_hist ? 1 : 0;
  p.prevCamera = ctx->hist_cam;
  std::atomic<uint64_t> samples{0}, rays{0};
  ctx->hdr.assign(pixels * 3, 0.0f);
  ctx->dbg.assign(pixels * 2, 0u);
  int chain = 0;
  if (use_spatial) {
    chain = 2;
    ctx->g.assign(pixels, GBuf{});
    ctx->rinit.assign(pixels, Reservoir{});
    ctx->rmerged.assign(pixels, Reservoir{});
    if (ctx->hist_g.size() != pixels) { ctx->hist_g.assign(pixels, GBuf{}); ctx->hist_r.assign(pixels, Reservoir{}); }
    if (ctx->hist_col.size() != pixels * 3) ctx->hist_col.assign(pixels * 3, 0.0f);
    // generate on a band wide enough for the spatial neighbourhood
    int pad = int(std::ceil(std::max(p.restir_radius, 16.0f))) + 2;
    int g0 = std::max(0, row0 - pad), g1 = std::min(c.height, row1 + pad);
    k_generate(s, p, seed, g0, g1, ctx->g.data(), ctx->rinit.data(), nthreads, rays);
    k_spatial(s, p, seed, row0, row1, ctx->g.data(), ctx->rinit.data(), ctx->rmerged.data(), ctx->hist_g.data(),
              ctx->hist_r.data(), nthreads, rays);
    k_shade(s, p, seed, row0, row1, ctx->g.data(), ctx->rmerged.data(), ctx->hdr.data(), ctx->dbg.data(), nthreads,
            samples, rays);
    bool denoise = !env.denoise_off;
    std::vector<float> final_col = ctx->hdr;
    if (denoise) {
      std::vector<float> den_a(pixels * 3), tmp(pixels * 3);
      k_temporal(p, ctx->g.data(), ctx->hist_g.data(), ctx->hdr.data(), ctx->hist_col.data(), den_a.data(), nthreads);
      k_atrous(p, ctx->g.data(), den_a.data(), tmp.data(), 0, nthreads);
      k_atrous(p, ctx->g.data(), tmp.data(), den_a.data(), 1, nthreads);
      final_col = den_a;
    }
    if (hdr) std::memcpy(hdr, final_col.data(), pixels * 3 * sizeof(float));
    if (rgb)
      for (size_t i = 0; i < pixels * 3; ++i) rgb[i] = tonemap8(final_col[i]);
    // publish history (metal.mm:374-385)
    ctx->hist_g = ctx->g;
    ctx->hist_r = ctx->rmerged;
    if (denoise) ctx->hist_col = final_col;
    ctx->have_hist_bufs = true;
    ctx->hist_cam = *cam;
    ctx->hist_w = c.width; ctx->hist_h = c.height;
    ctx->hist_seed = seed; ctx->hist_hash = hash; ctx->hist_valid = true;
  } else {
    int lanes = 1;
    if (c.spp >= 8 && (p.adapt_min <= 0 || p.adapt_step % 8 == 0)) lanes = 8;
    if (c.spp >= 32 && (p.adapt_min <= 0 || p.adapt_step % 32 == 0)) lanes = 32;
    chain = lanes;
    k_render_paths(s, p, seed, lanes, row0, row1, ctx->hdr.data(), ctx->dbg.data(), nthreads, samples, rays);
    if (hdr) std::memcpy(hdr, ctx->hdr.data(), pixels * 3 * sizeof(float));
    if (rgb)
      for (size_t i = 0; i < pixels * 3; ++i) rgb[i] = tonemap8(ctx->hdr[i]);
  }
  ctx->samples = samples.load();
  ctx->rays = rays.load();
  ctx->chain = chain;
  if (stats) { stats[0] = ctx->samples; stats[1] = ctx->rays; stats[2] = uint64_t(chain); }
  return RM_OK;
}

// Last frame's buffers: 0 G-buffer (76 B/px), 1 initial reservoir, 2 merged
// reservoir (60 B/px), 3 shaded HDR (12 B/px), 4 per-pixel (rng xor, samples).
int orc_debug_read(orc::Ctx* ctx, int which, void* host, size_t cap) {
  const void* src = nullptr;
  size_t n = 0;
  switch (which) {
    case 0: src = ctx->g.data(); n = ctx->g.size() * sizeof(GBuf); break;
    case 1: src = ctx->rinit.data(); n = ctx->rinit.size() * sizeof(Reservoir); break;
    case 2: src = ctx->rmerged.data(); n = ctx->rmerged.size() * sizeof(Reservoir); break;
    case 3: src = ctx->hdr.data(); n = ctx->hdr.size() * sizeof(float); break;
    case 4: src = ctx->dbg.data(); n = ctx->dbg.size() * sizeof(uint32_t); break;
    default: return RM_ERR_INVALID;
  }
  if (cap < n) return RM_ERR_INVALID;
  if (n) std::memcpy(host, src, n);
  return RM_OK;
}

// Closest-hit / any-hit queries: rays are n records of 7 floats.
int orc_trace(const rm_scene_view* sv, const float* rays, int n, int any_hit, int32_t* tri, float* t, float* u,
              float* v, int nthreads) {
  SceneRef s;
  s.tris = sv->tris; s.n_tris = sv->n_tris;
  s.nodes = to_preorder(sv->nodes, sv->n_nodes);
  s.indices = sv->bvh_tri;
  Params p{};
  p.nodes = int(s.nodes.size());
  p.opaque = 1;
  int chunks = (n + 1023) / 1024;
  parallel_for(chunks, nthreads, [&](int ci) {
    Tracer<float> pt{&s, &p, Rng{}, nullptr};
    for (int i = ci * 1024; i < std::min(n, ci * 1024 + 1024); ++i) {
      const float* r = rays + size_t(i) * 7;
      Hit<float> h = pt.intersect(mk(r[0], r[1], r[2]), mk(r[3], r[4], r[5]), r[6], any_hit != 0);
      tri[i] = h.tri;
      if (t) t[i] = h.tri >= 0 ? h.t : r[6];
      if (u) u[i] = h.u;
      if (v) v[i] = h.v;
    }
  });
  return RM_OK;
}

// FP64 instantiation of the plain path tracer with one RNG stream per
// (pixel, sample) and no adaptive stop: the ground truth for convergence
// (relMSE) checks.  Writes W*H*3 doubles of mean radiance.
int orc_render_f64(const rm_scene_view* sv, const rm_camera* cam, const rm_config* cfg, uint64_t seed, double* out,
                   int nthreads, const int32_t* pixel_list, int n_pixels) {
  SceneRef s;
  s.tris = sv->tris; s.n_tris = sv->n_tris;
  s.nodes = to_preorder(sv->nodes, sv->n_nodes);
  s.indices = sv->bvh_tri; s.lights = sv->light_tri; s.cdf = sv->light_cdf;
  s.n_lights = sv->n_lights; s.light_total = sv->light_total; s.texels = sv->texels;
  bool opaque = true;
  for (int i = 0; i < sv->n_tris; ++i)
    if (!(sv->tris[i].alpha >= 1)) { opaque = false; break; }
  Env env = read_env(cfg->flags | RM_FLAG_NO_ENV);
  Params p = resolve(*cfg, *cam, int(s.nodes.size()), sv->n_lights, sv->light_total, opaque, env);
  const int W = cfg->width;
  const int count = pixel_list ? n_pixels : W * cfg->height;
  parallel_for(count, nthreads, [&](int k) {
    int id = pixel_list ? pixel_list[k] : k;
    uint32_t x = uint32_t(id % W), y = uint32_t(id / W);
    double sum[3] = {0, 0, 0};
    for (int si = 0; si < p.spp; ++si) {
      Tracer<double> pt{&s, &p, Rng{}, nullptr};
      pt.rng.seed(seed_lane(seed, x, y, uint32_t(si)));
      double sx, sy;
      pt.jitter(x, y, sx, sy);
      double f = double(cam->focal);
      V3<double> c = pt.sample_sensor(sx, sy, *cam, f * f, p.bounces);
      if (p.clamp_value > 0) {
        c.x = std::fmin(c.x, double(p.clamp_value)); c.y = std::fmin(c.y, double(p.clamp_value));
        c.z = std::fmin(c.z, double(p.clamp_value));
      }
      sum[0] += c.x; sum[1] += c.y; sum[2] += c.z;
    }
    double* o = out + size_t(k) * 3;
    o[0] = sum[0] / p.spp; o[1] = sum[1] / p.spp; o[2] = sum[2] / p.spp;
  });
  return RM_OK;
}

// ---- reference CPU BVH (src/engine/bvh.cpp), fp64 -------------------------
// verts: n*9 doubles (v0, v1, v2 per triangle).  nodes_out: capacity 2n
// records of {mn[3], mx[3]} doubles; links_out: 2n records of
// {left, right, offset, count}; bvh_tri_out: n ints.  Returns the node count.

namespace {
struct BTri { double mn[3], mx[3], c[3]; };
inline double area_of(const double* mn, const double* mx) {
  double dx = mx[0] - mn[0], dy = mx[1] - mn[1], dz = mx[2] - mn[2];
  return 2.0 * (dx * dy + dy * dz + dz * dx);
}
}  // namespace

int orc_build_bvh(const double* verts, int n, int max_leaf, double* nodes_out, int32_t* links_out,
                  int32_t* bvh_tri_out) {
  const double inf = std::numeric_limits<double>::infinity();
  max_leaf = std::max(1, max_leaf);
  if (n <= 0) return 0;
  std::vector<BTri> T(static_cast<size_t>(n));
  for (int i = 0; i < n; ++i) {
    const double* v = verts + size_t(i) * 9;
    for (int a = 0; a < 3; ++a) {
      T[size_t(i)].mn[a] = std::min({v[a], v[3 + a], v[6 + a]});
      T[size_t(i)].mx[a] = std::max({v[a], v[3 + a], v[6 + a]});
      T[size_t(i)].c[a] = v[a] + v[3 + a] + v[6 + a];  // bvh.cpp:14-18: vertex sum
    }
  }
  std::vector<int> idx(static_cast<size_t>(n));
  std::iota(idx.begin(), idx.end(), 0);
  struct N { double mn[3], mx[3]; int left = -1, right = -1, offset = -1, count = 0; };
  std::vector<N> nodes;
  nodes.reserve(size_t(2 * n));
  nodes.push_back(N{});
  struct Job { int offset, count, node; };
  std::queue<Job> q;  // breadth-first job order, bvh.cpp:43-48
  q.push({0, n, 0});
  constexpr int kBins = 16;
  while (!q.empty()) {
    Job job = q.front();
    q.pop();
    double mn[3] = {inf, inf, inf}, mx[3] = {-inf, -inf, -inf}, cmn[3] = {inf, inf, inf}, cmx[3] = {-inf, -inf, -inf};
    int* base = idx.data() + job.offset;
    for (int k = 0; k < job.count; ++k) {
      const BTri& t = T[size_t(base[k])];
      for (int a = 0; a < 3; ++a) {
        if (t.mn[a] < mn[a]) mn[a] = t.mn[a];
        if (t.mx[a] > mx[a]) mx[a] = t.mx[a];
        if (t.c[a] < cmn[a]) cmn[a] = t.c[a];
        if (t.c[a] > cmx[a]) cmx[a] = t.c[a];
      }
    }
    N& nd = nodes[size_t(job.node)];
    for (int a = 0; a < 3; ++a) { nd.mn[a] = mn[a]; nd.mx[a] = mx[a]; }
    if (job.count <= max_leaf) {  // bvh.cpp:93-99
      nd.offset = job.offset; nd.count = job.count; nd.left = nd.right = -1;
      continue;
    }
    auto longest_axis = [&]() {
      double sx = mx[0] - mn[0], sy = mx[1] - mn[1], sz = mx[2] - mn[2];
      return (sx > sy) ? ((sx > sz) ? 0 : 2) : ((sy > sz) ? 1 : 2);
    };
    auto sort_axis = [&](int ax) {
      std::sort(base, base + job.count, [&](int a, int b) { return T[size_t(a)].c[ax] < T[size_t(b)].c[ax]; });
    };
    auto split_into = [&](int mid) {
      int l = int(nodes.size());
      nodes.push_back(N{});
      int r = int(nodes.size());
      nodes.push_back(N{});
      N& pn = nodes[size_t(job.node)];
      pn.left = l; pn.right = r; pn.offset = -1; pn.count = 0;
      q.push({job.offset, mid, l});
      q.push({job.offset + mid, job.count - mid, r});
    };
    double parent_area = area_of(mn, mx);
    if (!(parent_area > 0)) {  // degenerate box: median of the longest axis, bvh.cpp:103-124
      sort_axis(longest_axis());
      split_into(job.count / 2);
      continue;
    }
    double best_cost = double(job.count);
    int best_axis = -1, best_bin = -1;
    for (int axis = 0; axis < 3; ++axis) {  // 16-bin SAH sweep, bvh.cpp:125-209
      double c0 = cmn[axis], c1 = cmx[axis], span = c1 - c0;
      if (!(span > 0)) continue;
      int cnt[kBins];
      double bmn[kBins][3], bmx[kBins][3];
      for (int b = 0; b < kBins; ++b) {
        cnt[b] = 0;
        for (int a = 0; a < 3; ++a) { bmn[b][a] = inf; bmx[b][a] = -inf; }
      }
      double inv = kBins / span;
      for (int k = 0; k < job.count; ++k) {
        const BTri& t = T[size_t(base[k])];
        int b = int((t.c[axis] - c0) * inv);
        if (b < 0) b = 0;
        if (b >= kBins) b = kBins - 1;
        cnt[b]++;
        for (int a = 0; a < 3; ++a) {
          if (t.mn[a] < bmn[b][a]) bmn[b][a] = t.mn[a];
          if (t.mx[a] > bmx[b][a]) bmx[b][a] = t.mx[a];
        }
      }
      int rcount[kBins];
      double rmn[kBins][3], rmx[kBins][3];
      int acc = 0;
      double amn[3] = {inf, inf, inf}, amx[3] = {-inf, -inf, -inf};
      for (int b = kBins - 1; b >= 0; --b) {
        acc += cnt[b];
        rcount[b] = acc;
        if (cnt[b] > 0)
          for (int a = 0; a < 3; ++a) {
            if (bmn[b][a] < amn[a]) amn[a] = bmn[b][a];
            if (bmx[b][a] > amx[a]) amx[a] = bmx[b][a];
          }
        for (int a = 0; a < 3; ++a) { rmn[b][a] = amn[a]; rmx[b][a] = amx[a]; }
      }
      int lcount = 0;
      double lmn[3] = {inf, inf, inf}, lmx[3] = {-inf, -inf, -inf};
      for (int b = 0; b < kBins - 1; ++b) {
        lcount += cnt[b];
        if (cnt[b] > 0)
          for (int a = 0; a < 3; ++a) {
            if (bmn[b][a] < lmn[a]) lmn[a] = bmn[b][a];
            if (bmx[b][a] > lmx[a]) lmx[a] = bmx[b][a];
          }
        int rc = rcount[b + 1];
        if (lcount == 0 || rc == 0) continue;
        double cost = (area_of(lmn, lmx) * lcount + area_of(rmn[b + 1], rmx[b + 1]) * rc) / parent_area;
        if (cost < best_cost) { best_cost = cost; best_axis = axis; best_bin = b; }
      }
    }
    int mid = -1;
    if (best_axis >= 0) {  // partition at the best bin boundary, bvh.cpp:211-225
      double c0 = cmn[best_axis], c1 = cmx[best_axis];
      double split = c0 + (c1 - c0) * (best_bin + 1) / double(kBins);
      int* m = std::partition(base, base + job.count, [&](int a) { return T[size_t(a)].c[best_axis] < split; });
      mid = int(m - base);
      if (mid == 0 || mid == job.count) mid = -1;
    }
    if (mid < 0) {  // median of the longest axis, bvh.cpp:226-235
      sort_axis(longest_axis());
      mid = job.count / 2;
    }
    split_into(mid);
  }
  for (size_t i = 0; i < nodes.size(); ++i) {
    for (int a = 0; a < 3; ++a) { nodes_out[i * 6 + size_t(a)] = nodes[i].mn[a]; nodes_out[i * 6 + 3 + size_t(a)] = nodes[i].mx[a]; }
    links_out[i * 4] = nodes[i].left; links_out[i * 4 + 1] = nodes[i].right;
    links_out[i * 4 + 2] = nodes[i].offset; links_out[i * 4 + 3] = nodes[i].count;
  }
  std::memcpy(bvh_tri_out, idx.data(), sizeof(int) * size_t(n));
  return int(nodes.size());
}

// refit_bvh (bvh.cpp:250-272): reverse node order, leaves from triangle
// bounds, internal nodes from children.  tri_bounds: n*6 doubles (mn, mx).
void orc_refit_bvh(const double* tri_bounds, int n_nodes, double* nodes_io, const int32_t* links,
                   const int32_t* bvh_tri) {
  const double inf = std::numeric_limits<double>::infinity();
  for (int i = n_nodes - 1; i >= 0; --i) {
    double mn[3] = {inf, inf, inf}, mx[3] = {-inf, -inf, -inf};
    const int32_t* L = links + size_t(i) * 4;
    if (L[3] > 0) {
      for (int k = 0; k < L[3]; ++k) {
        const double* b = tri_bounds + size_t(bvh_tri[L[2] + k]) * 6;
        for (int a = 0; a < 3; ++a) { mn[a] = std::min(mn[a], b[a]); mx[a] = std::max(mx[a], b[3 + a]); }
      }
    } else {
      for (int c : {L[0], L[1]}) {
        const double* b = nodes_io + size_t(c) * 6;
        for (int a = 0; a < 3; ++a) { mn[a] = std::min(mn[a], b[a]); mx[a] = std::max(mx[a], b[3 + a]); }
      }
    }
    for (int a = 0; a < 3; ++a) { nodes_io[size_t(i) * 6 + size_t(a)] = mn[a]; nodes_io[size_t(i) * 6 + 3 + size_t(a)] = mx[a]; }
  }
}

// Deterministic math exported for the tests of include/rm_detmath.h.
void orc_detmath(int which, const float* x, float* y0, float* y1, int n) {
  for (int i = 0; i < n; ++i) {
    if (which == 0) rm_sincosf(x[i], &y0[i], &y1[i]);
    else if (which == 1) y0[i] = rm_atanf(x[i]);
    else if (which == 2) y0[i] = rm_expf(x[i]);
  }
}

// Frozen-path evaluation of the plain frame (see frozen_path): out receives
// W*H*3 doubles, the mean over spp samples of each pixel's clamped sample
// values with material parameters prm (n_materials x 8 doubles) applied
// through tri_material; every decision comes from the fp32 path of the scene
// as given.  The frame must have a fixed sample count and take the plain
// chain.  Returns 0, or RM_ERR_INVALID.
int orc_render_frozen(const rm_scene_view* sv, const rm_camera* cam, const rm_config* cfg, uint64_t seed,
                      const int32_t* tri_material, const double* prm, int n_materials, double* out, int nthreads) {
  using namespace orc;
  if (cfg->width <= 0 || cfg->height <= 0 || cfg->spp <= 0 || cfg->max_bounces < 0 || n_materials < 0)
    return RM_ERR_INVALID;
  SceneRef s;
  s.tris = sv->tris; s.n_tris = sv->n_tris;
  s.nodes = to_preorder(sv->nodes, sv->n_nodes);
  s.indices = sv->bvh_tri; s.lights = sv->light_tri; s.cdf = sv->light_cdf;
  s.n_lights = sv->n_lights; s.light_total = sv->light_total; s.texels = sv->texels;
  bool opaque = true;
  for (int i = 0; i < sv->n_tris; ++i)
    if (!(sv->tris[i].alpha >= 1)) { opaque = false; break; }
  Env env = read_env(cfg->flags);
  Params p = resolve(*cfg, *cam, int(s.nodes.size()), sv->n_lights, sv->light_total, opaque, env);
  if (p.adapt_min > 0) return RM_ERR_INVALID;
  // the ReSTIR chain's policy (metal.mm:236-237) would not render the plain frame
  if (p.restir_spatial > 0 && p.lights > 0 && p.bounces > 0 && p.opaque &&
      size_t(cfg->width) * size_t(cfg->height) * (76 + 2 * 60) <= size_t(512) * 1024 * 1024)
    return RM_ERR_INVALID;
  int lanes = 1;
  if (p.spp >= 8) lanes = 8;
  if (p.spp >= 32) lanes = 32;
  MatTable mt;
  mt.tri_mat = tri_material;
  mt.prm = prm;
  const int W = p.width;
  parallel_for(p.height, nthreads, [&](int y) {
    Counters ctr;
    for (int x = 0; x < W; ++x) {
      double sum[3] = {0, 0, 0};
      for (int l = 0; l < lanes; ++l) {
        Tracer<float> pt{&s, &p, Rng{}, &ctr};
        pt.rng.seed(lanes == 1 ? seed_pixel(seed, uint32_t(x), uint32_t(y))
                               : seed_lane(seed, uint32_t(x), uint32_t(y), uint32_t(l)));
        for (int si = l; si < p.spp; si += lanes) {
          float sx, sy;
          pt.jitter(uint32_t(x), uint32_t(y), sx, sy);
          const rm_camera& c = p.camera;
          float focal2 = c.focal * c.focal;
          float dist = 1.0f / std::sqrt(sx * sx + (sy * sy + focal2));
          float tx = sx * dist, ty = sy * dist, tz = c.focal * dist;
          V3<float> rd = mk(tx * c.m0 + (ty * c.m1 + tz * c.m2), tx * c.m3 + (ty * c.m4 + tz * c.m5),
                            tx * c.m6 + (ty * c.m7 + tz * c.m8));
          V3<double> v = frozen_path(pt, mt, mk(c.x, c.y, c.z), rd, p.bounces);
          if (p.clamp_value > 0) {
            const double cl = p.clamp_value;
            v.x = std::fmin(v.x, cl); v.y = std::fmin(v.y, cl); v.z = std::fmin(v.z, cl);
          }
          sum[0] += v.x; sum[1] += v.y; sum[2] += v.z;
        }
      }
      double* o = out + (size_t(y) * size_t(W) + size_t(x)) * 3;
      for (int k = 0; k < 3; ++k) o[k] = sum[k] / double(p.spp);
    }
  });
  return RM_OK;
}

// K7 (pathtrace.metal:1315-1354) in double on a held G-buffer geometry: the
// denoiser of the frozen frame, with the colour it filters and the albedo of
// its weights (each pixel's first-hit albedo at the parameters) in double.
static void atrous64(const Params& p, const GBuf* gb, const double* alb, const double* in, double* out, int step,
                     int nthreads) {
  const int W = p.width, H = p.height;
  const int stride = 1 << step;
  auto lum = [](const double* c) { return 0.2126 * c[0] + 0.7152 * c[1] + 0.0722 * c[2]; };
  parallel_for(H, nthreads, [&](int yi) {
    for (int x = 0; x < W; ++x) {
      const size_t id = size_t(yi) * size_t(W) + size_t(x);
      const GBuf& g0 = gb[id];
      double* o = out + id * 3;
      if (g0.kind == 0) { o[0] = o[1] = o[2] = 0; continue; }
      const double* c0 = in + id * 3;
      const double l0 = lum(c0);
      const double dcx = double(g0.pos.x) - p.camera.x, dcy = double(g0.pos.y) - p.camera.y,
                   dcz = double(g0.pos.z) - p.camera.z;
      const double dc = std::sqrt(dcx * dcx + dcy * dcy + dcz * dcz);
      double sum[3] = {0, 0, 0}, wsum = 0;
      for (int dy = -2; dy <= 2; ++dy)
        for (int dx = -2; dx <= 2; ++dx) {
          const int nx = x + dx * stride, ny = yi + dy * stride;
          if (nx < 0 || ny < 0 || nx >= W || ny >= H) continue;
          const size_t n = size_t(ny) * size_t(W) + size_t(nx);
          const GBuf& g = gb[n];
          if (g.kind == 0) continue;
          const double* c = in + n * 3;
          double nd = double(g.normal.x) * g0.normal.x + double(g.normal.y) * g0.normal.y +
                      double(g.normal.z) * g0.normal.z;
          double wn = std::max(nd, 0.0);
          wn *= wn; wn *= wn; wn *= wn; wn *= wn;
          const double ex = double(g.pos.x) - g0.pos.x, ey = double(g.pos.y) - g0.pos.y,
                       ez = double(g.pos.z) - g0.pos.z;
          const double wz = std::exp(-std::sqrt(ex * ex + ey * ey + ez * ez) / (0.1 * dc + 1e-4));
          const double wl = std::exp(-std::fabs(lum(c) - l0) / (0.3 * std::max(l0, 0.5) + 1e-3));
          const double ax = alb[n * 3] - alb[id * 3], ay = alb[n * 3 + 1] - alb[id * 3 + 1],
                       az = alb[n * 3 + 2] - alb[id * 3 + 2];
          const double wa = std::exp(-std::sqrt(ax * ax + ay * ay + az * az) / 0.25);
          const double w = wn * wz * wl * wa;
          for (int k = 0; k < 3; ++k) sum[k] += w * c[k];
          wsum += w;
        }
      if (wsum > 1e-12)
        for (int k = 0; k < 3; ++k) o[k] = sum[k] / wsum;
      else
        for (int k = 0; k < 3; ++k) o[k] = c0[k];
    }
  });
}

// K6 (pathtrace.metal:1263-1314) in double on held G-buffers and a held
// history colour: the blend of the frozen colour with the reprojected,
// neighbourhood-clamped history.
static void temporal64(const Params& p, const GBuf* gb, const GBuf* hg, const double* cur, const float* hc,
                       double* out, int nthreads) {
  const int W = p.width, H = p.height;
  parallel_for(H, nthreads, [&](int yi) {
    for (int x = 0; x < W; ++x) {
      const size_t id = size_t(yi) * size_t(W) + size_t(x);
      const double* c = cur + id * 3;
      double* o = out + id * 3;
      for (int k = 0; k < 3; ++k) o[k] = c[k];
      if (p.hasHistory == 0 || gb[id].kind != 1) continue;
      double mn[3] = {c[0], c[1], c[2]}, mx[3] = {c[0], c[1], c[2]};
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          const int nx = x + dx, ny = yi + dy;
          if (nx < 0 || ny < 0 || nx >= W || ny >= H) continue;
          const size_t n = size_t(ny) * size_t(W) + size_t(nx);
          for (int k = 0; k < 3; ++k) {
            mn[k] = std::min(mn[k], cur[n * 3 + size_t(k)]);
            mx[k] = std::max(mx[k], cur[n * 3 + size_t(k)]);
          }
        }
      const GBuf& g = gb[id];
      const Reproj rp = reproject(p, g.pos.x, g.pos.y, g.pos.z);
      if (!(rp.ok && hg[rp.hidx].kind == 1)) continue;
      const GBuf& h = hg[rp.hidx];
      float ddx = g.pos.x - h.pos.x, ddy = g.pos.y - h.pos.y, ddz = g.pos.z - h.pos.z;
      float dd = std::sqrt(ddx * ddx + ddy * ddy + ddz * ddz);
      float dcx = g.pos.x - p.camera.x, dcy = g.pos.y - p.camera.y, dcz = g.pos.z - p.camera.z;
      float dc = std::sqrt(dcx * dcx + dcy * dcy + dcz * dcz);
      if (!(dd < 0.02f * dc + 1e-3f &&
            (g.normal.x * h.normal.x + (g.normal.y * h.normal.y + g.normal.z * h.normal.z)) > 0.9f))
        continue;
      for (int k = 0; k < 3; ++k) {
        const double hv = std::min(std::max(double(hc[size_t(rp.hidx) * 3 + size_t(k)]), mn[k]), mx[k]);
        o[k] = hv + (c[k] - hv) * 0.2;
      }
    }
  });
}

// Frozen evaluation of a ReSTIR frame (K3, K4, K5 and the denoiser; the first
// frame of a history): K3 and K4 run in fp32 at the scene's own
// materials and their G-buffer and merged reservoirs are held (the adjoint's
// checkpoint), with each reservoir's light triangle; K5 is replayed from them
// with its decisions from the fp32 path and the material factors in double at
// `prm`: a kind-3 pixel's samples are frozen camera paths; a kind-1 pixel's
// base is the first hit's emission plus the held light sample's Le f cos
// alpha W w_MIS, and each indirect sample leaves the first hit with the BSDF
// sample f cos / pdf and goes on as a frozen path (pathtrace.metal:1056-1258).
// The first hit's triangle comes from K3's primary ray traced again.  Unless
// the frame's denoiser is off, K6 and the two a-trous passes then run in
// double on the held G-buffers and history colour.  With prev_cam, the frame
// is the second of a history: the first (prev_cam, prev_seed) is rendered in
// fp32 as the CUDA path renders it and supplies the history G-buffer,
// reservoirs (with their light indices) and final colour.
int orc_render_frozen_restir(const rm_scene_view* sv, const rm_camera* cam, const rm_config* cfg, uint64_t seed,
                             const int32_t* tri_material, const double* prm, int n_materials, double* out,
                             int nthreads, const rm_camera* prev_cam, uint64_t prev_seed) {
  using namespace orc;
  if (cfg->width <= 0 || cfg->height <= 0 || cfg->spp <= 0 || cfg->max_bounces < 0 || n_materials < 0)
    return RM_ERR_INVALID;
  SceneRef s;
  s.tris = sv->tris; s.n_tris = sv->n_tris;
  s.nodes = to_preorder(sv->nodes, sv->n_nodes);
  s.indices = sv->bvh_tri; s.lights = sv->light_tri; s.cdf = sv->light_cdf;
  s.n_lights = sv->n_lights; s.light_total = sv->light_total; s.texels = sv->texels;
  bool opaque = true;
  for (int i = 0; i < sv->n_tris; ++i)
    if (!(sv->tris[i].alpha >= 1)) { opaque = false; break; }
  Env env = read_env(cfg->flags);
  Params p = resolve(*cfg, *cam, int(s.nodes.size()), sv->n_lights, sv->light_total, opaque, env);
  const int W = p.width, H = p.height;
  const size_t pixels = size_t(W) * size_t(H);
  if (!(p.restir_spatial > 0 && p.lights > 0 && p.bounces > 0 && p.opaque &&
        pixels * (sizeof(GBuf) + 2 * sizeof(Reservoir)) <= size_t(512) * 1024 * 1024))
    return RM_ERR_INVALID;  // the policy renders the plain frame: orc_render_frozen
  p.hasHistory = 0;
  std::vector<GBuf> g(pixels), hg(pixels);
  std::vector<Reservoir> ri(pixels), rmg(pixels), hr(pixels);
  std::vector<int32_t> ril(pixels, -1), rml(pixels, -1), hrl(pixels, -1);
  std::vector<float> hcol(pixels * 3, 0.0f);
  std::atomic<uint64_t> rays{0};
  if (prev_cam) {
    // the history frame, in fp32 as rendered (its light indices tracked): the
    // held G-buffer, reservoirs and final colour the frame reuses
    Params p1 = resolve(*cfg, *prev_cam, int(s.nodes.size()), sv->n_lights, sv->light_total, opaque, env);
    p1.hasHistory = 0;
    std::vector<GBuf> g0(pixels);
    std::vector<Reservoir> r0(pixels), hr0(pixels);
    std::vector<int32_t> l0(pixels, -1);
    std::vector<float> h1(pixels * 3), t1(pixels * 3);
    std::atomic<uint64_t> smp{0};
    k_generate(s, p1, prev_seed, 0, H, hg.data(), r0.data(), nthreads, rays, l0.data());
    k_spatial(s, p1, prev_seed, 0, H, hg.data(), r0.data(), hr.data(), g0.data(), hr0.data(), nthreads, rays,
              l0.data(), hrl.data(), nullptr);
    k_shade(s, p1, prev_seed, 0, H, hg.data(), hr.data(), h1.data(), nullptr, nthreads, smp, rays);
    if (!env.denoise_off) {
      k_temporal(p1, hg.data(), g0.data(), h1.data(), hcol.data(), t1.data(), nthreads);
      k_atrous(p1, hg.data(), t1.data(), h1.data(), 0, nthreads);
      k_atrous(p1, hg.data(), h1.data(), hcol.data(), 1, nthreads);
    } else {
      hcol = h1;
    }
    p.hasHistory = 1;
    p.prevCamera = *prev_cam;
  }
  k_generate(s, p, seed, 0, H, g.data(), ri.data(), nthreads, rays, ril.data());
  k_spatial(s, p, seed, 0, H, g.data(), ri.data(), rmg.data(), hg.data(), hr.data(), nthreads, rays, ril.data(),
            rml.data(), hrl.data());
  MatTable mt;
  mt.tri_mat = tri_material;
  mt.prm = prm;
  std::vector<double> alb64(pixels * 3, 0.0);
  const double cl = p.clamp_value;
  parallel_for(H, nthreads, [&](int yy) {
    Counters ctr;
    const uint32_t y = uint32_t(yy);
    for (uint32_t x = 0; x < uint32_t(W); ++x) {
      const uint32_t id = y * uint32_t(W) + x;
      double* o = out + size_t(id) * 3;
      o[0] = o[1] = o[2] = 0;
      const GBuf& gg = g[id];
      if (gg.kind == 0) continue;
      Tracer<float> pt{&s, &p, Rng{}, &ctr};
      pt.rng.seed(seed_shade(seed, id));
      auto clampd = [&](double* v) {
        if (cl > 0)
          for (int c = 0; c < 3; ++c) v[c] = std::fmin(v[c], cl);
      };
      const rm_camera& c = p.camera;
      // the first hit's triangle, from K3's primary ray
      Hit<float> h0;
      {
        Tracer<float> p3{&s, &p, Rng{}, &ctr};
        p3.rng.seed(seed_pixel(seed, x, y));
        float sx = float(x) + 1e-12f + (p.resolution - 2e-12f) * p3.U() - float(p.width) * 0.5f;
        float sy = float(p.height) * 0.5f - (float(y) + 1e-12f + (p.resolution - 2e-12f) * p3.U());
        float f2 = c.focal * c.focal;
        float dinv = 1.0f / std::sqrt(sx * sx + sy * sy + f2);
        float tx = sx * dinv, ty = sy * dinv, tz = c.focal * dinv;
        V3<float> rd = mk(tx * c.m0 + (ty * c.m1 + tz * c.m2), tx * c.m3 + (ty * c.m4 + tz * c.m5),
                          tx * c.m6 + (ty * c.m7 + tz * c.m8));
        h0 = p3.cast_alpha_ray(mk(c.x, c.y, c.z), rd, 1e30f);
      }
      if (h0.tri < 0) continue;
      // the G-buffer albedo at the parameters (the denoiser's weights)
      {
        const double tx[3] = {double(h0.txr), double(h0.txg), double(h0.txb)};
        const double own[3] = {double(h0.ar), double(h0.ag), double(h0.ab)};
        for (int k = 0; k < 3; ++k) alb64[size_t(id) * 3 + k] = h0.shader == 1 ? own[k] : mt.get(s.tris, h0.tri, k) * tx[k];
      }
      if (gg.kind == 3) {
        double sum[3] = {0, 0, 0};
        for (int si = 0; si < p.spp; ++si) {
          float sx, sy;
          pt.jitter(x, y, sx, sy);
          float focal2 = c.focal * c.focal;
          float dist = 1.0f / std::sqrt(sx * sx + (sy * sy + focal2));
          float tx = sx * dist, ty = sy * dist, tz = c.focal * dist;
          V3<float> rd = mk(tx * c.m0 + (ty * c.m1 + tz * c.m2), tx * c.m3 + (ty * c.m4 + tz * c.m5),
                            tx * c.m6 + (ty * c.m7 + tz * c.m8));
          const V3<double> v = frozen_path(pt, mt, mk(c.x, c.y, c.z), rd, p.bounces);
          double vv[3] = {v.x, v.y, v.z};
          clampd(vv);
          for (int k = 0; k < 3; ++k) sum[k] += vv[k];
        }
        for (int k = 0; k < 3; ++k) o[k] = sum[k] / double(p.spp);
        clampd(o);
        continue;
      }
      V3<float> gpos = vf<float>(gg.pos), gnor = vf<float>(gg.normal), galb = vf<float>(gg.albedo),
                gwo = vf<float>(gg.wo);
      float rough = gg.rough; if (rough < 0) rough = 0; if (rough > 1) rough = 1;
      float metallic = gg.metallic; if (metallic < 0) metallic = 0; if (metallic > 1) metallic = 1;
      float r2 = rough; if (r2 < 0.02f) r2 = 0.02f;
      float alpha2 = (r2 * r2) * (r2 * r2);
      float spec_prob = 0.05f + 0.95f * metallic; if (spec_prob > 0.98f) spec_prob = 0.98f;
      if (metallic >= 0.999f) spec_prob = 1.0f;
      double base[3];
      for (int k = 0; k < 3; ++k) base[k] = mt.get(s.tris, h0.tri, 4 + k);
      float m_sumWu = 0;
      uint32_t m_M = 0;
      const Reservoir& R = rmg[id];
      if (R.valid != 0 && R.M > 0 && R.sumWu > 0 && R.sumWs > 0 && R.p_hat > 0) {
        m_sumWu = R.sumWu; m_M = R.M;
        float ldx = R.lightPos.x - gpos.x, ldy = R.lightPos.y - gpos.y, ldz = R.lightPos.z - gpos.z;
        float dist = std::sqrt(ldx * ldx + ldy * ldy + ldz * ldz);
        if (dist > 0.003f) {
          float inv = 1.0f / dist;
          float dxn = ldx * inv, dyn = ldy * inv, dzn = ldz * inv;
          float lcos = -(R.lightNormal.x * dxn + (R.lightNormal.y * dyn + R.lightNormal.z * dzn));
          float scos = gnor.x * dxn + (gnor.y * dyn + gnor.z * dzn);
          if (lcos > 1e-8f && scos > 1e-8f) {
            auto e = Tracer<float>::eval_bsdf(dxn, dyn, dzn, gwo.x, gwo.y, gwo.z, gnor.x, gnor.y, gnor.z, alpha2,
                                              metallic, spec_prob, galb.x, galb.y, galb.z);
            float Fr = R.emission.x * e.r * scos * R.alpha, Fg = R.emission.y * e.g * scos * R.alpha,
                  Fb = R.emission.z * e.b * scos * R.alpha;
            float ph = lum3(Fr, Fg, Fb);
            if (ph > 0 && rml[id] >= 0) {
              float pdf_ris = float(m_M) * ph / m_sumWu;
              float wnee = 1.0f;
              if (!p.nomis && e.pdf > 1e-20f) wnee = pdf_ris / (pdf_ris + e.pdf);
              float Wt = R.sumWs / (float(m_M) * ph);
              const double k = double(scos) * double(R.alpha) * double(Wt) * double(wnee);
              const V3<double> f = bsdf64(mt, s, h0, dxn, dyn, dzn, gwo.x, gwo.y, gwo.z, gnor.x, gnor.y, gnor.z,
                                          metallic, spec_prob);
              const double fv[3] = {f.x, f.y, f.z};
              for (int q = 0; q < 3; ++q) base[q] += mt.get(s.tris, rml[id], 4 + q) * fv[q] * k;
            }
          }
        }
      }
      if (p.bounces <= 1) {
        for (int k = 0; k < 3; ++k) o[k] = base[k];
        clampd(o);
        continue;
      }
      double sum[3] = {0, 0, 0};
      for (int si = 0; si < p.spp; ++si) {
        float nx2 = 0, ny2 = 0, nz2 = 0;
        int pdelta = 0;
        bool early = false;
        if (pt.U() < spec_prob) {
          float hx, hy, hz;
          pt.sample_ggx_half(alpha2, gnor.x, gnor.y, gnor.z, hx, hy, hz);
          float md = gwo.x * hx + (gwo.y * hy + gwo.z * hz);
          if (!(md > 1e-8f)) early = true;
          else {
            nx2 = 2.0f * md * hx - gwo.x; ny2 = 2.0f * md * hy - gwo.y; nz2 = 2.0f * md * hz - gwo.z;
            pdelta = (rough <= 0.0201f) ? 1 : 0;
          }
        } else {
          pt.sample_cosine(gnor.x, gnor.y, gnor.z, nx2, ny2, nz2);
          pdelta = 0;
        }
        Tracer<float>::Bsdf e0;
        if (!early) {
          float ncos = nx2 * gnor.x + (ny2 * gnor.y + nz2 * gnor.z);
          if (!(ncos > 1e-8f)) early = true;
          else {
            float d = 1.0f / std::sqrt(nx2 * nx2 + ny2 * ny2 + nz2 * nz2);
            nx2 *= d; ny2 *= d; nz2 *= d;
            e0 = Tracer<float>::eval_bsdf(nx2, ny2, nz2, gwo.x, gwo.y, gwo.z, gnor.x, gnor.y, gnor.z, alpha2,
                                          metallic, spec_prob, galb.x, galb.y, galb.z);
            if (!(e0.pdf > 1e-12f)) early = true;
          }
        }
        double v[3] = {base[0], base[1], base[2]};
        if (!early) {
          float cos0 = nx2 * gnor.x + (ny2 * gnor.y + nz2 * gnor.z);
          const V3<double> f0 = bsdf64(mt, s, h0, nx2, ny2, nz2, gwo.x, gwo.y, gwo.z, gnor.x, gnor.y, gnor.z,
                                       metallic, spec_prob);
          FrozenFrom ff;
          ff.thr[0] = e0.r * cos0 / e0.pdf; ff.thr[1] = e0.g * cos0 / e0.pdf; ff.thr[2] = e0.b * cos0 / e0.pdf;
          ff.t64[0] = f0.x * double(cos0) / double(e0.pdf);
          ff.t64[1] = f0.y * double(cos0) / double(e0.pdf);
          ff.t64[2] = f0.z * double(cos0) / double(e0.pdf);
          ff.last_pdf = e0.pdf;
          ff.prev_b[0] = e0.r; ff.prev_b[1] = e0.g; ff.prev_b[2] = e0.b; ff.prev_cos = cos0;
          ff.prev_sumW = m_sumWu; ff.prev_M = m_M; ff.prev_delta = pdelta;
          const V3<double> a = frozen_path(pt, mt, mk(gpos.x + gnor.x * 0.001f, gpos.y + gnor.y * 0.001f,
                                                      gpos.z + gnor.z * 0.001f),
                                           mk(nx2, ny2, nz2), p.bounces - 1, &ff);
          v[0] += a.x; v[1] += a.y; v[2] += a.z;
        }
        clampd(v);
        for (int k = 0; k < 3; ++k) sum[k] += v[k];
      }
      for (int k = 0; k < 3; ++k) o[k] = sum[k] / double(p.spp);
    }
  });
  if (!env.denoise_off) {
    // the frame's denoiser on the frozen HDR, in double on the held G-buffers
    // and history colour
    std::vector<double> tmp(pixels * 3);
    temporal64(p, g.data(), hg.data(), out, hcol.data(), tmp.data(), nthreads);
    atrous64(p, g.data(), alb64.data(), tmp.data(), out, 0, nthreads);
    for (size_t i = 0; i < pixels * 3; ++i) tmp[i] = out[i];
    atrous64(p, g.data(), alb64.data(), tmp.data(), out, 1, nthreads);
  }
  return RM_OK;
}

}  // extern "C"
