// shim_metal.cpp - raymotion::render_image_metal on top of the C ABI.
//
// Drop-in for the reference's Objective-C++ backend (src/engine/metal.mm:95-414):
// same signature, same validation and error strings, one process-wide context
// created on first use and serialised by a mutex (metal.mm:102-104),
// synchronous return.  The engine's fp64 Scene is packed into the fp32 records
// that metal.mm builds (metal.mm:109-145: triangles, textures in order of first
// use, the CDF as float); the BVH is the engine's own Scene::nodes, passed as
// is and converted on the device side of the ABI.  Environment switches are
// read by the library exactly as metal.mm reads them.
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "raymotion/metal.hpp"
#include "rmcuda.h"

namespace raymotion {
namespace {

struct Shared {
  std::mutex mu;
  rmcuda_ctx* ctx = nullptr;
  std::string error;
  bool tried = false;
};

Shared& shared() {
  static Shared s;  // lives for the process, like metal.mm's static Context
  return s;
}

inline rm_vec3 pack(const Vec3& v) { return rm_vec3{float(v.x), float(v.y), float(v.z)}; }

}  // namespace

bool render_image_metal(const Scene& scene, const Camera& cam, const RenderConfig& cfg, uint64_t seed,
                        std::vector<uint8_t>& output, std::string& error) {
  if (cfg.width <= 0 || cfg.height <= 0 || cfg.spp <= 0 || cfg.max_bounces < 0 ||
      size_t(cfg.width) * size_t(cfg.height) > 100000000) {
    error = "Invalid Metal render dimensions or sample count";
    return false;
  }
  Shared& sh = shared();
  std::lock_guard<std::mutex> lock(sh.mu);
  if (!sh.tried) {
    sh.tried = true;
    char e[512] = {0};
    int device = 0;
    if (const char* d = std::getenv("RAYMOTION_CUDA_DEVICE")) device = std::atoi(d);
    if (rmcuda_create(&sh.ctx, device, e, sizeof(e)) != RM_OK) {
      sh.ctx = nullptr;
      sh.error = e;
    }
  }
  if (!sh.ctx) {
    error = sh.error;
    return false;
  }
  std::vector<rm_triangle> tris(scene.tris.size());
  std::vector<rm_vec3> texels;
  std::unordered_map<const Texture*, int> offsets;
  for (size_t i = 0; i < tris.size(); ++i) {
    const Triangle& s = scene.tris[i];
    rm_triangle& t = tris[i];
    t.v0 = pack(s.v0); t.v1 = pack(s.v1); t.v2 = pack(s.v2);
    t.n = pack(s.n); t.nn = pack(s.nn);
    t.n0 = pack(s.n0); t.n1 = pack(s.n1); t.n2 = pack(s.n2);
    t.ar = float(s.ar); t.ag = float(s.ag); t.ab = float(s.ab);
    t.er = float(s.er); t.eg = float(s.eg); t.eb = float(s.eb);
    t.ior = float(s.ior); t.rough = float(s.rough); t.metallic = float(s.metallic); t.alpha = float(s.alpha);
    t.shader = s.shader;
    t.tu0 = float(s.tu0); t.tv0 = float(s.tv0); t.tu1 = float(s.tu1);
    t.tv1 = float(s.tv1); t.tu2 = float(s.tu2); t.tv2 = float(s.tv2);
    t.texture_offset = -1;
    t.texture_width = 0;
    t.texture_height = 0;
    if (s.texture) {
      auto ins = offsets.emplace(s.texture.get(), int(texels.size()));
      if (ins.second)
        for (const Vec3& px : s.texture->pixels) texels.push_back(pack(px));
      t.texture_offset = ins.first->second;
      t.texture_width = s.texture->width;
      t.texture_height = s.texture->height;
    }
  }
  std::vector<rm_bvh_node> nodes(scene.nodes.size());
  for (size_t i = 0; i < nodes.size(); ++i) {
    const BvhNode& s = scene.nodes[i];
    nodes[i] = rm_bvh_node{pack(s.mn), pack(s.mx), s.left, s.right, s.offset, s.count};
  }
  std::vector<float> cdf(scene.light_cdf.begin(), scene.light_cdf.end());
  static const rm_bvh_node kNoNodes{};
  rm_scene_view sv{};
  sv.tris = tris.data();
  sv.n_tris = int32_t(tris.size());
  // an engine scene without a BVH renders as empty, as in the reference
  sv.nodes = nodes.empty() ? &kNoNodes : nodes.data();
  sv.n_nodes = int32_t(nodes.size());
  sv.bvh_tri = scene.bvh_tri.data();
  sv.light_tri = scene.light_tri.data();
  sv.light_cdf = cdf.data();
  sv.n_lights = int32_t(scene.light_tri.size());
  sv.light_total = float(scene.light_total);
  sv.texels = texels.data();
  sv.n_texels = int64_t(texels.size());
  rm_camera c{float(cam.x), float(cam.y), float(cam.z), float(cam.focal), float(cam.m0), float(cam.m1),
              float(cam.m2), float(cam.m3), float(cam.m4), float(cam.m5), float(cam.m6), float(cam.m7),
              float(cam.m8)};
  rm_config rc{};
  rc.width = cfg.width; rc.height = cfg.height; rc.spp = cfg.spp; rc.max_bounces = cfg.max_bounces;
  rc.resolution = float(cfg.resolution); rc.clamp = float(cfg.clamp);
  rc.adapt_rel = float(cfg.adapt_rel); rc.adapt_abs = float(cfg.adapt_abs);
  rc.adapt_min = cfg.adapt_min; rc.adapt_step = cfg.adapt_step;
  rc.restir_candidates = cfg.restir_candidates; rc.restir_spatial = cfg.restir_spatial;
  rc.restir_radius = float(cfg.restir_radius); rc.restir_mcap = cfg.restir_mcap;
  rc.flags = 0;
  output.resize(size_t(cfg.width) * size_t(cfg.height) * 3);
  char e[512] = {0};
  if (rmcuda_render(sh.ctx, &sv, &c, &rc, seed, output.data(), output.size(), nullptr, e, sizeof(e)) != RM_OK) {
    error = e;
    return false;
  }
  return true;
}

}  // namespace raymotion
