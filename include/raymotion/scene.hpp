#pragma once
// raymotion/scene.hpp - the engine's fp64 scene, as the backend receives it.
//
// Same members, order and types as the reference's
// include/raymotion/scene.hpp:26-96 (Texture, Triangle with an inline material,
// BvhNode, Scene): render_image_metal reads these objects directly, so the
// layout is an ABI shared with the engine.  Scene::add_triangle and
// Texture::sample are defined by the engine (reference src/engine/scene.cpp).
#include <cstddef>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "raymotion/math.hpp"

namespace raymotion {

struct Texture {
  int width = 0, height = 0;
  std::vector<Vec3> pixels;  // linear RGB, top row first
  Vec3 sample(double u, double v) const;
};

struct Triangle {
  std::shared_ptr<const Texture> texture;
  Vec3 v0, v1, v2;
  Vec3 n;  // (v1 - v0) x (v2 - v0)
  double d = 0;
  Vec3 U, V;
  double denom = 0;
  Vec3 nn;  // normalize(n)
  double tu0 = 0, tv0 = 0, tu1 = 0, tv1 = 0, tu2 = 0, tv2 = 0;
  Vec3 n0, n1, n2;  // vertex normals
  Vec3 mn, mx;      // bounds
  double ar = 1, ag = 1, ab = 1;
  double er = 0, eg = 0, eb = 0;
  double ior = 1;    // dielectric when > 1.0001
  double alpha = 1;  // coverage in [0, 1]
  double rough = 0.5;
  int shader = 0;  // 1: HSV "rainbow" albedo
  double metallic = 0;
};

struct BvhNode {
  Vec3 mn, mx;
  int left = -1;    // internal nodes
  int right = -1;   // internal nodes
  int offset = -1;  // leaves: first entry in Scene::bvh_tri
  int count = 0;    // leaves: triangle count (0 for internal nodes)
  bool is_leaf() const { return count > 0; }
};

struct Scene {
  std::vector<Triangle> tris;
  std::vector<BvhNode> nodes;
  std::vector<int> bvh_tri;
  int max_leaf_tris = 8;
  std::vector<int> light_tri;
  std::vector<double> light_cdf;
  double light_total = 0;

  void clear_triangles() { tris.clear(); light_tri.clear(); light_cdf.clear(); light_total = 0; }
  void clear_bvh() { nodes.clear(); bvh_tri.clear(); }
  int add_triangle(const Vec3& p0, const Vec3& p1, const Vec3& p2, double u0, double v0, double u1, double v1,
                   double u2, double v2, const Vec3& n0, const Vec3& n1, const Vec3& n2, double ar, double ag,
                   double ab, double er, double eg, double eb, double metallic, double ior, double rough, int shader,
                   double alpha = 1);
};

}  // namespace raymotion
