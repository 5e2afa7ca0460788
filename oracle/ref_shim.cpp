// ref_shim.cpp - C entry points over the reference's own CPU engine code.
//
// TEST INFRASTRUCTURE ONLY.  Compiled together with the reference sources
// src/engine/{scene,bvh,camera}.cpp where they lie (never copied into this
// repository) into oracle/_ref/libref.so, so that the tests can pin the oracle
// and the numpy scene builder against the reference itself:
//   Scene::add_triangle (src/engine/scene.cpp:16-87), build_bvh / refit_bvh
//   (src/engine/bvh.cpp:29-272), Camera::update_trig / update_focal
//   (src/engine/camera.cpp:3-22).
#include <cmath>
#include <cstdint>
#include <optional>
#include <cstring>

#include "raymotion/bvh.hpp"
#include "raymotion/pathtrace.hpp"
#include "raymotion/scene.hpp"

using namespace raymotion;

namespace {
struct RefScene { Scene s; };
}

extern "C" {

void* ref_scene_new() { return new RefScene(); }
void ref_scene_free(void* h) { delete static_cast<RefScene*>(h); }

// rec: 3*3 positions, 6 uvs, 3*3 normals, ar ag ab er eg eb metallic ior rough alpha (34 doubles) + shader
int ref_add_triangle(void* h, const double* r, int shader) {
  Scene& s = static_cast<RefScene*>(h)->s;
  return s.add_triangle({r[0], r[1], r[2]}, {r[3], r[4], r[5]}, {r[6], r[7], r[8]}, r[9], r[10], r[11], r[12], r[13],
                        r[14], {r[15], r[16], r[17]}, {r[18], r[19], r[20]}, {r[21], r[22], r[23]}, r[24], r[25], r[26],
                        r[27], r[28], r[29], r[30], r[31], r[32], shader, r[33]);
}

int ref_tri_count(void* h) { return int(static_cast<RefScene*>(h)->s.tris.size()); }

// Per triangle 33 doubles: v0 v1 v2 n nn n0 n1 n2 (24), ar ag ab er eg eb ior rough metallic alpha (10)... minus one:
// layout: v0,v1,v2,n,nn,n0,n1,n2 (24) + ar,ag,ab,er,eg,eb,ior,rough,metallic,alpha (10) = 34
void ref_tri_read(void* h, double* out) {
  const Scene& s = static_cast<RefScene*>(h)->s;
  for (size_t i = 0; i < s.tris.size(); ++i) {
    const Triangle& t = s.tris[i];
    double* o = out + i * 34;
    const Vec3* vs[8] = {&t.v0, &t.v1, &t.v2, &t.n, &t.nn, &t.n0, &t.n1, &t.n2};
    for (int k = 0; k < 8; ++k) { o[k * 3] = vs[k]->x; o[k * 3 + 1] = vs[k]->y; o[k * 3 + 2] = vs[k]->z; }
    double m[10] = {t.ar, t.ag, t.ab, t.er, t.eg, t.eb, t.ior, t.rough, t.metallic, t.alpha};
    std::memcpy(o + 24, m, sizeof(m));
  }
}

int ref_light_count(void* h) { return int(static_cast<RefScene*>(h)->s.light_tri.size()); }
double ref_lights(void* h, int32_t* tri, double* cdf) {
  const Scene& s = static_cast<RefScene*>(h)->s;
  for (size_t i = 0; i < s.light_tri.size(); ++i) { tri[i] = s.light_tri[i]; cdf[i] = s.light_cdf[i]; }
  return s.light_total;
}

int ref_build_bvh(void* h, int max_leaf) {
  Scene& s = static_cast<RefScene*>(h)->s;
  build_bvh(s, max_leaf);
  return int(s.nodes.size());
}
void ref_refit_bvh(void* h) { refit_bvh(static_cast<RefScene*>(h)->s); }
int ref_node_count(void* h) { return int(static_cast<RefScene*>(h)->s.nodes.size()); }
// nodes: {mn, mx} doubles; links: {left, right, offset, count}
void ref_nodes(void* h, double* bounds, int32_t* links, int32_t* bvh_tri) {
  const Scene& s = static_cast<RefScene*>(h)->s;
  for (size_t i = 0; i < s.nodes.size(); ++i) {
    const BvhNode& n = s.nodes[i];
    double b[6] = {n.mn.x, n.mn.y, n.mn.z, n.mx.x, n.mx.y, n.mx.z};
    std::memcpy(bounds + i * 6, b, sizeof(b));
    links[i * 4] = n.left; links[i * 4 + 1] = n.right; links[i * 4 + 2] = n.offset; links[i * 4 + 3] = n.count;
  }
  for (size_t i = 0; i < s.bvh_tri.size(); ++i) bvh_tri[i] = s.bvh_tri[i];
}
// Replace vertex positions (n*9 doubles) of existing triangles, recomputing
// their AABBs the way add_triangle does (scene.cpp:55-58); for refit tests.
void ref_move_vertices(void* h, const double* v) {
  Scene& s = static_cast<RefScene*>(h)->s;
  for (size_t i = 0; i < s.tris.size(); ++i) {
    Triangle& t = s.tris[i];
    const double* p = v + i * 9;
    t.v0 = {p[0], p[1], p[2]}; t.v1 = {p[3], p[4], p[5]}; t.v2 = {p[6], p[7], p[8]};
    t.mn = {std::min({p[0], p[3], p[6]}), std::min({p[1], p[4], p[7]}), std::min({p[2], p[5], p[8]})};
    t.mx = {std::max({p[0], p[3], p[6]}), std::max({p[1], p[4], p[7]}), std::max({p[2], p[5], p[8]})};
  }
}

// Camera (camera.cpp): out = focal, m0..m8
void ref_camera(double x, double y, double z, double rx, double ry, double rz, double fov, double* out) {
  Camera c;
  c.set({x, y, z}, {rx, ry, rz}, fov);
  double m[10] = {c.focal, c.m0, c.m1, c.m2, c.m3, c.m4, c.m5, c.m6, c.m7, c.m8};
  std::memcpy(out, m, sizeof(m));
}

// One Objects::push + Objects::append (include/raymotion/runtime.hpp:76-113)
// into the scene: the instance's model triangles `model` (n records in the
// layout of ref_add_triangle, shaders in `shader`), placed with
// inst = position[3], rotation[3] (degrees), scale[3], albedo[3],
// emission[3], refract, rough, metallic, alpha (NaN: unset).  The transform
// uses the reference's own cos_deg / sin_deg / normalize (math.hpp) and its
// order of operations (Objects::append is private, so its three lambdas are
// restated here); add_triangle is the reference's.
void ref_append_instance(void* h, const double* model, const int* shader, int n, const double* inst) {
  Scene& s = static_cast<RefScene*>(h)->s;
  const Vec3 position{inst[0], inst[1], inst[2]}, rotation{inst[3], inst[4], inst[5]}, scale{inst[6], inst[7], inst[8]};
  const Vec3 albedo{inst[9], inst[10], inst[11]}, emission{inst[12], inst[13], inst[14]};
  auto opt = [](double v) { return std::isnan(v) ? std::optional<double>() : std::optional<double>(v); };
  const std::optional<double> refract = opt(inst[15]), rough = opt(inst[16]), metallic = opt(inst[17]),
                              alpha = opt(inst[18]);
  const double cx = cos_deg(rotation.x), sx = sin_deg(rotation.x);
  const double cy = cos_deg(rotation.y), sy = sin_deg(rotation.y);
  const double cz = cos_deg(rotation.z), sz = sin_deg(rotation.z);
  auto rotate = [&](Vec3 v) {
    double c = cx, si = sx;
    v = {v.x, c * v.y - si * v.z, si * v.y + c * v.z};
    c = cy; si = sy;
    v = {c * v.x + si * v.z, v.y, -si * v.x + c * v.z};
    c = cz; si = sz;
    return Vec3{c * v.x - si * v.y, si * v.x + c * v.y, v.z};
  };
  auto point = [&](Vec3 v) { return rotate({v.x * scale.x, v.y * scale.y, v.z * scale.z}) + position; };
  auto normal = [&](Vec3 v) { return normalize(rotate({v.x / scale.x, v.y / scale.y, v.z / scale.z})); };
  for (int i = 0; i < n; ++i) {
    const double* r = model + size_t(i) * 34;
    const Vec3 v0{r[0], r[1], r[2]}, v1{r[3], r[4], r[5]}, v2{r[6], r[7], r[8]};
    const Vec3 n0{r[15], r[16], r[17]}, n1{r[18], r[19], r[20]}, n2{r[21], r[22], r[23]};
    s.add_triangle(point(v0), point(v1), point(v2), r[9], r[10], r[11], r[12], r[13], r[14], normal(n0), normal(n1),
                   normal(n2), albedo.x < 0 ? r[24] : albedo.x, albedo.y < 0 ? r[25] : albedo.y,
                   albedo.z < 0 ? r[26] : albedo.z, emission.x < 0 ? r[27] : emission.x,
                   emission.y < 0 ? r[28] : emission.y, emission.z < 0 ? r[29] : emission.z,
                   metallic.value_or(r[30]), refract.value_or(r[31]), rough.value_or(r[32]), shader[i],
                   alpha.value_or(r[33]));
  }
}

}  // extern "C"
