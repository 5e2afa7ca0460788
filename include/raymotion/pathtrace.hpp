#pragma once
// raymotion/pathtrace.hpp - Camera and RenderConfig of the engine API.
//
// Same members, order, defaults and layout as the reference's
// include/raymotion/pathtrace.hpp:12-81 (the Camera's `get` view of references
// included, since it is part of the object).  Camera::update_trig and
// update_focal are defined by the engine (reference src/engine/camera.cpp).
#include <cstdint>
#include <functional>
#include <vector>

#include "raymotion/math.hpp"
#include "raymotion/scene.hpp"

namespace raymotion {

struct Camera {
  double x = 0, y = 0, z = 0;
  double dirx = 0, diry = 0, dirz = 0;  // degrees
  double fov = 60;                      // degrees
  double focal = 201.3839114815688;     // pixels: 240 / tan(fov / 2)
  double m0 = 1, m1 = 0, m2 = 0;
  double m3 = 0, m4 = 1, m5 = 0;
  double m6 = 0, m7 = 0, m8 = 1;
  struct VectorView {
    const double &x, &y, &z;
    operator Vec3() const { return {x, y, z}; }
  };
  struct View {
    VectorView position, rotation;
    const double& fov;
  };
  const View get{{x, y, z}, {dirx, diry, dirz}, fov};

  Camera() = default;
  Camera(const Camera& other) : Camera() { *this = other; }
  Camera& operator=(const Camera& o) {
    x = o.x; y = o.y; z = o.z;
    dirx = o.dirx; diry = o.diry; dirz = o.dirz;
    fov = o.fov; focal = o.focal;
    m0 = o.m0; m1 = o.m1; m2 = o.m2; m3 = o.m3; m4 = o.m4; m5 = o.m5; m6 = o.m6; m7 = o.m7; m8 = o.m8;
    return *this;
  }
  void update_trig();
  void update_focal();
  void set(Vec3 position = {}, Vec3 rotation = {}, double field_of_view = 60) {
    x = position.x; y = position.y; z = position.z;
    dirx = rotation.x; diry = rotation.y; dirz = rotation.z;
    fov = field_of_view;
    update_trig();
    update_focal();
  }
};

struct RenderConfig {
  int width = 640;
  int height = 360;
  int spp = 1;
  int max_bounces = 5;
  double resolution = 1;
  double clamp = 16;  // per-sample radiance clamp, 0 = off
  int adapt_min = 16;
  int adapt_step = 8;
  double adapt_rel = 0.02;
  double adapt_abs = 0.002;
  int restir_candidates = 8;
  int restir_spatial = 4;
  double restir_radius = 16;
  int restir_mcap = 128;
};

}  // namespace raymotion
