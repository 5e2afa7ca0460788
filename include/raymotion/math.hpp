#pragma once
// raymotion/math.hpp - Vec3 and degree trigonometry of the raymotion engine API.
//
// Declares the same types, with the same layout, as the reference's
// include/raymotion/math.hpp:12-68, so that code compiled against either header
// shares one ABI with librmcuda's render_image_metal.  (The reference's CPU
// xorshift Rng, math.hpp:77-112, is not used by the render path and is not
// part of this header.)
#include <cmath>
#include <cstdint>

namespace raymotion {

inline constexpr double kPi = 3.141592653589793;
inline constexpr double kFarClip = 1e30;
inline constexpr double kEps = 1e-8;
inline constexpr double kDenomEps = 1e-12;

inline double deg2rad(double d) { return d * kPi / 180.0; }
inline double rad2deg(double r) { return r * 180.0 / kPi; }
inline double cos_deg(double d) { return std::cos(deg2rad(d)); }
inline double sin_deg(double d) { return std::sin(deg2rad(d)); }
inline double tan_deg(double d) { return std::tan(deg2rad(d)); }
inline double atan_deg(double v) { return rad2deg(std::atan(v)); }
inline double gobo_mod(double a, double b) { return b == 0 ? 0 : a - std::floor(a / b) * b; }

struct Vec3 {
  double x = 0, y = 0, z = 0;
  Vec3() = default;
  Vec3(double x_, double y_, double z_) : x(x_), y(y_), z(z_) {}
  Vec3 operator+(const Vec3& o) const { return {x + o.x, y + o.y, z + o.z}; }
  Vec3 operator-(const Vec3& o) const { return {x - o.x, y - o.y, z - o.z}; }
  Vec3 operator*(double s) const { return {x * s, y * s, z * s}; }
  Vec3 operator/(double s) const { return {x / s, y / s, z / s}; }
  Vec3& operator+=(const Vec3& o) { x += o.x; y += o.y; z += o.z; return *this; }
};

inline double dot(const Vec3& a, const Vec3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline Vec3 cross(const Vec3& a, const Vec3& b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline double length(const Vec3& v) { return std::sqrt(dot(v, v)); }
inline Vec3 normalize(const Vec3& v) {
  double l = length(v);
  return l < 1e-30 ? Vec3{0, 0, 0} : v / l;
}

}  // namespace raymotion
