// host_math.h — float3 / AABB arithmetic for the host-side scene build.
//
// Every operation keeps the operand order of the reference's Vec3 and AABB
// (src/math/vec3.h:12-73, src/geometry/aabb.h:14-38) and this file is compiled without
// FMA contraction, so BVH bounds, SAH costs and bin indices come out bit-identical to the
// reference build; the device receives exactly the node arrays the reference would build.
#pragma once

#include <cmath>
#include <cstdint>
#include <limits>

namespace xb {

constexpr float kInf = std::numeric_limits<float>::infinity();
constexpr float kPiF = 3.14159265358979323846f;

struct F3 {
  float x = 0.f, y = 0.f, z = 0.f;
  F3() = default;
  constexpr F3(float a, float b, float c) : x(a), y(b), z(c) {}
  static constexpr F3 splat(float s) { return F3(s, s, s); }
  float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
  float& at(int i) { return i == 0 ? x : (i == 1 ? y : z); }
};

inline F3 operator+(F3 a, F3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline F3 operator-(F3 a, F3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline F3 operator*(F3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline F3 operator*(float s, F3 a) { return a * s; }
inline F3 operator-(F3 a) { return {-a.x, -a.y, -a.z}; }
// v / s is v * (1/s) in the reference (vec3.h:27)
inline F3 div_scalar(F3 a, float s) { float r = 1.f / s; return {a.x * r, a.y * r, a.z * r}; }
inline float dot3(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline F3 cross3(F3 a, F3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline float len3(F3 a) { return std::sqrt(dot3(a, a)); }
inline F3 normalize3(F3 a) { return div_scalar(a, len3(a)); }
// std::min / std::max semantics: min(a,b) = (b < a) ? b : a, max(a,b) = (a < b) ? b : a
inline float smin(float a, float b) { return (b < a) ? b : a; }
inline float smax(float a, float b) { return (a < b) ? b : a; }
inline F3 min3(F3 a, F3 b) { return {smin(a.x, b.x), smin(a.y, b.y), smin(a.z, b.z)}; }
inline F3 max3(F3 a, F3 b) { return {smax(a.x, b.x), smax(a.y, b.y), smax(a.z, b.z)}; }
inline F3 lerp3(F3 a, F3 b, float t) { return a + t * (b - a); }
inline int max_axis3(F3 v) { return (v.x > v.y && v.x > v.z) ? 0 : (v.y > v.z ? 1 : 2); }

struct Bounds {
  F3 mn = F3::splat(kInf);
  F3 mx = F3::splat(-kInf);
  void grow(F3 p) { mn = min3(mn, p); mx = max3(mx, p); }
  void grow(const Bounds& b) { mn = min3(mn, b.mn); mx = max3(mx, b.mx); }
  F3 center() const { return (mn + mx) * 0.5f; }
  F3 extent() const { return mx - mn; }
  float area() const {
    F3 e = extent();
    return 2.f * (e.x * e.y + e.y * e.z + e.z * e.x);
  }
};

// Column-major 3x4 affine matrix (src/geometry/transform.h:32-63): c0..c2 basis, c3 translation.
struct Affine {
  F3 c[4];
  static Affine identity() {
    Affine a;
    a.c[0] = {1, 0, 0}; a.c[1] = {0, 1, 0}; a.c[2] = {0, 0, 1}; a.c[3] = {0, 0, 0};
    return a;
  }
  F3 point(F3 p) const { return c[0] * p.x + c[1] * p.y + c[2] * p.z + c[3]; }
};

}  // namespace xb
