// dev_math.cuh — device float3 arithmetic, PCG32 and the Duff ONB.
//
// The renderer translation unit is compiled with -fmad=false and IEEE division/sqrt, and
// every expression below keeps the operand order of the reference's Vec3 / Onb / PCGState
// (src/math/vec3.h:12-73, src/math/ray.h:95-113, src/camera/sampler.h:13-36). That makes a
// camera ray, a triangle test or a BSDF value the same float the reference CPU code computes,
// transcendental functions (CUDA's vs glibc's, both within 2 ulp) aside.
#pragma once

#include <cstdint>

namespace xbd {

constexpr float kInf = __builtin_huge_valf();
constexpr float kPi = 3.14159265358979323846f;
constexpr float kInvPi = 1.f / kPi;
constexpr float kRayEps = 1e-4f;     // src/math/ray.h:16
constexpr float kShadowEps = 5e-4f;  // src/math/ray.h:17

struct V3 {
  float x, y, z;
};

__host__ __device__ __forceinline__ V3 v3(float x, float y, float z) { return V3{x, y, z}; }
__device__ __forceinline__ V3 v3s(float s) { return V3{s, s, s}; }
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3 operator*(V3 a, V3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
__device__ __forceinline__ V3 operator/(V3 a, V3 b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
__device__ __forceinline__ V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ V3 operator*(float s, V3 a) { return {a.x * s, a.y * s, a.z * s}; }
// Vec3 / float multiplies by the reciprocal (vec3.h:27)
__device__ __forceinline__ V3 operator/(V3 a, float s) {
  float r = 1.f / s;
  return {a.x * r, a.y * r, a.z * r};
}
__device__ __forceinline__ V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
__device__ __forceinline__ float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 cross(V3 a, V3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ float length_sq(V3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
__device__ __forceinline__ float length(V3 a) { return sqrtf(length_sq(a)); }
__device__ __forceinline__ V3 normalize(V3 a) { return a / length(a); }
__device__ __forceinline__ V3 reflect(V3 v, V3 n) { return v - 2.f * dot(v, n) * n; }
__device__ __forceinline__ V3 lerp(V3 a, V3 b, float t) { return a + t * (b - a); }
__device__ __forceinline__ float comp(V3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }

// std::min / std::max / std::clamp semantics (ties and NaN resolve as libstdc++ does)
__device__ __forceinline__ float smin(float a, float b) { return (b < a) ? b : a; }
__device__ __forceinline__ float smax(float a, float b) { return (a < b) ? b : a; }
__device__ __forceinline__ float sclamp(float v, float lo, float hi) {
  return (v < lo) ? lo : ((hi < v) ? hi : v);
}
// std::max({x, y, z}) (max_element keeps the first of equals)
__device__ __forceinline__ float max_component(V3 v) {
  float r = v.x;
  if (r < v.y) r = v.y;
  if (r < v.z) r = v.z;
  return r;
}

__device__ __forceinline__ V3 ld3(const float4& f) { return V3{f.x, f.y, f.z}; }

// offset_ray_origin (src/math/ray.h:22-26)
__device__ __forceinline__ V3 offset_origin(V3 p, V3 ng, V3 dir, float eps) {
  V3 n = ng;
  if (dot(n, dir) < 0.f) n = -n;
  return p + n * eps;
}

// Orthonormal basis, Duff et al. 2017 (src/math/ray.h:95-113)
struct Onb {
  V3 u, v, n;
  __device__ __forceinline__ explicit Onb(V3 nn) : n(nn) {
    float s = (n.z >= 0.f) ? 1.f : -1.f;
    float a = -1.f / (s + n.z);
    float b = n.x * n.y * a;
    u = v3(1.f + s * n.x * n.x * a, s * b, -s * n.x);
    v = v3(b, s + n.y * n.y * a, -n.y);
  }
  __device__ __forceinline__ V3 to_world(V3 l) const { return l.x * u + l.y * v + l.z * n; }
  __device__ __forceinline__ V3 to_local(V3 w) const { return v3(dot(w, u), dot(w, v), dot(w, n)); }
};

// PCG-XSH-RR 32 with increment 1 (seed_pcg with seq 0), src/camera/sampler.h:13-36.
struct Pcg {
  uint64_t state;
  __device__ __forceinline__ uint32_t next_uint() {
    uint64_t old = state;
    state = old * 6364136223846793005ULL + 1ULL;
    uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    uint32_t rot = (uint32_t)(old >> 59u);
    return (xs >> rot) | (xs << ((~rot + 1u) & 31u));
  }
  __device__ __forceinline__ float next_float() {
    return (float)(next_uint() >> 8) * (1.f / 16777216.f);
  }
};

__host__ __device__ __forceinline__ uint64_t pcg_seed_state(uint64_t seed) {
  // seed_pcg: state 0 → step → += seed → step, with increment 1
  uint64_t s = 0ULL * 6364136223846793005ULL + 1ULL;
  s += seed;
  return s * 6364136223846793005ULL + 1ULL;
}

}  // namespace xbd
