// dev_scene.cuh — the scene as laid out in HBM, and its traversal.
//
// Layout (all read-only, loaded through the non-coherent path):
//   blas      float4[2 * N]: node i = {mn.x, mn.y, mn.z, mx.x}, {mx.y, mx.z, child, count}.
//             All meshes' BLAS arrays are concatenated; each mesh's nodes start at an odd
//             index so that every child pair (left, left+1) is one 64-byte aligned block:
//             an internal node costs one 64 B pair load, as in the reference's two-child
//             test (src/geometry/blas.cpp:103-152). child fields are global indices.
//   tris      float4[3 * S]: the triangle of BLAS prim slot s, pre-gathered in slot order
//             {v0, local tri id}, {v1, global tri id}, {v2, -}: a leaf's triangles are
//             contiguous 48 B records (src/geometry/mesh.h:37-44 gather, done once on upload).
//   pnodes    the PrimBLAS nodes, same 32 B records; prims the analytic primitives.
//   tlas      TLAS nodes, 32 B each; inst the instances (world_to_local + BLAS root).
//
// Traversal restates the reference's order and float semantics exactly:
//   BLAS closest / any       src/geometry/blas.cpp:211-307 (+ aabb_pair_sse :25-74)
//   TLAS closest / any       src/geometry/tlas.cpp:172-290 (+ AABB::intersect_fast aabb.h:59-71)
//   PrimBLAS closest / any   src/geometry/prim_blas.cpp:142-229 (+ AABB::intersect aabb.h:41-56)
//   Moller-Trumbore          src/geometry/primitives.h:25-49
//   analytic prims           src/geometry/primitives.h:54-318
//   hit fix-up               src/geometry/tlas.cpp:156-168, mesh.h:104-129
#pragma once

#include "dev_math.cuh"

namespace xbd {

constexpr int kStackSize = 64;   // BLAS / TLAS / PrimBLAS stacks are 64 deep in the reference
constexpr int kShStride = 128;   // threads per block of every traversal kernel
constexpr int kSharedStack = 16; // BLAS stack entries the shared-stack kernels keep in shared memory

// The BLAS / PrimBLAS traversal stack. Its first NSH entries live in shared memory (entry k of
// thread t at sh[k * kShStride + t]: a warp's 32 accesses fall in 32 distinct banks at any mix of
// depths), the rest in the thread's local array (entries k >= NSH at loc[k]). NSH = 0 keeps the
// whole stack in local memory and compiles to plain local-array accesses.
template <int NSH>
struct BStack {
  uint32_t* sh;
  uint32_t* loc;
  __device__ __forceinline__ uint32_t get(int k) const {
    if constexpr (NSH == 0) return loc[k];
    else return k < NSH ? sh[k * kShStride] : loc[k];
  }
  __device__ __forceinline__ void put(int k, uint32_t v) const {
    if constexpr (NSH == 0) loc[k] = v;
    else if (k < NSH) sh[k * kShStride] = v;
    else loc[k] = v;
  }
};

struct DevInstance {     // 64 bytes
  float w2l[12];         // world_to_local, columns c0 c1 c2 c3
  int32_t kind;          // 0 = triangle BLAS, 1 = prim BLAS
  int32_t root;          // global index of the BLAS root node
  int32_t instance_id;
  int32_t mesh;          // mesh index (kind 0)
};

struct DevMaterial {     // derived principled parameters used by the BSDF
  float base[3];
  float metallic;
  float ior;
  float alpha, alpha_x, alpha_y;
  float f0[3];
  float subsurface;
  float ss_color[3];
  int32_t flags;         // XB_MAT_* bits
  float ms_k1, ms_k2;    // multiple scattering: 5 exp(-2.69 a), 1 + 22.7 a^1.5
  float ms_fms[3];       // F_avg^2 E_avg / denom
};

struct DevLight {        // one emitting triangle, vertices in world space (scene.meshes[mesh_id])
  float4 p0;             // xyz, w = area
  float4 p1;             // xyz, w = bits(mesh_id)
  float4 p2;             // xyz, w = bits(tri_idx)
  float4 n;              // geo_normal(tri) xyz
  float4 emission;       // xyz
};

struct DevSun {
  float dir[3];
  float emission[3];     // color * intensity
};

struct DevMesh {
  int32_t tri_offset;    // first global triangle
  int32_t vtx_offset;    // first global vertex
  int32_t has_normals;
  int32_t pad;
};

struct DevScene {
  const float4* blas;
  const float4* tris;
  const float4* pnodes;
  const float4* prims;       // 4 float4 per prim slot: {type, mat, prim index, -}, p0..p3, p4..p7, p8 p9
  const float4* tlas;
  const uint32_t* tlas_inst;
  const DevInstance* inst;
  const DevMesh* meshes;
  const int32_t* tri_index;  // 3 global vertex ids per global triangle
  const int32_t* tri_mat;    // per global triangle
  const float* nx;           // per global vertex, shading normals
  const float* ny;
  const float* nz;
  const DevMaterial* mats;
  const DevLight* lights;
  const DevSun* suns;
  int32_t num_lights;
  int32_t num_suns;
  int32_t num_tlas_nodes;
  int32_t num_materials;
  float sky_zenith[3], sky_horizon[3], sky_ground[3];
  float sky_inv_sharpness;
  float sky_intensity;
  int32_t sun_nee;   // XB_FLAG_SUN_NEE: directional lights weighted as delta lights (else the reference's 1e8)
  const float* sky_cdf;   // XB_FLAG_SKY_IS: kSkyBins + 1 cumulative bin masses over y in [-1, 1] (or nullptr)
  int32_t watertight;     // XB_FLAG_WATERTIGHT: ray_triangle_wt instead of Moller-Trumbore
};

// The sky's luminance distribution over directions. The gradient sky (Environment::evaluate)
// depends on the direction's y alone, so its distribution is a piecewise-constant density of y
// over kSkyBins equal bins of [-1, 1] times a uniform azimuth: pdf(w) = mass(bin(w.y)) / (dy 2 pi).
constexpr int kSkyBins = 256;

__device__ __forceinline__ float sky_pdf(const float* cdf, V3 d) {
  int b = (int)((d.y + 1.f) * (0.5f * kSkyBins));
  b = b < 0 ? 0 : (b > kSkyBins - 1 ? kSkyBins - 1 : b);
  return (__ldg(cdf + b + 1) - __ldg(cdf + b)) * ((float)kSkyBins / (4.f * 3.14159265358979f));
}

__device__ __forceinline__ V3 sky_sample(const float* cdf, float u0, float u1) {
  int lo = 0, hi = kSkyBins;                 // the bin b with cdf[b] <= u0 < cdf[b + 1]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(cdf + mid) <= u0) lo = mid;
    else hi = mid;
  }
  const float c0 = __ldg(cdf + lo), c1 = __ldg(cdf + lo + 1);
  const float t = c1 > c0 ? fminf(fmaxf((u0 - c0) / (c1 - c0), 0.f), 1.f) : 0.5f;
  const float y = fminf(fmaxf(-1.f + ((float)lo + t) * (2.f / kSkyBins), -1.f), 1.f);
  const float rr = sqrtf(fmaxf(0.f, 1.f - y * y));
  float sp, cp;
  sincospif(2.f * u1, &sp, &cp);
  return v3(rr * cp, y, rr * sp);
}

struct Ray {
  V3 o, d;
  float tmin, tmax;
};

// Closest-hit state kept during traversal; everything else is rebuilt afterwards.
struct HitState {
  float t, u, v;
  int32_t prim;    // triangle: BLAS slot; analytic: prim index
  int32_t inst;    // instance index (-1: no hit)
};

struct TraversalCounters {
  uint32_t nodes;  // internal BLAS nodes expanded (each loads its 64 B child pair)
  uint32_t tris;   // triangle tests (48 B each)
  uint32_t tlas;   // TLAS nodes tested (32 B each)
  uint32_t inst;   // instance visits (world_to_local, 48 B)
};

__device__ __forceinline__ float4 ldg4(const float4* p) { return __ldg(p); }

// BLAS stack entries carry the node's own (child, count) — both already loaded with the
// parent's 64 B child pair — so popping needs no further node load: count in the top 4 bits,
// child (a node or triangle-slot index < 2^28) below. A count >= 15 (only degenerate leaves)
// stores the node index instead, marked by 15, and the node is re-read when popped.
constexpr uint32_t kEntryEscape = 15u;
__device__ __forceinline__ uint32_t blas_entry(uint32_t child, uint32_t count, uint32_t node) {
  return count < kEntryEscape ? ((count << 28) | child) : ((kEntryEscape << 28) | node);
}
__device__ __forceinline__ void blas_unpack(const DevScene& sc, uint32_t e, uint32_t& child,
                                            uint32_t& count) {
  count = e >> 28;
  child = e & 0x0fffffffu;
  if (count == kEntryEscape) {
    const float4 nb = __ldg(sc.blas + 2 * (size_t)child + 1);
    child = __float_as_uint(nb.z);
    count = __float_as_uint(nb.w);
  }
}
__device__ __forceinline__ uint32_t blas_root_entry(const DevScene& sc, int root) {
  const float4 nb = __ldg(sc.blas + 2 * (size_t)root + 1);
  return blas_entry(__float_as_uint(nb.z), __float_as_uint(nb.w), (uint32_t)root);
}

// ── world → local (AffineTransform::to_local, transform.h:44-51) ────────────────
__device__ __forceinline__ Ray to_local(const DevInstance& in, const Ray& w) {
  const float* c = in.w2l;
  V3 c0 = v3(c[0], c[1], c[2]), c1 = v3(c[3], c[4], c[5]), c2 = v3(c[6], c[7], c[8]),
     c3 = v3(c[9], c[10], c[11]);
  Ray r;
  r.o = c0 * w.o.x + c1 * w.o.y + c2 * w.o.z + c3;
  r.d = c0 * w.d.x + c1 * w.d.y + c2 * w.d.z;
  r.tmin = w.tmin;
  r.tmax = w.tmax;
  return r;
}

// normal_to_world: normalize(world_to_local.transform_normal(n)) (transform.h:41-45, 56-58)
__device__ __forceinline__ V3 normal_to_world(const DevInstance& in, V3 n) {
  const float* c = in.w2l;
  V3 r = v3(c[0] * n.x + c[1] * n.y + c[2] * n.z, c[3] * n.x + c[4] * n.y + c[5] * n.z,
            c[6] * n.x + c[7] * n.y + c[8] * n.z);
  return normalize(r);
}

// ── Moller-Trumbore (primitives.h:25-49); accepts t in [tmin, t_max] ─────────────
__device__ __forceinline__ bool ray_triangle(V3 o, V3 d, float tmin, V3 v0, V3 v1, V3 v2,
                                             float t_max, float& t, float& u, float& v) {
  V3 e1 = v1 - v0;
  V3 e2 = v2 - v0;
  V3 h = cross(d, e2);
  float a = dot(e1, h);
  if (fabsf(a) < 1e-7f) return false;
  float inv_a = 1.f / a;
  V3 s = o - v0;
  u = inv_a * dot(s, h);
  if (u < 0.f || u > 1.f) return false;
  V3 q = cross(s, e1);
  v = inv_a * dot(d, q);
  if (v < 0.f || u + v > 1.f) return false;
  t = inv_a * dot(e2, q);
  return t >= tmin && t <= t_max;
}

// Watertight ray-triangle test (Woop, Benthin, Wald, "Watertight Ray/Triangle Intersection",
// JCGT 2(1), 2013): the vertices are translated to the ray origin and sheared so that the ray
// runs along +z; the 2D edge functions U, V, W then decide the hit. Two triangles that share an
// edge evaluate its edge function from the same two transformed vertices, in opposite order, so
// (with no fused multiply-add: this file is compiled with -fmad=false) the values are exact
// negatives and a ray cannot pass between them. A zero edge function is re-evaluated in FP64.
// Same interface as ray_triangle (u, v: the weights of v1 and v2), and the same acceptance
// tmin <= t <= t_max; inv = 1 / d.
__device__ __forceinline__ bool ray_triangle_wt(V3 o, V3 d, V3 inv, float tmin, V3 v0, V3 v1, V3 v2,
                                                float t_max, float& t, float& u, float& v) {
  const float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
  const int kz = (ax > ay && ax > az) ? 0 : (ay > az ? 1 : 2);
  int kx = kz == 2 ? 0 : kz + 1, ky = kx == 2 ? 0 : kx + 1;
  const float dz = comp(d, kz);
  if (dz < 0.f) { const int k = kx; kx = ky; ky = k; }   // keeps the winding
  const float sz = comp(inv, kz);
  const float sx = comp(d, kx) * sz, sy = comp(d, ky) * sz;
  const V3 A = v0 - o, B = v1 - o, C = v2 - o;
  const float Ax = comp(A, kx) - sx * comp(A, kz), Ay = comp(A, ky) - sy * comp(A, kz);
  const float Bx = comp(B, kx) - sx * comp(B, kz), By = comp(B, ky) - sy * comp(B, kz);
  const float Cx = comp(C, kx) - sx * comp(C, kz), Cy = comp(C, ky) - sy * comp(C, kz);
  float U = Cx * By - Cy * Bx;
  float V = Ax * Cy - Ay * Cx;
  float W = Bx * Ay - By * Ax;
  if (U == 0.f || V == 0.f || W == 0.f) {
    U = (float)((double)Cx * (double)By - (double)Cy * (double)Bx);
    V = (float)((double)Ax * (double)Cy - (double)Ay * (double)Cx);
    W = (float)((double)Bx * (double)Ay - (double)By * (double)Ax);
  }
  if ((U < 0.f || V < 0.f || W < 0.f) && (U > 0.f || V > 0.f || W > 0.f)) return false;
  const float det = U + V + W;
  if (det == 0.f) return false;
  const float T = U * (sz * comp(A, kz)) + V * (sz * comp(B, kz)) + W * (sz * comp(C, kz));
  const float rdet = 1.f / det;
  t = T * rdet;
  if (!(t >= tmin && t <= t_max)) return false;
  u = V * rdet;
  v = W * rdet;
  return true;
}

// The scene's triangle test: Moller-Trumbore (the reference's, bit-exact), or the watertight one.
__device__ __forceinline__ bool tri_hit(const DevScene& sc, V3 o, V3 d, V3 inv, float tmin, V3 v0, V3 v1,
                                        V3 v2, float t_max, float& t, float& u, float& v) {
  if (sc.watertight) return ray_triangle_wt(o, d, inv, tmin, v0, v1, v2, t_max, t, u, v);
  return ray_triangle(o, d, tmin, v0, v1, v2, t_max, t, u, v);
}

// SSE minps / maxps: (a < b) ? a : b and (a > b) ? a : b (NaN → second operand)
__device__ __forceinline__ float mmin(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float mmax(float a, float b) { return a > b ? a : b; }

// aabb_pair_sse for one child: returns near t via tn, hit flag
__device__ __forceinline__ bool slab_sse(float4 a, float4 b, V3 inv, V3 org, float tmin,
                                         float tmax, float& tn) {
  // a = {mn.x, mn.y, mn.z, mx.x}, b = {mx.y, mx.z, ...}
  float t0x = (a.x - org.x) * inv.x, t1x = (a.w - org.x) * inv.x;
  float t0y = (a.y - org.y) * inv.y, t1y = (b.x - org.y) * inv.y;
  float t0z = (a.z - org.z) * inv.z, t1z = (b.y - org.z) * inv.z;
  float lx = mmin(t0x, t1x), ly = mmin(t0y, t1y), lz = mmin(t0z, t1z);
  float hx = mmax(t0x, t1x), hy = mmax(t0y, t1y), hz = mmax(t0z, t1z);
  float tnear = mmax(mmax(mmax(lx, ly), lz), tmin);
  float tfar = mmin(mmin(mmin(hx, hy), hz), tmax);
  tn = tnear;
  return tnear <= tfar;
}

// AABB::intersect_fast (aabb.h:59-71) with std::max/min over initializer lists
__device__ __forceinline__ bool aabb_fast(float4 a, float4 b, V3 inv, V3 org, const int sign[3],
                                          float tmin, float tmax) {
  float mnx = a.x, mny = a.y, mnz = a.z, mxx = a.w, mxy = b.x, mxz = b.y;
  float txmin = ((sign[0] ? mxx : mnx) - org.x) * inv.x;
  float txmax = ((sign[0] ? mnx : mxx) - org.x) * inv.x;
  float tymin = ((sign[1] ? mxy : mny) - org.y) * inv.y;
  float tymax = ((sign[1] ? mny : mxy) - org.y) * inv.y;
  float tzmin = ((sign[2] ? mxz : mnz) - org.z) * inv.z;
  float tzmax = ((sign[2] ? mnz : mxz) - org.z) * inv.z;
  float lo = tmin;
  if (lo < txmin) lo = txmin;
  if (lo < tymin) lo = tymin;
  if (lo < tzmin) lo = tzmin;
  float hi = tmax;
  if (txmax < hi) hi = txmax;
  if (tymax < hi) hi = tymax;
  if (tzmax < hi) hi = tzmax;
  return lo <= hi;
}

// AABB::intersect (aabb.h:41-56): division slabs, std::max / std::min folds
__device__ __forceinline__ bool aabb_div(float4 a, float4 b, const Ray& r, float& tn) {
  float tx0 = (a.x - r.o.x) / r.d.x, tx1 = (a.w - r.o.x) / r.d.x;
  float ty0 = (a.y - r.o.y) / r.d.y, ty1 = (b.x - r.o.y) / r.d.y;
  float tz0 = (a.z - r.o.z) / r.d.z, tz1 = (b.y - r.o.z) / r.d.z;
  float lo = smin(tx0, tx1);
  float e = smin(ty0, ty1); if (lo < e) lo = e;
  e = smin(tz0, tz1); if (lo < e) lo = e;
  if (lo < r.tmin) lo = r.tmin;
  float hi = smax(tx0, tx1);
  e = smax(ty0, ty1); if (e < hi) hi = e;
  e = smax(tz0, tz1); if (e < hi) hi = e;
  if (r.tmax < hi) hi = r.tmax;
  tn = lo;
  return lo <= hi;
}

// ── analytic primitives (primitives.h:54-318) ───────────────────────────────────
// Returns the hit t (and for boxes the entering face) if t is in [tmin, best) — strict
// upper bound, unlike triangles.
struct PrimHit {
  float t;
  int face;   // box: near_axis | (near_min_face << 2)
};

__device__ __forceinline__ bool prim_intersect(const float4* pr, const Ray& r, float best,
                                               PrimHit& out) {
  const float4 h0 = ldg4(pr), h1 = ldg4(pr + 1), h2 = ldg4(pr + 2), h3 = ldg4(pr + 3);
  const int type = __float_as_int(h0.x);
  const float p[10] = {h1.x, h1.y, h1.z, h1.w, h2.x, h2.y, h2.z, h2.w, h3.x, h3.y};
  if (type == 0) {  // sphere
    V3 c = v3(p[0], p[1], p[2]);
    float rad = p[3];
    V3 oc = r.o - c;
    float a = dot(r.d, r.d);
    float hb = dot(oc, r.d);
    float cc = dot(oc, oc) - rad * rad;
    float disc = hb * hb - a * cc;
    if (disc < 0.f) return false;
    float sq = sqrtf(disc);
    float t = (-hb - sq) / a;
    if (t < r.tmin || t >= best) {
      t = (-hb + sq) / a;
      if (t < r.tmin || t >= best) return false;
    }
    out.t = t; out.face = 0;
    return true;
  } else if (type == 1) {  // plane
    V3 n = v3(p[0], p[1], p[2]);
    float denom = dot(n, r.d);
    if (fabsf(denom) < 1e-7f) return false;
    float t = (p[3] - dot(n, r.o)) / denom;
    if (t < r.tmin || t >= best) return false;
    out.t = t; out.face = 0;
    return true;
  } else if (type == 2) {  // box
    V3 c = v3(p[0], p[1], p[2]), hh = v3(p[3], p[4], p[5]);
    V3 mn = c - hh, mx = c + hh;
    float tmn = r.tmin, tmx = best;
    int axis = 0, minface = 0;
    for (int i = 0; i < 3; ++i) {
      float invd = 1.f / comp(r.d, i);
      float t0 = (comp(mn, i) - comp(r.o, i)) * invd;
      float t1 = (comp(mx, i) - comp(r.o, i)) * invd;
      bool flip = invd < 0.f;
      if (flip) { float tmp = t0; t0 = t1; t1 = tmp; }
      if (t0 > tmn) { tmn = t0; axis = i; minface = flip ? 0 : 1; }
      tmx = smin(tmx, t1);
      if (tmn > tmx) return false;
    }
    out.t = tmn; out.face = axis | (minface << 2);
    return true;
  } else if (type == 3) {  // disk
    V3 c = v3(p[0], p[1], p[2]), n = v3(p[3], p[4], p[5]);
    float denom = dot(n, r.d);
    if (fabsf(denom) < 1e-7f) return false;
    float t = dot(c - r.o, n) / denom;
    if (t < r.tmin || t >= best) return false;
    V3 pt = r.o + t * r.d;
    V3 op = pt - c;
    if (dot(op, op) > p[6] * p[6]) return false;
    out.t = t; out.face = 0;
    return true;
  } else {  // quad
    V3 o = v3(p[0], p[1], p[2]), uu = v3(p[3], p[4], p[5]), vv = v3(p[6], p[7], p[8]);
    V3 nr = cross(uu, vv);
    float area_sq = dot(nr, nr);
    if (area_sq < 1e-14f) return false;
    float denom = dot(nr, r.d);
    if (fabsf(denom) < 1e-9f) return false;
    float t = dot(nr, o - r.o) / denom;
    if (t < r.tmin || t >= best) return false;
    V3 pt = r.o + t * r.d;
    V3 op = pt - o;
    float s = dot(cross(op, vv), nr) / area_sq;
    float tv = dot(cross(uu, op), nr) / area_sq;
    if (s < 0.f || s > 1.f || tv < 0.f || tv > 1.f) return false;
    out.t = t; out.face = 0;
    return true;
  }
}

// ── BLAS closest hit (blas.cpp:211-265) ──────────────────────────────────────────
template <bool kCount, class Stack>
__device__ __forceinline__ bool blas_closest(const DevScene& sc, int root, const Ray& r,
                                             HitState& h, int inst_idx, const Stack& stack,
                                             TraversalCounters& cnt, bool& overflow) {
  // The reference pushes (far, near) and pops near at once; here the near child continues in
  // a register and only the far one is pushed: the same visit order, half the stack traffic.
  const V3 inv = v3(1.f / r.d.x, 1.f / r.d.y, 1.f / r.d.z);
  int ptr = 0;
  uint32_t cur = blas_root_entry(sc, root);
  bool hit = false;
  for (;;) {
    uint32_t child, count;
    blas_unpack(sc, cur, child, count);
    if (count > 0) {
      for (uint32_t i = 0; i < count; ++i) {
        const float4* tp = sc.tris + 3 * (size_t)(child + i);
        const float4 a = ldg4(tp), b = ldg4(tp + 1), c = ldg4(tp + 2);
        if (kCount) cnt.tris++;
        float t, u, v;
        if (tri_hit(sc, r.o, r.d, inv, r.tmin, ld3(a), ld3(b), ld3(c), h.t, t, u, v)) {
          h.t = t; h.u = u; h.v = v;
          h.prim = (int32_t)(child + i);
          h.inst = inst_idx;
          hit = true;
        }
      }
      if (ptr == 0) break;
      cur = stack.get(--ptr);
      continue;
    }
    if (kCount) cnt.nodes++;
    const float4* pp = sc.blas + 2 * (size_t)child;
    const float4 la = ldg4(pp), lb = ldg4(pp + 1), ra = ldg4(pp + 2), rb = ldg4(pp + 3);
    float tl, tr;
    const bool hl = slab_sse(la, lb, inv, r.o, r.tmin, h.t, tl);
    const bool hr = slab_sse(ra, rb, inv, r.o, r.tmin, h.t, tr);
    const uint32_t el = blas_entry(__float_as_uint(lb.z), __float_as_uint(lb.w), child);
    const uint32_t er = blas_entry(__float_as_uint(rb.z), __float_as_uint(rb.w), child + 1);
    if (hl && hr) {
      if (ptr + 1 > kStackSize) { overflow = true; break; }
      if (tl < tr) { stack.put(ptr++, er); cur = el; }
      else { stack.put(ptr++, el); cur = er; }
    } else if (hl || hr) {
      cur = hl ? el : er;
    } else {
      if (ptr == 0) break;
      cur = stack.get(--ptr);
    }
  }
  return hit;
}

// ── BLAS any hit (blas.cpp:269-307) ──────────────────────────────────────────────
template <bool kCount, class Stack>
__device__ __forceinline__ bool blas_any(const DevScene& sc, int root, const Ray& r,
                                         const Stack& stack, TraversalCounters& cnt, bool& overflow,
                                         bool far_first = false) {
  // Whether some triangle lies in [tmin, tmax] does not depend on the visit order, so the order
  // is a tuning choice: nearest child first, or farthest first (shadow rays start on a surface,
  // where their occluder rarely is).
  const V3 inv = v3(1.f / r.d.x, 1.f / r.d.y, 1.f / r.d.z);
  int ptr = 0;
  uint32_t cur = blas_root_entry(sc, root);
  for (;;) {
    uint32_t child, count;
    blas_unpack(sc, cur, child, count);
    if (count > 0) {
      for (uint32_t i = 0; i < count; ++i) {
        const float4* tp = sc.tris + 3 * (size_t)(child + i);
        const float4 a = ldg4(tp), b = ldg4(tp + 1), c = ldg4(tp + 2);
        if (kCount) cnt.tris++;
        float t, u, v;
        if (tri_hit(sc, r.o, r.d, inv, r.tmin, ld3(a), ld3(b), ld3(c), r.tmax, t, u, v)) return true;
      }
      if (ptr == 0) return false;
      cur = stack.get(--ptr);
      continue;
    }
    if (kCount) cnt.nodes++;
    const float4* pp = sc.blas + 2 * (size_t)child;
    const float4 la = ldg4(pp), lb = ldg4(pp + 1), ra = ldg4(pp + 2), rb = ldg4(pp + 3);
    float tl, tr;
    const bool hl = slab_sse(la, lb, inv, r.o, r.tmin, r.tmax, tl);
    const bool hr = slab_sse(ra, rb, inv, r.o, r.tmin, r.tmax, tr);
    const uint32_t el = blas_entry(__float_as_uint(lb.z), __float_as_uint(lb.w), child);
    const uint32_t er = blas_entry(__float_as_uint(rb.z), __float_as_uint(rb.w), child + 1);
    if (hl && hr) {
      if (ptr + 1 > kStackSize) { overflow = true; return false; }
      if ((tl < tr) != far_first) { stack.put(ptr++, er); cur = el; }
      else { stack.put(ptr++, el); cur = er; }
    } else if (hl || hr) {
      cur = hl ? el : er;
    } else {
      if (ptr == 0) return false;
      cur = stack.get(--ptr);
    }
  }
}

// ── PrimBLAS closest hit (prim_blas.cpp:142-194) ───────────────────────────────
template <class Stack>
__device__ __forceinline__ bool pblas_closest(const DevScene& sc, const Ray& r, HitState& h,
                                              int inst_idx, const Stack& stack, bool& overflow) {
  int ptr = 0;
  stack.put(ptr++, 0);
  bool hit = false;
  while (ptr > 0) {
    const uint32_t idx = stack.get(--ptr);
    const float4 na = ldg4(sc.pnodes + 2 * idx), nb = ldg4(sc.pnodes + 2 * idx + 1);
    float tn;
    if (!aabb_div(na, nb, r, tn) || tn > h.t) continue;
    const uint32_t child = __float_as_uint(nb.z), count = __float_as_uint(nb.w);
    if (count > 0) {
      for (uint32_t i = 0; i < count; ++i) {
        const uint32_t pi = child + i;   // pnode leaves index the reordered prim array
        PrimHit ph;
        if (prim_intersect(sc.prims + 4 * (size_t)pi, r, h.t, ph)) {
          h.t = ph.t; h.u = 0.f; h.v = __int_as_float(ph.face);
          h.prim = (int32_t)pi;
          h.inst = inst_idx;
          hit = true;
        }
      }
      continue;
    }
    const float4 la = ldg4(sc.pnodes + 2 * child), lb = ldg4(sc.pnodes + 2 * child + 1);
    const float4 ra = ldg4(sc.pnodes + 2 * child + 2), rb = ldg4(sc.pnodes + 2 * child + 3);
    float tl, tr;
    const bool hl = aabb_div(la, lb, r, tl) && tl <= h.t;
    const bool hr = aabb_div(ra, rb, r, tr) && tr <= h.t;
    if (ptr + 2 > kStackSize) { overflow = true; break; }
    if (hl && hr) {
      if (tl < tr) { stack.put(ptr++, child + 1); stack.put(ptr++, child); }
      else { stack.put(ptr++, child); stack.put(ptr++, child + 1); }
    } else if (hl) {
      stack.put(ptr++, child);
    } else if (hr) {
      stack.put(ptr++, child + 1);
    }
  }
  return hit;
}

// ── PrimBLAS any hit (prim_blas.cpp:197-229) ───────────────────────────────────
template <class Stack>
__device__ __forceinline__ bool pblas_any(const DevScene& sc, const Ray& r, const Stack& stack,
                                          bool& overflow) {
  int ptr = 0;
  stack.put(ptr++, 0);
  while (ptr > 0) {
    const uint32_t idx = stack.get(--ptr);
    const float4 na = ldg4(sc.pnodes + 2 * idx), nb = ldg4(sc.pnodes + 2 * idx + 1);
    float tn;
    if (!aabb_div(na, nb, r, tn)) continue;
    const uint32_t child = __float_as_uint(nb.z), count = __float_as_uint(nb.w);
    if (count > 0) {
      for (uint32_t i = 0; i < count; ++i) {
        PrimHit ph;
        if (prim_intersect(sc.prims + 4 * (size_t)(child + i), r, r.tmax, ph)) return true;
      }
      continue;
    }
    if (ptr + 2 > kStackSize) { overflow = true; return false; }
    stack.put(ptr++, child);
    stack.put(ptr++, child + 1);
  }
  return false;
}

// ── TLAS closest hit (tlas.cpp:172-245) ──────────────────────────────────────────
template <bool kCount, class Stack>
__device__ __forceinline__ bool scene_closest(const DevScene& sc, const Ray& w, HitState& h,
                                              uint32_t* tstack, const Stack& bstack,
                                              TraversalCounters& cnt, bool& overflow) {
  h.t = kInf; h.u = 0.f; h.v = 0.f; h.prim = -1; h.inst = -1;
  if (sc.num_tlas_nodes == 0) return false;
  const V3 inv = v3(1.f / w.d.x, 1.f / w.d.y, 1.f / w.d.z);
  const int sign[3] = {w.d.x < 0.f, w.d.y < 0.f, w.d.z < 0.f};
  int ptr = 0;
  tstack[ptr++] = 0;
  bool hit = false;
  while (ptr > 0) {
    const uint32_t idx = tstack[--ptr];
    const float4 na = ldg4(sc.tlas + 2 * idx), nb = ldg4(sc.tlas + 2 * idx + 1);
    if (kCount) cnt.tlas++;
    if (!aabb_fast(na, nb, inv, w.o, sign, w.tmin, h.t)) continue;
    const uint32_t child = __float_as_uint(nb.z), count = __float_as_uint(nb.w);
    if (count > 0) {
      for (uint32_t i = 0; i < count; ++i) {
        const int ii = (int)__ldg(sc.tlas_inst + child + i);
        const DevInstance& in = sc.inst[ii];
        if (kCount) cnt.inst++;
        const Ray lr = to_local(in, w);
        bool got;
        if (in.kind == 0) got = blas_closest<kCount>(sc, in.root, lr, h, ii, bstack, cnt, overflow);
        else got = pblas_closest(sc, lr, h, ii, bstack, overflow);
        hit |= got;
      }
      continue;
    }
    // order by the children's centre projections on the parent's widest axis
    const float ex = na.w - na.x, ey = nb.x - na.y, ez = nb.y - na.z;
    const int ax = (ex > ey && ex > ez) ? 0 : (ey > ez ? 1 : 2);
    const float4 la = ldg4(sc.tlas + 2 * child), lb = ldg4(sc.tlas + 2 * child + 1);
    const float4 ra = ldg4(sc.tlas + 2 * child + 2), rb = ldg4(sc.tlas + 2 * child + 3);
    float cl, cr;
    if (ax == 0) { cl = (la.x + la.w) * 0.5f; cr = (ra.x + ra.w) * 0.5f; }
    else if (ax == 1) { cl = (la.y + lb.x) * 0.5f; cr = (ra.y + rb.x) * 0.5f; }
    else { cl = (la.z + lb.y) * 0.5f; cr = (ra.z + rb.y) * 0.5f; }
    const float tl = (cl - comp(w.o, ax)) * comp(inv, ax);
    const float tr = (cr - comp(w.o, ax)) * comp(inv, ax);
    if (ptr + 2 > kStackSize) { overflow = true; break; }
    if (tl < tr) { tstack[ptr++] = child + 1; tstack[ptr++] = child; }
    else { tstack[ptr++] = child; tstack[ptr++] = child + 1; }
  }
  return hit;
}

// ── TLAS any hit (tlas.cpp:248-290) ──────────────────────────────────────────────
template <bool kCount, class Stack>
__device__ __forceinline__ bool scene_any(const DevScene& sc, const Ray& w, uint32_t* tstack,
                                          const Stack& bstack, TraversalCounters& cnt, bool& overflow,
                                          bool far_first = false) {
  if (sc.num_tlas_nodes == 0) return false;
  const V3 inv = v3(1.f / w.d.x, 1.f / w.d.y, 1.f / w.d.z);
  const int sign[3] = {w.d.x < 0.f, w.d.y < 0.f, w.d.z < 0.f};
  int ptr = 0;
  tstack[ptr++] = 0;
  while (ptr > 0) {
    const uint32_t idx = tstack[--ptr];
    const float4 na = ldg4(sc.tlas + 2 * idx), nb = ldg4(sc.tlas + 2 * idx + 1);
    if (kCount) cnt.tlas++;
    if (!aabb_fast(na, nb, inv, w.o, sign, w.tmin, w.tmax)) continue;
    const uint32_t child = __float_as_uint(nb.z), count = __float_as_uint(nb.w);
    if (count > 0) {
      for (uint32_t i = 0; i < count; ++i) {
        const DevInstance& in = sc.inst[__ldg(sc.tlas_inst + child + i)];
        if (kCount) cnt.inst++;
        const Ray lr = to_local(in, w);
        const bool got = (in.kind == 0) ? blas_any<kCount>(sc, in.root, lr, bstack, cnt, overflow, far_first)
                                        : pblas_any(sc, lr, bstack, overflow);
        if (got) return true;
      }
      continue;
    }
    if (ptr + 2 > kStackSize) { overflow = true; return false; }
    tstack[ptr++] = child;
    tstack[ptr++] = child + 1;
  }
  return false;
}

// ── hit completion: the rest of the HitRecord for the final closest hit ─────────
struct FullHit {
  V3 pos, normal, geo_normal;
  int32_t mat_id, prim_id, instance_id;
  float u, v;
  bool front_face;
};

__device__ __forceinline__ void complete_hit(const DevScene& sc, const Ray& w, const HitState& h,
                                             FullHit& f) {
  const DevInstance& in = sc.inst[h.inst];
  const Ray lr = to_local(in, w);
  V3 n, gn;
  if (in.kind == 0) {
    // TriangleMesh::intersect_triangle (mesh.h:104-129)
    const float4* tp = sc.tris + 3 * (size_t)h.prim;
    const float4 a = ldg4(tp), b = ldg4(tp + 1), c = ldg4(tp + 2);
    const int local = __float_as_int(a.w), gtri = __float_as_int(b.w);
    V3 p0 = ld3(a), p1 = ld3(b), p2 = ld3(c);
    gn = normalize(cross(p1 - p0, p2 - p0));
    const DevMesh& m = sc.meshes[in.mesh];
    if (m.has_normals) {
      const int i0 = __ldg(sc.tri_index + 3 * gtri), i1 = __ldg(sc.tri_index + 3 * gtri + 1),
                i2 = __ldg(sc.tri_index + 3 * gtri + 2);
      V3 n0 = v3(__ldg(sc.nx + i0), __ldg(sc.ny + i0), __ldg(sc.nz + i0));
      V3 n1 = v3(__ldg(sc.nx + i1), __ldg(sc.ny + i1), __ldg(sc.nz + i1));
      V3 n2 = v3(__ldg(sc.nx + i2), __ldg(sc.ny + i2), __ldg(sc.nz + i2));
      n = normalize(n0 * (1.f - h.u - h.v) + n1 * h.u + n2 * h.v);
    } else {
      n = gn;
    }
    f.mat_id = __ldg(sc.tri_mat + gtri);
    f.prim_id = local;
    f.u = h.u; f.v = h.v;
  } else {
    // the analytic prim's own normal and UV (primitives.h), on the local ray
    const float4* pr = sc.prims + 4 * (size_t)h.prim;
    const float4 h0 = ldg4(pr), h1 = ldg4(pr + 1), h2 = ldg4(pr + 2), h3 = ldg4(pr + 3);
    const int type = __float_as_int(h0.x);
    const float p[10] = {h1.x, h1.y, h1.z, h1.w, h2.x, h2.y, h2.z, h2.w, h3.x, h3.y};
    const float t = h.t;
    V3 pt = lr.o + t * lr.d;
    float uu = 0.f, vv = 0.f;
    if (type == 0) {
      V3 c = v3(p[0], p[1], p[2]);
      V3 outward = (pt - c) / p[3];
      float phi = atan2f(-outward.z, outward.x) + kPi;
      float theta = acosf(sclamp(-outward.y, -1.f, 1.f));
      bool front = dot(outward, lr.d) < 0.f;
      n = gn = front ? outward : -outward;
      uu = phi * (0.5f * kInvPi);
      vv = theta * kInvPi;
    } else if (type == 1) {
      V3 nn = v3(p[0], p[1], p[2]);
      float denom = dot(nn, lr.d);
      n = gn = (denom < 0.f) ? nn : -nn;
      uu = pt.x - floorf(pt.x);
      vv = pt.z - floorf(pt.z);
    } else if (type == 2) {
      V3 c = v3(p[0], p[1], p[2]), hh = v3(p[3], p[4], p[5]);
      V3 mn = c - hh;
      const int face = __float_as_int(h.v);
      const int axis = face & 3, minface = face >> 2;
      V3 nn = v3s(0.f);
      const float s = minface ? -1.f : 1.f;
      if (axis == 0) nn.x = s; else if (axis == 1) nn.y = s; else nn.z = s;
      if (dot(nn, lr.d) > 0.f) nn = -nn;
      n = gn = nn;
      const int ua = (axis + 1) % 3, va = (axis + 2) % 3;
      uu = (comp(pt, ua) - comp(mn, ua)) / (2.f * comp(hh, ua));
      vv = (comp(pt, va) - comp(mn, va)) / (2.f * comp(hh, va));
    } else if (type == 3) {
      V3 c = v3(p[0], p[1], p[2]), nn = v3(p[3], p[4], p[5]);
      float denom = dot(nn, lr.d);
      V3 op = pt - c;
      n = gn = (denom < 0.f) ? nn : -nn;
      V3 ref = (fabsf(nn.x) < 0.9f) ? v3(1, 0, 0) : v3(0, 1, 0);
      V3 tang = normalize(cross(nn, ref));
      V3 bita = cross(nn, tang);
      float px = dot(op, tang), py = dot(op, bita);
      float phi = atan2f(py, px);
      if (phi < 0.f) phi += 2.f * kPi;
      uu = phi * (0.5f * kInvPi);
      vv = sqrtf(dot(op, op)) / p[6];
    } else {
      V3 o = v3(p[0], p[1], p[2]), ue = v3(p[3], p[4], p[5]), ve = v3(p[6], p[7], p[8]);
      V3 nr = cross(ue, ve);
      float area_sq = dot(nr, nr);
      float denom = dot(nr, lr.d);
      V3 op = pt - o;
      uu = dot(cross(op, ve), nr) / area_sq;
      vv = dot(cross(ue, op), nr) / area_sq;
      V3 nn = normalize(nr);
      if (denom > 0.f) nn = -nn;
      n = gn = nn;
    }
    f.mat_id = __float_as_int(h0.y);
    f.prim_id = __float_as_int(h0.z);   // index in the prim group (prim_blas.h:48-52)
    f.u = uu; f.v = vv;
  }
  // TLAS::fixup_hit (tlas.cpp:156-168)
  f.pos = w.o + h.t * w.d;
  f.normal = normal_to_world(in, n);
  f.geo_normal = normal_to_world(in, gn);
  f.front_face = dot(f.geo_normal, w.d) < 0.f;
  f.instance_id = in.instance_id;
}

}  // namespace xbd
