// oracle.cpp — CPU restatement of the reference wavefront path (the checker; never shipped).
//
// Scalar C++ over the flattened xb_scene_view, compiled without FMA contraction and without
// fast-math, so every float is the one the reference's strict build computes:
//   PCG32 + seeding                  src/camera/sampler.h:13-36
//   Moller-Trumbore                  src/geometry/primitives.h:25-49, mesh.h:104-129
//   analytic prims                   src/geometry/primitives.h:54-318
//   BLAS closest / any               src/geometry/blas.cpp:211-307 (SSE pair test :25-74)
//   PrimBLAS closest / any           src/geometry/prim_blas.cpp:142-229
//   TLAS closest / any + fix-up      src/geometry/tlas.cpp:156-290, transform.h:44-89
//   principled BSDF                  src/material/bsdf.h:31-708, material.h:55-75
//   tiled integrator (one path)      src/render/cpu_tiled.cpp:20-218
// Two rules of the reference that are easy to miss are kept: bsdf.h passes two
// rng.next_float() calls as arguments, which GCC evaluates right to left (the first draw is the
// second parameter); and closest-hit traversal decides equal-t ties by visit order.

#include "oracle.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <limits>
#include <thread>
#include <vector>

namespace {

constexpr float kInf = std::numeric_limits<float>::infinity();
constexpr float kPi = 3.14159265358979323846f;
constexpr float kInvPi = 1.f / kPi;
constexpr float kRayEps = 1e-4f;
constexpr float kShadowEps = 5e-4f;

struct V {
  float x = 0, y = 0, z = 0;
  V() = default;
  V(float a, float b, float c) : x(a), y(b), z(c) {}
  explicit V(float s) : x(s), y(s), z(s) {}
  float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
V operator+(V a, V b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
V operator-(V a, V b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V operator*(V a, V b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
V operator/(V a, V b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
V operator*(V a, float s) { return {a.x * s, a.y * s, a.z * s}; }
V operator*(float s, V a) { return a * s; }
V operator/(V a, float s) { float r = 1.f / s; return {a.x * r, a.y * r, a.z * r}; }
V operator-(V a) { return {-a.x, -a.y, -a.z}; }
float dot(V a, V b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
V cross(V a, V b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
float len2(V a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
V norm(V a) { return a / std::sqrt(len2(a)); }
V reflect(V v, V n) { return v - 2.f * dot(v, n) * n; }
V lerp(V a, V b, float t) { return a + t * (b - a); }
float maxc(V v) { return std::max({v.x, v.y, v.z}); }

struct Pcg {
  uint64_t s;
  uint32_t next() {
    uint64_t o = s;
    s = o * 6364136223846793005ULL + 1ULL;
    uint32_t xs = (uint32_t)(((o >> 18u) ^ o) >> 27u);
    uint32_t rot = (uint32_t)(o >> 59u);
    return (xs >> rot) | (xs << ((~rot + 1u) & 31u));
  }
  float nf() { return (float)(next() >> 8) * (1.f / 16777216.f); }
};
uint64_t seed_state(uint64_t seed) {
  Pcg g{0};
  g.next();
  g.s += seed;
  g.next();
  return g.s;
}

struct Ray { V o, d; float tmin, tmax; };
struct Hit {
  float t = kInf, u = 0, v = 0;
  V pos, n, gn;
  int mat = -1, prim = -1, inst = -1;
  bool front = true;
};

struct Node { V mn, mx; uint32_t child, count; };
struct Mesh {
  std::vector<float> vx, vy, vz, nx, ny, nz;
  std::vector<int32_t> idx, mat;
  std::vector<Node> nodes;
  std::vector<uint32_t> prims;
  V vert(int i) const { return {vx[i], vy[i], vz[i]}; }
  void tri(int t, V& a, V& b, V& c) const { a = vert(idx[3 * t]); b = vert(idx[3 * t + 1]); c = vert(idx[3 * t + 2]); }
};
struct Inst { int geom, id; V l2w[4], w2l[4]; };
struct Mat {
  V base, f0, ssc;
  float metallic, ior, alpha, ax, ay, subsurface;
  bool conductor, transmissive, sss, delta;
};

struct Scene {
  std::vector<Mesh> meshes;
  std::vector<xb_prim> prims;
  std::vector<Node> pnodes;
  std::vector<uint32_t> pidx;
  std::vector<Inst> insts;
  std::vector<Node> tlas;
  std::vector<uint32_t> tinst;
  std::vector<Mat> mats;
  std::vector<xb_light> lights;
  std::vector<xb_sun> suns;
  xb_sky sky;
};

struct Work { int64_t nodes = 0, tris = 0, tlas = 0, inst = 0; };

Node to_node(const xb_bvh_node& n) { return {V(n.mn[0], n.mn[1], n.mn[2]), V(n.mx[0], n.mx[1], n.mx[2]), n.child, n.count}; }

Mat prepare(const xb_material& p) {
  Mat m;
  m.base = V(p.base_color[0], p.base_color[1], p.base_color[2]);
  m.metallic = p.metallic;
  m.ior = p.ior;
  m.subsurface = p.subsurface;
  m.ssc = V(p.subsurface_color[0], p.subsurface_color[1], p.subsurface_color[2]);
  m.alpha = std::max(p.roughness * p.roughness, 1e-6f);
  float aspect = std::sqrt(1.0f - 0.9f * std::abs(p.anisotropy));
  m.ax = std::max(m.alpha / aspect, 1e-6f);
  m.ay = std::max(m.alpha * aspect, 1e-6f);
  float f0d = ((p.ior - 1.0f) * (p.ior - 1.0f)) / ((p.ior + 1.0f) * (p.ior + 1.0f));
  m.f0 = lerp(V(f0d), m.base, p.metallic);
  m.conductor = p.metallic > 0.5f;
  m.transmissive = p.transmission > 0.01f;
  m.sss = p.subsurface > 0.01f;
  m.delta = m.alpha < 0.001f;
  return m;
}

// ── geometry ────────────────────────────────────────────────────────────────────
bool ray_tri(const Ray& r, V v0, V v1, V v2, float tmax, float& t, float& u, float& v) {
  V e1 = v1 - v0, e2 = v2 - v0;
  V h = cross(r.d, e2);
  float a = dot(e1, h);
  if (std::abs(a) < 1e-7f) return false;
  float ia = 1.f / a;
  V s = r.o - v0;
  u = ia * dot(s, h);
  if (u < 0.f || u > 1.f) return false;
  V q = cross(s, e1);
  v = ia * dot(r.d, q);
  if (v < 0.f || u + v > 1.f) return false;
  t = ia * dot(e2, q);
  return t >= r.tmin && t <= tmax;
}

// one child of the SSE pair test: minps/maxps pick the second operand on NaN
float mmin(float a, float b) { return a < b ? a : b; }
float mmax(float a, float b) { return a > b ? a : b; }
bool pair_slab(const Node& c, V inv, V org, float tmin, float tmax, float& tn) {
  float t0x = (c.mn.x - org.x) * inv.x, t1x = (c.mx.x - org.x) * inv.x;
  float t0y = (c.mn.y - org.y) * inv.y, t1y = (c.mx.y - org.y) * inv.y;
  float t0z = (c.mn.z - org.z) * inv.z, t1z = (c.mx.z - org.z) * inv.z;
  float nx = mmax(mmax(mmin(t0x, t1x), mmin(t0y, t1y)), mmin(t0z, t1z));
  float fx = mmin(mmin(mmax(t0x, t1x), mmax(t0y, t1y)), mmax(t0z, t1z));
  float near = mmax(nx, tmin), far = mmin(fx, tmax);
  tn = near;
  return near <= far;
}

bool box_div(const Node& b, const Ray& r, float& tn) {
  float tx0 = (b.mn.x - r.o.x) / r.d.x, tx1 = (b.mx.x - r.o.x) / r.d.x;
  float ty0 = (b.mn.y - r.o.y) / r.d.y, ty1 = (b.mx.y - r.o.y) / r.d.y;
  float tz0 = (b.mn.z - r.o.z) / r.d.z, tz1 = (b.mx.z - r.o.z) / r.d.z;
  float lo = std::max({std::min(tx0, tx1), std::min(ty0, ty1), std::min(tz0, tz1), r.tmin});
  float hi = std::min({std::max(tx0, tx1), std::max(ty0, ty1), std::max(tz0, tz1), r.tmax});
  tn = lo;
  return lo <= hi;
}

bool box_fast(const Node& b, V inv, V org, const int sg[3], float tmin, float tmax) {
  const V* bd[2] = {&b.mn, &b.mx};
  float txmin = ((*bd[sg[0]]).x - org.x) * inv.x, txmax = ((*bd[1 - sg[0]]).x - org.x) * inv.x;
  float tymin = ((*bd[sg[1]]).y - org.y) * inv.y, tymax = ((*bd[1 - sg[1]]).y - org.y) * inv.y;
  float tzmin = ((*bd[sg[2]]).z - org.z) * inv.z, tzmax = ((*bd[1 - sg[2]]).z - org.z) * inv.z;
  tmin = std::max({tmin, txmin, tymin, tzmin});
  tmax = std::min({tmax, txmax, tymax, tzmax});
  return tmin <= tmax;
}

// analytic prim: fills the full record on a hit in [tmin, rec.t)
bool prim_hit(const xb_prim& q, const Ray& r, Hit& rec) {
  const float* p = q.p;
  switch (q.type) {
    case XB_PRIM_SPHERE: {
      V c(p[0], p[1], p[2]);
      V oc = r.o - c;
      float a = dot(r.d, r.d), hb = dot(oc, r.d), cc = dot(oc, oc) - p[3] * p[3];
      float disc = hb * hb - a * cc;
      if (disc < 0.f) return false;
      float sq = std::sqrt(disc);
      float t = (-hb - sq) / a;
      if (t < r.tmin || t >= rec.t) {
        t = (-hb + sq) / a;
        if (t < r.tmin || t >= rec.t) return false;
      }
      V pt = r.o + t * r.d;
      V out = (pt - c) / p[3];
      float phi = std::atan2(-out.z, out.x) + kPi;
      float theta = std::acos(std::clamp(-out.y, -1.f, 1.f));
      rec.t = t; rec.pos = pt;
      rec.front = dot(out, r.d) < 0.f;
      rec.gn = rec.n = rec.front ? out : -out;
      rec.mat = q.mat_id;
      rec.u = phi * (0.5f * kInvPi);
      rec.v = theta * kInvPi;
      return true;
    }
    case XB_PRIM_PLANE: {
      V n(p[0], p[1], p[2]);
      float den = dot(n, r.d);
      if (std::abs(den) < 1e-7f) return false;
      float t = (p[3] - dot(n, r.o)) / den;
      if (t < r.tmin || t >= rec.t) return false;
      V pt = r.o + t * r.d;
      rec.t = t; rec.pos = pt;
      rec.gn = rec.n = den < 0.f ? n : -n;
      rec.front = den < 0.f;
      rec.mat = q.mat_id;
      rec.u = pt.x - std::floor(pt.x);
      rec.v = pt.z - std::floor(pt.z);
      return true;
    }
    case XB_PRIM_BOX: {
      V c(p[0], p[1], p[2]), h(p[3], p[4], p[5]);
      V mn = c - h, mx = c + h;
      float tmn = r.tmin, tmx = rec.t;
      int axis = 0;
      bool minface = false;
      for (int i = 0; i < 3; ++i) {
        float inv = 1.f / r.d[i];
        float t0 = (mn[i] - r.o[i]) * inv, t1 = (mx[i] - r.o[i]) * inv;
        bool flip = inv < 0.f;
        if (flip) std::swap(t0, t1);
        if (t0 > tmn) { tmn = t0; axis = i; minface = !flip; }
        tmx = std::min(tmx, t1);
        if (tmn > tmx) return false;
      }
      rec.t = tmn;
      rec.pos = r.o + tmn * r.d;
      rec.mat = q.mat_id;
      float nn[3] = {0.f, 0.f, 0.f};
      nn[axis] = minface ? -1.f : 1.f;
      V n(nn[0], nn[1], nn[2]);
      if (dot(n, r.d) > 0.f) n = -n;
      rec.gn = rec.n = n;
      rec.front = dot(n, r.d) < 0.f;
      int ua = (axis + 1) % 3, va = (axis + 2) % 3;
      rec.u = (rec.pos[ua] - mn[ua]) / (2.f * h[ua]);
      rec.v = (rec.pos[va] - mn[va]) / (2.f * h[va]);
      return true;
    }
    case XB_PRIM_DISK: {
      V c(p[0], p[1], p[2]), n(p[3], p[4], p[5]);
      float den = dot(n, r.d);
      if (std::abs(den) < 1e-7f) return false;
      float t = dot(c - r.o, n) / den;
      if (t < r.tmin || t >= rec.t) return false;
      V pt = r.o + t * r.d;
      V op = pt - c;
      if (dot(op, op) > p[6] * p[6]) return false;
      rec.t = t; rec.pos = pt;
      rec.gn = rec.n = den < 0.f ? n : -n;
      rec.front = den < 0.f;
      rec.mat = q.mat_id;
      V ref = (std::abs(n.x) < 0.9f) ? V(1, 0, 0) : V(0, 1, 0);
      V tg = norm(cross(n, ref));
      V bt = cross(n, tg);
      float phi = std::atan2(dot(op, bt), dot(op, tg));
      if (phi < 0.f) phi += 2.f * kPi;
      rec.u = phi * (0.5f * kInvPi);
      rec.v = std::sqrt(dot(op, op)) / p[6];
      return true;
    }
    default: {
      V o(p[0], p[1], p[2]), ue(p[3], p[4], p[5]), ve(p[6], p[7], p[8]);
      V nr = cross(ue, ve);
      float a2 = dot(nr, nr);
      if (a2 < 1e-14f) return false;
      float den = dot(nr, r.d);
      if (std::abs(den) < 1e-9f) return false;
      float t = dot(nr, o - r.o) / den;
      if (t < r.tmin || t >= rec.t) return false;
      V pt = r.o + t * r.d;
      V op = pt - o;
      float s = dot(cross(op, ve), nr) / a2;
      float tv = dot(cross(ue, op), nr) / a2;
      if (s < 0.f || s > 1.f || tv < 0.f || tv > 1.f) return false;
      V n = norm(nr);
      if (den > 0.f) n = -n;
      rec.t = t; rec.pos = pt; rec.gn = rec.n = n;
      rec.front = den < 0.f;
      rec.mat = q.mat_id;
      rec.u = s; rec.v = tv;
      return true;
    }
  }
}

bool mesh_tri_hit(const Mesh& m, const Ray& r, int t_idx, Hit& rec) {
  V a, b, c;
  m.tri(t_idx, a, b, c);
  float t, u, v;
  if (!ray_tri(r, a, b, c, rec.t, t, u, v)) return false;
  rec.t = t; rec.pos = r.o + t * r.d; rec.u = u; rec.v = v;
  rec.mat = m.mat[t_idx];
  rec.prim = t_idx;
  V gn = norm(cross(b - a, c - a));
  rec.gn = gn;
  rec.front = dot(gn, r.d) < 0.f;
  if (!m.nx.empty()) {
    int i0 = m.idx[3 * t_idx], i1 = m.idx[3 * t_idx + 1], i2 = m.idx[3 * t_idx + 2];
    V n0(m.nx[i0], m.ny[i0], m.nz[i0]), n1(m.nx[i1], m.ny[i1], m.nz[i1]), n2(m.nx[i2], m.ny[i2], m.nz[i2]);
    rec.n = norm(n0 * (1.f - u - v) + n1 * u + n2 * v);
  } else {
    rec.n = gn;
  }
  return true;
}

bool blas_closest(const Mesh& m, const Ray& r, Hit& rec, Work& w) {
  if (m.nodes.empty()) return false;
  V inv(1.f / r.d.x, 1.f / r.d.y, 1.f / r.d.z);
  uint32_t st[64];
  int sp = 0;
  st[sp++] = 0;
  bool hit = false;
  while (sp > 0) {
    const Node& nd = m.nodes[st[--sp]];
    if (nd.count > 0) {
      for (uint32_t i = 0; i < nd.count; ++i) {
        w.tris++;
        if (mesh_tri_hit(m, r, (int)m.prims[nd.child + i], rec)) hit = true;
      }
      continue;
    }
    w.nodes++;
    const uint32_t l = nd.child, rr = l + 1;
    float tl, tr;
    bool hl = pair_slab(m.nodes[l], inv, r.o, r.tmin, rec.t, tl);
    bool hr = pair_slab(m.nodes[rr], inv, r.o, r.tmin, rec.t, tr);
    if (!hl && !hr) continue;
    if (hl && hr) {
      if (tl < tr) { st[sp++] = rr; st[sp++] = l; }
      else { st[sp++] = l; st[sp++] = rr; }
    } else {
      st[sp++] = hl ? l : rr;
    }
  }
  return hit;
}

bool blas_any(const Mesh& m, const Ray& r, Work& w) {
  if (m.nodes.empty()) return false;
  V inv(1.f / r.d.x, 1.f / r.d.y, 1.f / r.d.z);
  uint32_t st[64];
  int sp = 0;
  st[sp++] = 0;
  while (sp > 0) {
    const Node& nd = m.nodes[st[--sp]];
    if (nd.count > 0) {
      Hit tmp;
      tmp.t = r.tmax;
      for (uint32_t i = 0; i < nd.count; ++i) {
        w.tris++;
        if (mesh_tri_hit(m, r, (int)m.prims[nd.child + i], tmp)) return true;
      }
      continue;
    }
    w.nodes++;
    float tl, tr;
    bool hl = pair_slab(m.nodes[nd.child], inv, r.o, r.tmin, r.tmax, tl);
    bool hr = pair_slab(m.nodes[nd.child + 1], inv, r.o, r.tmin, r.tmax, tr);
    if (hr) st[sp++] = nd.child + 1;
    if (hl) st[sp++] = nd.child;
  }
  return false;
}

bool pblas_closest(const Scene& sc, const Ray& r, Hit& rec) {
  if (sc.pnodes.empty()) return false;
  uint32_t st[64];
  int sp = 0;
  st[sp++] = 0;
  bool hit = false;
  while (sp > 0) {
    const Node& nd = sc.pnodes[st[--sp]];
    float tn;
    if (!box_div(nd, r, tn) || tn > rec.t) continue;
    if (nd.count > 0) {
      for (uint32_t i = 0; i < nd.count; ++i) {
        const uint32_t pi = sc.pidx[nd.child + i];
        if (prim_hit(sc.prims[pi], r, rec)) { rec.prim = (int)pi; hit = true; }
      }
      continue;
    }
    float tl, tr;
    bool hl = box_div(sc.pnodes[nd.child], r, tl) && tl <= rec.t;
    bool hr = box_div(sc.pnodes[nd.child + 1], r, tr) && tr <= rec.t;
    if (hl && hr) {
      if (tl < tr) { st[sp++] = nd.child + 1; st[sp++] = nd.child; }
      else { st[sp++] = nd.child; st[sp++] = nd.child + 1; }
    } else if (hl) {
      st[sp++] = nd.child;
    } else if (hr) {
      st[sp++] = nd.child + 1;
    }
  }
  return hit;
}

bool pblas_any(const Scene& sc, const Ray& r) {
  if (sc.pnodes.empty()) return false;
  uint32_t st[64];
  int sp = 0;
  st[sp++] = 0;
  while (sp > 0) {
    const Node& nd = sc.pnodes[st[--sp]];
    float tn;
    if (!box_div(nd, r, tn)) continue;
    if (nd.count > 0) {
      for (uint32_t i = 0; i < nd.count; ++i) {
        Hit tmp;
        tmp.t = r.tmax;
        if (prim_hit(sc.prims[sc.pidx[nd.child + i]], r, tmp)) return true;
      }
      continue;
    }
    st[sp++] = nd.child;
    st[sp++] = nd.child + 1;
  }
  return false;
}

V xf_point(const V c[4], V p) { return c[0] * p.x + c[1] * p.y + c[2] * p.z + c[3]; }
V xf_dir(const V c[4], V d) { return c[0] * d.x + c[1] * d.y + c[2] * d.z; }
V xf_normal(const V c[4], V n) { return norm(V(dot(c[0], n), dot(c[1], n), dot(c[2], n))); }

bool scene_closest(const Scene& sc, const Ray& w, Hit& rec, Work& wk) {
  if (sc.tlas.empty()) return false;
  V inv(1.f / w.d.x, 1.f / w.d.y, 1.f / w.d.z);
  int sg[3] = {w.d.x < 0, w.d.y < 0, w.d.z < 0};
  uint32_t st[64];
  int sp = 0;
  st[sp++] = 0;
  bool hit = false;
  while (sp > 0) {
    const Node& nd = sc.tlas[st[--sp]];
    wk.tlas++;
    if (!box_fast(nd, inv, w.o, sg, w.tmin, rec.t)) continue;
    if (nd.count > 0) {
      for (uint32_t i = 0; i < nd.count; ++i) {
        const Inst& in = sc.insts[sc.tinst[nd.child + i]];
        wk.inst++;
        Ray lr{xf_point(in.w2l, w.o), xf_dir(in.w2l, w.d), w.tmin, w.tmax};
        Hit lrec = rec;
        bool got = in.geom >= 0 ? blas_closest(sc.meshes[in.geom], lr, lrec, wk) : pblas_closest(sc, lr, lrec);
        if (got) {
          lrec.pos = w.o + lrec.t * w.d;
          lrec.n = xf_normal(in.w2l, lrec.n);
          lrec.gn = xf_normal(in.w2l, lrec.gn);
          lrec.front = dot(lrec.gn, w.d) < 0.f;
          lrec.inst = in.id;
          rec = lrec;
          hit = true;
        }
      }
      continue;
    }
    const Node& L = sc.tlas[nd.child];
    const Node& R = sc.tlas[nd.child + 1];
    V ext = nd.mx - nd.mn;
    int ax = (ext.x > ext.y && ext.x > ext.z) ? 0 : (ext.y > ext.z ? 1 : 2);
    float tl = (((L.mn + L.mx) * 0.5f)[ax] - w.o[ax]) * inv[ax];
    float tr = (((R.mn + R.mx) * 0.5f)[ax] - w.o[ax]) * inv[ax];
    if (tl < tr) { st[sp++] = nd.child + 1; st[sp++] = nd.child; }
    else { st[sp++] = nd.child; st[sp++] = nd.child + 1; }
  }
  return hit;
}

bool scene_any(const Scene& sc, const Ray& w, Work& wk) {
  if (sc.tlas.empty()) return false;
  V inv(1.f / w.d.x, 1.f / w.d.y, 1.f / w.d.z);
  int sg[3] = {w.d.x < 0, w.d.y < 0, w.d.z < 0};
  uint32_t st[64];
  int sp = 0;
  st[sp++] = 0;
  while (sp > 0) {
    const Node& nd = sc.tlas[st[--sp]];
    wk.tlas++;
    if (!box_fast(nd, inv, w.o, sg, w.tmin, w.tmax)) continue;
    if (nd.count > 0) {
      for (uint32_t i = 0; i < nd.count; ++i) {
        const Inst& in = sc.insts[sc.tinst[nd.child + i]];
        wk.inst++;
        Ray lr{xf_point(in.w2l, w.o), xf_dir(in.w2l, w.d), w.tmin, w.tmax};
        if (in.geom >= 0 ? blas_any(sc.meshes[in.geom], lr, wk) : pblas_any(sc, lr)) return true;
      }
      continue;
    }
    st[sp++] = nd.child;
    st[sp++] = nd.child + 1;
  }
  return false;
}

// ── BSDF (bsdf.h) ─────────────────────────────────────────────────────────────
struct Smp { V wi, f; float pdf = 0.f; bool delta = false; };

float c2(V w) { return w.z * w.z; }
float s2(V w) { return std::max(0.f, 1.f - c2(w)); }
float st_(V w) { return std::sqrt(s2(w)); }
float t2(V w) { float c = c2(w); return (c < 1e-8f) ? 0.f : s2(w) / c; }
float cphi(V w) { float s = st_(w); return (s == 0.f) ? 1.f : std::clamp(w.x / s, -1.f, 1.f); }
float sphi(V w) { float s = st_(w); return (s == 0.f) ? 0.f : std::clamp(w.y / s, -1.f, 1.f); }
bool same_hemi(V a, V b) { return a.z * b.z > 0.f; }
float mis2(float a, float b) { float a2 = a * a, b2 = b * b, s = a2 + b2; return (s > 0.f) ? a2 / s : 0.f; }

float D(V wh, float ax, float ay) {
  float c = c2(wh);
  if (c <= 0.f) return 0.f;
  float ex = cphi(wh) / ax, ey = sphi(wh) / ay;
  float tn = (ex * ex + ey * ey) * t2(wh);
  float d = c * c * (1.f + tn);
  return 1.f / (kPi * ax * ay * d * d);
}
float lam(V w, float ax, float ay) {
  float t = t2(w);
  if (t == 0.f) return 0.f;
  float cp = cphi(w), sp = sphi(w);
  float a2 = (cp * ax) * (cp * ax) + (sp * ay) * (sp * ay);
  return (-1.f + std::sqrt(1.f + a2 * t)) * 0.5f;
}
float G1(V w, float ax, float ay) { return 1.f / (1.f + lam(w, ax, ay)); }
float G2(V o, V i, float ax, float ay) { return 1.f / (1.f + lam(o, ax, ay) + lam(i, ax, ay)); }
float fres(float ci, float ior) {
  ci = std::clamp(ci, -1.f, 1.f);
  float ei = 1.f, et = ior;
  if (ci < 0.f) { std::swap(ei, et); ci = -ci; }
  float s2i = 1.f - ci * ci;
  float s2t = (ei / et) * (ei / et) * s2i;
  if (s2t >= 1.f) return 1.f;
  float ct = std::sqrt(std::max(0.f, 1.f - s2t));
  float rp = ((et * ci) - (ei * ct)) / ((et * ci) + (ei * ct));
  float rs = ((ei * ci) - (et * ct)) / ((ei * ci) + (et * ct));
  return (rp * rp + rs * rs) * 0.5f;
}
V schlick(float c, V f0) {
  float m = std::clamp(1.f - c, 0.f, 1.f);
  float m2 = m * m;
  return f0 + (V(1.f) - f0) * (m2 * m2 * m);
}
V cos_hemi(float u1, float u2) {
  float r = std::sqrt(u1), phi = 2.0f * kPi * u2;
  return {r * std::cos(phi), r * std::sin(phi), std::sqrt(std::max(0.0f, 1.0f - u1))};
}
V vndf(V wo, float ax, float ay, float u1, float u2) {
  V vh = norm(V(ax * wo.x, ay * wo.y, wo.z));
  float l2 = vh.x * vh.x + vh.y * vh.y;
  V T1 = (l2 > 1e-7f) ? V(-vh.y, vh.x, 0.f) * (1.f / std::sqrt(l2)) : V(1.f, 0.f, 0.f);
  V T2 = cross(vh, T1);
  float r = std::sqrt(u1), phi = 2.0f * kPi * u2;
  float a = r * std::cos(phi), b = r * std::sin(phi);
  float s = 0.5f * (1.0f + vh.z);
  b = (1.0f - s) * std::sqrt(std::max(0.f, 1.0f - a * a)) + s * b;
  V nh = a * T1 + b * T2 + std::sqrt(std::max(0.f, 1.0f - a * a - b * b)) * vh;
  return norm(V(ax * nh.x, ay * nh.y, std::max(0.f, nh.z)));
}
float vpdf(V wo, V wh, float ax, float ay) {
  float d = D(wh, ax, ay), g = G1(wo, ax, ay), co = std::abs(wo.z);
  if (co < 1e-8f) return 0.f;
  return d * g * std::max(0.f, dot(wo, wh)) / co;
}
float Edir(float c, float a) {
  float e = 1.0f - std::pow(1.0f - c, 5.0f * std::exp(-2.69f * a)) / (1.0f + 22.7f * std::pow(a, 1.5f));
  return std::clamp(e, 0.f, 1.f);
}
V ms(V f0, float co, float ci, float a) {
  float eo = Edir(std::abs(co), a), ei = Edir(std::abs(ci), a);
  float eavg = 1.0f / (1.0f + 0.3037f * a + 0.1218f * a * a);
  V favg = (V(1.f) + f0 * 20.f) * (1.f / 21.f);
  float den = std::max(1.f - favg.x * (1.f - eavg), 1e-4f);
  V fms = favg * favg * eavg / V(den);
  float cm = (1.f - eo) * (1.f - ei);
  return V(1.f) + fms * cm / V(std::max(eo * ei, 1e-4f));
}
V mfr_eval(V wo, V wi, const Mat& m) {
  if (wo.z <= 0.f || wi.z <= 0.f) return V(0.f);
  V wh = norm(wo + wi);
  if (wh.z <= 0.f) return V(0.f);
  float d = D(wh, m.ax, m.ay), g = G2(wo, wi, m.ax, m.ay);
  V F = m.conductor ? schlick(std::abs(dot(wo, wh)), m.f0) : V(fres(dot(wo, wh), m.ior));
  float den = 4.f * wo.z * wi.z;
  if (den < 1e-8f) return V(0.f);
  V res = F * d * g / den;
  if (!m.transmissive) res = res * ms(m.f0, wo.z, wi.z, m.alpha);
  return res;
}
float mfr_pdf(V wo, V wi, const Mat& m) {
  if (wo.z <= 0.f || wi.z <= 0.f) return 0.f;
  V wh = norm(wo + wi);
  if (wh.z <= 0.f) return 0.f;
  return vpdf(wo, wh, m.ax, m.ay) * (1.f / (4.f * std::abs(dot(wo, wh))));
}
bool mfr_sample(V wo, const Mat& m, Pcg& g, Smp& s) {
  if (wo.z <= 0.f) return false;
  float u2 = g.nf(), u1 = g.nf();   // GCC evaluates the two argument draws right to left
  V wh = vndf(wo, m.ax, m.ay, u1, u2);
  if (wh.z <= 0.f) return false;
  s.wi = reflect(-wo, wh);
  if (s.wi.z <= 0.f) return false;
  s.pdf = mfr_pdf(wo, s.wi, m);
  if (s.pdf < 1e-8f) return false;
  s.f = mfr_eval(wo, s.wi, m);
  s.delta = false;
  return true;
}
V mft_eval(V wo, V wi, const Mat& m) {
  if (wo.z == 0.f || wi.z == 0.f || same_hemi(wo, wi)) return V(0.f);
  float eta = wo.z > 0.f ? 1.f / m.ior : m.ior;
  V wh = norm(wo + eta * wi);
  if (wh.z < 0.f) wh = -wh;
  float dwo = dot(wo, wh), dwi = dot(wi, wh);
  if (dwo * dwi >= 0.f) return V(0.f);
  float d = D(wh, m.ax, m.ay), g = G2(wo, wi, m.ax, m.ay), F = fres(dwo, m.ior);
  float co = std::abs(wo.z), ci = std::abs(wi.z);
  if (co < 1e-8f || ci < 1e-8f) return V(0.f);
  float den = dwo + eta * dwi, den2 = den * den;
  if (std::abs(den) < 1e-8f) return V(0.f);
  float fac = std::abs(dwo * dwi) * (eta * eta) / (co * ci * den2);
  return m.base * ((1.f - F) * d * g * fac);
}
float mft_pdf(V wo, V wi, const Mat& m) {
  if (wo.z == 0.f || wi.z == 0.f || same_hemi(wo, wi)) return 0.f;
  float eta = wo.z > 0.f ? 1.f / m.ior : m.ior;
  V wh = norm(wo + eta * wi);
  if (wh.z < 0.f) wh = -wh;
  float dwo = dot(wo, wh), dwi = dot(wi, wh);
  if (dwo * dwi >= 0.f) return 0.f;
  float pwh = vpdf(wo, wh, m.ax, m.ay);
  float den = dwo + eta * dwi;
  if (std::abs(den) < 1e-8f) return 0.f;
  return pwh * std::abs((eta * eta * dwi) / (den * den));
}
bool mft_sample(V wo, const Mat& m, Pcg& g, Smp& s) {
  if (std::abs(wo.z) < 1e-8f) return false;
  float u2 = g.nf(), u1 = g.nf();
  V wh = vndf(wo, m.ax, m.ay, u1, u2);
  if (wh.z < 0.f) wh = -wh;
  float eta = wo.z > 0.f ? 1.f / m.ior : m.ior;
  float dwo = dot(wo, wh);
  float s2o = std::max(0.f, 1.f - dwo * dwo), s2i = eta * eta * s2o;
  if (s2i >= 1.f) return false;
  float cti = std::sqrt(std::max(0.f, 1.f - s2i));
  float sg = dwo > 0.f ? 1.f : -1.f;
  s.wi = norm((-eta * wo) + (eta * dwo - sg * cti) * wh);
  if (same_hemi(wo, s.wi)) return false;
  s.pdf = mft_pdf(wo, s.wi, m);
  if (s.pdf < 1e-8f) return false;
  s.f = mft_eval(wo, s.wi, m);
  s.delta = false;
  return true;
}
bool drefl(V wo, const Mat& m, Smp& s) {
  if (std::abs(wo.z) < 1e-8f) return false;
  V n(0.f, 0.f, wo.z > 0.f ? 1.f : -1.f);
  s.wi = reflect(-wo, n);
  V F = m.conductor ? schlick(std::abs(wo.z), m.f0) : V(fres(std::abs(wo.z), m.ior));
  float ci = std::abs(s.wi.z);
  if (ci < 1e-8f) return false;
  s.f = F / ci; s.pdf = 1.f; s.delta = true;
  return true;
}
bool dtrans(V wo, const Mat& m, Smp& s) {
  if (std::abs(wo.z) < 1e-8f) return false;
  float eta = wo.z > 0.f ? 1.f / m.ior : m.ior;
  V n(0.f, 0.f, wo.z > 0.f ? 1.f : -1.f);
  V v = -wo;
  float ci = -dot(norm(v), n);
  float s2t = eta * eta * (1.f - ci * ci);
  if (s2t >= 1.f) return false;
  s.wi = norm(eta * v + (eta * ci - std::sqrt(1.f - s2t)) * n);
  float F = fres(std::abs(wo.z), m.ior);
  float c = std::abs(s.wi.z);
  if (c < 1e-8f) return false;
  s.f = m.base * ((1.f - F) * eta * eta / c); s.pdf = 1.f; s.delta = true;
  return true;
}
bool cosine(V wo, V color, const Mat& m, Pcg& g, Smp& s) {
  float u2 = g.nf(), u1 = g.nf();
  s.wi = cos_hemi(u1, u2);
  if (wo.z < 0.f) s.wi.z = -s.wi.z;
  s.pdf = std::abs(s.wi.z) * kInvPi;
  if (s.pdf < 1e-8f) return false;
  s.f = color * (1.f - m.metallic) * kInvPi;
  s.delta = false;
  return true;
}
V ss_col(const Mat& m) { return lerp(m.base, m.ssc, m.subsurface); }
V eval(V wo, V wi, const Mat& m) {
  if (m.delta) return V(0.f);
  if (m.conductor) return mfr_eval(wo, wi, m);
  if (m.transmissive) return wi.z > 0.f ? mfr_eval(wo, wi, m) : mft_eval(wo, wi, m);
  if (m.sss) return wi.z <= 0.f ? V(0.f) : ss_col(m) * (1.f - m.metallic) * kInvPi;
  float sw = m.f0.x, dw = 1.f - sw;
  if (wi.z > 0.f) return (wi.z <= 0.f ? V(0.f) : m.base * (1.f - m.metallic) * kInvPi) * dw + mfr_eval(wo, wi, m) * sw;
  return V(0.f);
}
float pdf(V wo, V wi, const Mat& m) {
  if (m.delta) return 0.f;
  if (m.conductor) return mfr_pdf(wo, wi, m);
  if (m.transmissive) {
    float F = fres(std::abs(wo.z), m.ior);
    return wi.z > 0.f ? F * mfr_pdf(wo, wi, m) : (1.f - F) * mft_pdf(wo, wi, m);
  }
  if (m.sss) return wi.z <= 0.f ? 0.f : wi.z * kInvPi;
  float sw = m.f0.x, dw = 1.f - sw;
  if (wi.z > 0.f) return (wi.z * kInvPi) * dw + mfr_pdf(wo, wi, m) * sw;
  return 0.f;
}
bool sample(V wo, const Mat& m, Pcg& g, Smp& s) {
  if (m.delta) {
    if (m.transmissive) return g.nf() < fres(wo.z, m.ior) ? drefl(wo, m, s) : dtrans(wo, m, s);
    return drefl(wo, m, s);
  }
  if (m.conductor) return mfr_sample(wo, m, g, s);
  if (m.sss) return cosine(wo, ss_col(m), m, g, s);
  if (m.transmissive) {
    float F = fres(std::abs(wo.z), m.ior);
    if (g.nf() < F) {
      if (!mfr_sample(wo, m, g, s)) return false;
      s.pdf *= F;
      return true;
    }
    if (!mft_sample(wo, m, g, s)) return false;
    s.pdf *= (1.f - F);
    return true;
  }
  float sw = std::clamp(m.f0.x, 0.f, 1.f), dw = 1.f - sw;
  if (g.nf() < sw) {
    if (!mfr_sample(wo, m, g, s)) return false;
    s.pdf *= sw;
    return true;
  }
  if (!cosine(wo, m.base, m, g, s)) return false;
  s.pdf *= dw;
  return true;
}

struct Onb {
  V u, v, n;
  explicit Onb(V nn) : n(nn) {
    float s = (n.z >= 0.f) ? 1.f : -1.f;
    float a = -1.f / (s + n.z);
    float b = n.x * n.y * a;
    u = V(1.f + s * n.x * n.x * a, s * b, -s * n.x);
    v = V(b, s + n.y * n.y * a, -n.y);
  }
  V world(V l) const { return l.x * u + l.y * v + l.z * n; }
  V local(V w) const { return {dot(w, u), dot(w, v), dot(w, n)}; }
};
V offset(V p, V ng, V dir, float eps) {
  V n = ng;
  if (dot(n, dir) < 0.f) n = -n;
  return p + n * eps;
}

V sky_eval(const xb_sky& k, V d) {
  V hz(k.horizon[0], k.horizon[1], k.horizon[2]);
  if (d.y < 0.f) return k.intensity * lerp(hz, V(k.ground[0], k.ground[1], k.ground[2]), std::min(-d.y, 1.f));
  return k.intensity * lerp(hz, V(k.zenith[0], k.zenith[1], k.zenith[2]), std::pow(d.y, 1.0f / k.sharpness));
}

// One path of render_frame_tiled (cpu_tiled.cpp:20-217).
V trace_path(const Scene& sc, const xb_camera& cam, int W, int H, int x, int y, int spp, int min_b, int max_b,
             int64_t& n_closest, int64_t& n_shadow) {
  Work wk;
  const uint64_t seed = (uint64_t)(y * W + x) + (uint64_t)spp * 0xdeadbeefULL;
  Pcg g{seed_state(seed)};
  float u = (float)x + g.nf();
  float v = (float)y + g.nf();
  V eye(cam.eye[0], cam.eye[1], cam.eye[2]), ll(cam.lower_left[0], cam.lower_left[1], cam.lower_left[2]);
  V hz(cam.horizontal[0], cam.horizontal[1], cam.horizontal[2]), vt(cam.vertical[0], cam.vertical[1], cam.vertical[2]);
  Ray ray{eye, norm(ll + (u / (float)W) * hz + (v / (float)H) * vt - eye), kRayEps, kInf};
  V tp(1.f), acc(0.f);
  float prev_pdf = 0.f;
  bool prev_delta = true;
  const int nl = (int)sc.lights.size(), ns = (int)sc.suns.size();
  for (int depth = 0; depth < max_b; ++depth) {
    Hit rec;
    n_closest++;
    if (!scene_closest(sc, ray, rec, wk)) {
      if (sc.sky.intensity > 0.f) acc = acc + tp * sky_eval(sc.sky, ray.d);
      break;
    }
    const Mat& m = sc.mats[rec.mat];
    bool hit_light = false;
    for (const xb_light& l : sc.lights) {
      if (l.tri_idx == (uint32_t)rec.prim && l.mesh_id == (uint32_t)rec.inst) {
        float w = 1.0f;
        float cl = std::max(0.0f, dot(rec.gn, -ray.d));
        if (cl > 1e-6f) {
          if (depth > 0 && !prev_delta) {
            float pa = (1.0f / l.area) * (1.0f / (float)nl);
            float lpdf = (pa * (rec.t * rec.t)) / cl;
            w = mis2(prev_pdf, lpdf);
          }
          acc = acc + tp * V(l.emission[0], l.emission[1], l.emission[2]) * w;
        }
        hit_light = true;
        break;
      }
    }
    if (hit_light) break;
    if (nl > 0 && !m.delta) {
      int li = std::clamp((int)(g.nf() * (float)nl), 0, nl - 1);
      float pick = 1.f / (float)nl;
      const xb_light& l = sc.lights[li];
      V p0, p1, p2;
      sc.meshes[l.mesh_id].tri((int)l.tri_idx, p0, p1, p2);
      float u1 = g.nf(), u2 = g.nf();
      float su1 = std::sqrt(u1);
      float b0 = 1.0f - su1, b1 = u2 * su1, b2 = 1.0f - b0 - b1;
      V lp = p0 * b0 + p1 * b1 + p2 * b2;
      V ln = norm(cross(p1 - p0, p2 - p0));
      V sd = lp - rec.pos;
      float dsq = len2(sd), dist = std::sqrt(dsq);
      if (dist > 1e-6f) {
        V wi = sd / dist;
        float cl = std::max(0.0f, dot(ln, -wi));
        Onb on(rec.gn);
        V wol = on.local(-ray.d), wil = on.local(wi);
        if (cl > 1e-6f && wil.z > 1e-6f) {
          V f = eval(wol, wil, m);
          float bp = pdf(wol, wil, m);
          float lpdf = ((1.0f / l.area) * pick) * (dsq / cl);
          float w = mis2(lpdf, bp);
          if (w > 0.0f && lpdf > 1e-12f) {
            Ray sr{offset(rec.pos, rec.gn, wi, kShadowEps), wi, kShadowEps, dist - kShadowEps};
            n_shadow++;
            if (!scene_any(sc, sr, wk))
              acc = acc + tp * f * wil.z * (V(l.emission[0], l.emission[1], l.emission[2]) / lpdf) * w;
          }
        }
      }
    }
    if (ns > 0 && !m.delta) {
      float dpick = 0.f;
      int di = std::clamp((int)(g.nf() * (float)ns), 0, ns - 1);
      dpick = 1.f / (float)ns;
      if (di >= 0 && dpick > 0.f) {
        const xb_sun& s = sc.suns[di];
        V sdir(s.direction[0], s.direction[1], s.direction[2]);
        Onb on(rec.gn);
        V wol = on.local(-ray.d), wil = on.local(sdir);
        if (wil.z > 1e-6f) {
          V f = eval(wol, wil, m);
          float bp = pdf(wol, wil, m);
          float lpdf = 1e8f * dpick;
          float w = mis2(lpdf, bp);
          Ray sr{offset(rec.pos, rec.gn, sdir, kShadowEps), sdir, kShadowEps, kInf};
          n_shadow++;
          if (!scene_any(sc, sr, wk)) {
            V em = V(s.color[0], s.color[1], s.color[2]) * s.intensity;
            acc = acc + tp * f * wil.z * (em / lpdf) * w;
          }
        }
      }
    }
    if (depth >= min_b) {
      float p = std::max(0.05f, maxc(tp));
      if (g.nf() > p) break;
      tp = tp * (1.f / p);
    }
    Onb on(rec.n);
    V wol = on.local(-ray.d);
    Smp s;
    if (!sample(wol, m, g, s)) break;
    if (s.delta) {
      tp = tp * s.f;
    } else {
      float ci = std::abs(s.wi.z);
      if (s.pdf < 1e-8f || ci < 1e-8f) break;
      tp = tp * (s.f * ci / s.pdf);
    }
    V ww = on.world(s.wi);
    ray = Ray{offset(rec.pos, rec.gn, ww, kRayEps), ww, kRayEps, kInf};
    prev_pdf = s.pdf;
    prev_delta = s.delta;
  }
  return acc;
}

void fill_hit(const Hit& h, bool hit, xb_hit* o) {
  std::memset(o, 0, sizeof(*o));
  if (!hit) { o->t = kInf; o->prim_id = o->instance_id = o->mat_id = -1; return; }
  o->t = h.t; o->u = h.u; o->v = h.v;
  o->prim_id = h.prim; o->instance_id = h.inst; o->mat_id = h.mat; o->front_face = h.front;
  const V* src[3] = {&h.pos, &h.n, &h.gn};
  float* dst[3] = {o->pos, o->normal, o->geo_normal};
  for (int k = 0; k < 3; ++k) { dst[k][0] = src[k]->x; dst[k][1] = src[k]->y; dst[k][2] = src[k]->z; }
}

}  // namespace

extern "C" {

void* xo_scene_new(const xb_scene_view* v) {
  auto* s = new Scene();
  for (int i = 0; i < v->num_meshes; ++i) {
    const xb_mesh_view& mv = v->meshes[i];
    Mesh m;
    const int nv = mv.num_vertices, nt = mv.num_triangles;
    m.vx.assign(mv.vx, mv.vx + nv); m.vy.assign(mv.vy, mv.vy + nv); m.vz.assign(mv.vz, mv.vz + nv);
    if (mv.nx) { m.nx.assign(mv.nx, mv.nx + nv); m.ny.assign(mv.ny, mv.ny + nv); m.nz.assign(mv.nz, mv.nz + nv); }
    m.idx.assign(mv.indices, mv.indices + 3 * nt);
    m.mat.resize(nt);
    for (int t = 0; t < nt; ++t) m.mat[t] = mv.mat_ids ? mv.mat_ids[t] : 0;
    for (int k = 0; k < mv.num_blas_nodes; ++k) m.nodes.push_back(to_node(mv.blas_nodes[k]));
    m.prims.assign(mv.blas_prims, mv.blas_prims + nt);
    s->meshes.push_back(std::move(m));
  }
  s->prims.assign(v->prims, v->prims + v->num_prims);
  for (int k = 0; k < v->num_prim_nodes; ++k) s->pnodes.push_back(to_node(v->prim_nodes[k]));
  if (v->num_prims) s->pidx.assign(v->prim_indices, v->prim_indices + v->num_prims);
  for (int k = 0; k < v->num_instances; ++k) {
    const xb_instance_view& iv = v->instances[k];
    Inst in;
    in.geom = iv.geom;
    in.id = iv.instance_id;
    for (int c = 0; c < 4; ++c) {
      in.l2w[c] = V(iv.local_to_world[3 * c], iv.local_to_world[3 * c + 1], iv.local_to_world[3 * c + 2]);
      in.w2l[c] = V(iv.world_to_local[3 * c], iv.world_to_local[3 * c + 1], iv.world_to_local[3 * c + 2]);
    }
    s->insts.push_back(in);
  }
  for (int k = 0; k < v->num_tlas_nodes; ++k) s->tlas.push_back(to_node(v->tlas_nodes[k]));
  s->tinst.assign(v->tlas_inst_indices, v->tlas_inst_indices + v->num_instances);
  for (int k = 0; k < v->num_materials; ++k) s->mats.push_back(prepare(v->materials[k]));
  s->lights.assign(v->lights, v->lights + v->num_lights);
  s->suns.assign(v->suns, v->suns + v->num_suns);
  s->sky = v->sky;
  return s;
}

void xo_scene_free(void* s) { delete static_cast<Scene*>(s); }

int xo_trace(void* sp, int64_t n, const xb_ray* rays, xb_hit* hits, int mode, int64_t* work) {
  const Scene& sc = *static_cast<Scene*>(sp);
  Work wk;
  for (int64_t i = 0; i < n; ++i) {
    Ray r{V(rays[i].org[0], rays[i].org[1], rays[i].org[2]), V(rays[i].dir[0], rays[i].dir[1], rays[i].dir[2]),
          rays[i].tmin, rays[i].tmax};
    if (mode == 0) {
      Hit h;
      bool hit = scene_closest(sc, r, h, wk);
      fill_hit(h, hit, &hits[i]);
    } else {
      fill_hit(Hit(), false, &hits[i]);
      if (scene_any(sc, r, wk)) hits[i].t = 0.f;
    }
  }
  if (work) { work[0] += wk.nodes; work[1] += wk.tris; work[2] += wk.tlas; work[3] += wk.inst; }
  return 0;
}

void xo_material_prepare(const xb_material* p, xb_material_derived* out) {
  Mat m = prepare(*p);
  out->alpha = m.alpha; out->alpha_x = m.ax; out->alpha_y = m.ay;
  out->f0[0] = m.f0.x; out->f0[1] = m.f0.y; out->f0[2] = m.f0.z;
  bool emissive = p->emission[0] > 0.f || p->emission[1] > 0.f || p->emission[2] > 0.f;
  out->flags = (m.conductor ? XB_MAT_CONDUCTOR : 0) | (m.transmissive ? XB_MAT_TRANSMISSIVE : 0) |
               (m.sss ? XB_MAT_SUBSURFACE : 0) | (m.delta ? XB_MAT_DELTA : 0) | (emissive ? XB_MAT_EMISSIVE : 0);
}

void xo_bsdf_eval(const xb_material* p, int64_t n, const float* wo, const float* wi, float* f, float* pd) {
  Mat m = prepare(*p);
  for (int64_t i = 0; i < n; ++i) {
    V o(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]), w(wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]);
    V fv = eval(o, w, m);
    f[3 * i] = fv.x; f[3 * i + 1] = fv.y; f[3 * i + 2] = fv.z;
    pd[i] = pdf(o, w, m);
  }
}

void xo_bsdf_sample(const xb_material* p, int64_t n, const float* wo, uint64_t* states, float* wi,
                    float* f, float* pd, int32_t* flags) {
  Mat m = prepare(*p);
  for (int64_t i = 0; i < n; ++i) {
    Pcg g{states[i]};
    V o(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]);
    Smp s;
    bool ok = sample(o, m, g, s);
    states[i] = g.s;
    wi[3 * i] = s.wi.x; wi[3 * i + 1] = s.wi.y; wi[3 * i + 2] = s.wi.z;
    f[3 * i] = s.f.x; f[3 * i + 1] = s.f.y; f[3 * i + 2] = s.f.z;
    pd[i] = s.pdf;
    flags[i] = (ok ? 1 : 0) | (s.delta ? 2 : 0);
  }
}

uint64_t xo_seed_pcg(uint64_t seed) { return seed_state(seed); }

int xo_render(void* sp, const xb_camera* cam, int W, int H, int min_b, int max_b, int spp_first,
              int spp_count, double* sum, int64_t* rays, int threads) {
  const Scene& sc = *static_cast<Scene*>(sp);
  if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
  std::atomic<int> next{0};
  std::atomic<int64_t> nc{0}, ns{0};
  auto work = [&]() {
    int64_t c = 0, s = 0;
    for (;;) {
      const int y = next.fetch_add(1);
      if (y >= H) break;
      for (int x = 0; x < W; ++x) {
        double a0 = 0, a1 = 0, a2 = 0;
        for (int k = 0; k < spp_count; ++k) {
          V L = trace_path(sc, *cam, W, H, x, y, spp_first + k, min_b, max_b, c, s);
          a0 += L.x; a1 += L.y; a2 += L.z;
        }
        const size_t d = ((size_t)(H - 1 - y) * W + x) * 3;
        sum[d] += a0; sum[d + 1] += a1; sum[d + 2] += a2;
      }
    }
    nc += c;
    ns += s;
  };
  std::vector<std::thread> th;
  for (int t = 0; t < threads; ++t) th.emplace_back(work);
  for (auto& t : th) t.join();
  if (rays) { rays[0] += nc.load(); rays[1] += ns.load(); }
  return 0;
}

}  // extern "C"
