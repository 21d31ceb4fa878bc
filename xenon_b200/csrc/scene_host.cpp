// scene_host.cpp — the host side of the scene: material preparation, mesh utilities,
// binned-SAH BLAS / PrimBLAS / TLAS build, and the flattened view handed to the device.
//
// The build restates the reference's algorithm step for step so that node arrays are
// bit-identical (the device traversal then visits nodes in the reference's order, which is
// what decides equal-t ties): src/geometry/blas.cpp:97-205 (12 bins, leaves of <= 2, leaf
// cost check, std::partition then nth_element fallback), src/geometry/prim_blas.cpp:34-134
// (same for analytic prims) and src/geometry/tlas.cpp:34-128 (8 bins, leaves of 1).
// Compiled with -ffp-contract=off.

#include "scene_host.h"
#include "bvh_build.h"
#include "bvh_refit.h"
#include "refit_kernels.h"

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <exception>
#include <future>
#include <stdexcept>
#include <thread>

namespace xb {

HostScene::HostScene() {
  // Environment defaults (src/scene/environment.h:15-19): the sky is on by default.
  sky = xb_sky{{0.10f, 0.30f, 0.80f}, {0.55f, 0.70f, 0.85f}, {0.10f, 0.08f, 0.05f}, 3.0f, 1.0f};
}

void default_material(xb_material* m) {
  // Material defaults (src/material/material.h:23-35).
  std::memset(m, 0, sizeof(*m));
  m->base_color[0] = m->base_color[1] = m->base_color[2] = 0.5f;
  m->roughness = 0.5f;
  m->metallic = 0.f;
  m->ior = 1.5f;
  m->subsurface_color[0] = m->subsurface_color[1] = m->subsurface_color[2] = 1.f;
  m->subsurface_mfp[0] = m->subsurface_mfp[1] = m->subsurface_mfp[2] = 1.f;
  m->clearcoat_roughness = 0.03f;
  m->emission_temperature = 6500.f;
}

// material_prepare (src/material/material.h:55-75)
xb_material_derived prepare_material(const xb_material& m) {
  xb_material_derived d{};
  d.alpha = std::max(m.roughness * m.roughness, 1e-6f);
  float aspect = std::sqrt(1.0f - 0.9f * std::abs(m.anisotropy));
  d.alpha_x = std::max(d.alpha / aspect, 1e-6f);
  d.alpha_y = std::max(d.alpha * aspect, 1e-6f);
  float f0d = ((m.ior - 1.0f) * (m.ior - 1.0f)) / ((m.ior + 1.0f) * (m.ior + 1.0f));
  F3 base(m.base_color[0], m.base_color[1], m.base_color[2]);
  F3 f0 = lerp3(F3::splat(f0d), base, m.metallic);
  d.f0[0] = f0.x; d.f0[1] = f0.y; d.f0[2] = f0.z;
  int fl = 0;
  if (m.metallic > 0.5f) fl |= XB_MAT_CONDUCTOR;
  if (m.transmission > 0.01f) fl |= XB_MAT_TRANSMISSIVE;
  if (m.subsurface > 0.01f) fl |= XB_MAT_SUBSURFACE;
  if (d.alpha < 0.001f) fl |= XB_MAT_DELTA;
  if (m.emission[0] > 0.f || m.emission[1] > 0.f || m.emission[2] > 0.f) fl |= XB_MAT_EMISSIVE;
  d.flags = fl;
  return d;
}

// TriangleMesh::compute_smooth_normals (src/geometry/mesh.cpp:13-35): area-weighted sums.
void HostMesh::compute_smooth_normals() {
  const int nv = num_vertices(), nt = num_triangles();
  nx.assign(nv, 0.f); ny.assign(nv, 0.f); nz.assign(nv, 0.f);
  for (int t = 0; t < nt; ++t) {
    const int i0 = indices[3 * t], i1 = indices[3 * t + 1], i2 = indices[3 * t + 2];
    F3 p0 = vertex(i0), p1 = vertex(i1), p2 = vertex(i2);
    F3 fn = cross3(p1 - p0, p2 - p0);
    for (int i : {i0, i1, i2}) { nx[i] += fn.x; ny[i] += fn.y; nz[i] += fn.z; }
  }
  for (int i = 0; i < nv; ++i) {
    F3 n = normalize3(F3(nx[i], ny[i], nz[i]));
    nx[i] = n.x; ny[i] = n.y; nz[i] = n.z;
  }
}

// TriangleMesh::transform (src/geometry/mesh.cpp:156-205): scale, then Y, X, Z rotations,
// then translate; normals rotated and renormalised. The degree→radian factor is the double
// M_PI / 180 narrowed to float, as in the reference.
void HostMesh::transform(F3 pos, float scale, F3 rot_deg) {
  const float k = (float)(3.14159265358979323846 / 180.f);
  F3 rad = rot_deg * k;
  const float cx = std::cos(rad.x), sx = std::sin(rad.x);
  const float cy = std::cos(rad.y), sy = std::sin(rad.y);
  const float cz = std::cos(rad.z), sz = std::sin(rad.z);
  auto rotate = [&](F3 v) {
    float ax = v.x * cy + v.z * sy;
    float az = -v.x * sy + v.z * cy;
    v.x = ax; v.z = az;
    float ay = v.y * cx - v.z * sx;
    az = v.y * sx + v.z * cx;
    v.y = ay; v.z = az;
    ax = v.x * cz - v.y * sz;
    ay = v.x * sz + v.y * cz;
    v.x = ax; v.y = ay;
    return v;
  };
  for (size_t i = 0; i < vx.size(); ++i) {
    F3 v(vx[i], vy[i], vz[i]);
    v = v * scale;
    v = rotate(v);
    v = v + pos;
    vx[i] = v.x; vy[i] = v.y; vz[i] = v.z;
  }
  for (size_t i = 0; i < nx.size(); ++i) {
    F3 n = normalize3(rotate(F3(nx[i], ny[i], nz[i])));
    nx[i] = n.x; ny[i] = n.y; nz[i] = n.z;
  }
}

// AffineTransform::from_trs (src/geometry/transform.h:105-146): M = Rz * (Rx * Ry),
// local_to_world = s*M + t, world_to_local = M^T / s with translation -(M^T/s) t.
Affine affine_from_trs(F3 t, float s, F3 rot_deg, Affine* inv) {
  const float k = kPiF / 180.f;
  F3 rad = rot_deg * k;
  const float cx = std::cos(rad.x), sx = std::sin(rad.x);
  const float cy = std::cos(rad.y), sy = std::sin(rad.y);
  const float cz = std::cos(rad.z), sz = std::sin(rad.z);
  const float rxy[3][3] = {{cy, 0.f, sy}, {sx * sy, cx, -sx * cy}, {-cx * sy, sx, cx * cy}};
  const float rz[3][3] = {{cz, -sz, 0}, {sz, cz, 0}, {0, 0, 1}};
  float m[3][3] = {};
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c)
      for (int q = 0; q < 3; ++q) m[r][c] += rz[r][q] * rxy[q][c];
  Affine l2w;
  for (int j = 0; j < 3; ++j) l2w.c[j] = F3(m[0][j] * s, m[1][j] * s, m[2][j] * s);
  l2w.c[3] = t;
  const float is = 1.f / s;
  for (int j = 0; j < 3; ++j) inv->c[j] = F3(m[j][0] * is, m[j][1] * is, m[j][2] * is);
  inv->c[3] = F3(-(m[0][0] * t.x + m[1][0] * t.y + m[2][0] * t.z) * is,
                 -(m[0][1] * t.x + m[1][1] * t.y + m[2][1] * t.z) * is,
                 -(m[0][2] * t.x + m[1][2] * t.y + m[2][2] * t.z) * is);
  return l2w;
}

// Analytic prim bounds (src/geometry/primitives.h: Sphere 97-100, Plane 134-148, Box 203-205,
// Disk 250-261, Quad 307-317).
Bounds prim_bounds(const xb_prim& q) {
  const float* p = q.p;
  Bounds b;
  switch (q.type) {
    case XB_PRIM_SPHERE: {
      F3 c(p[0], p[1], p[2]), r = F3::splat(p[3]);
      b.mn = c - r; b.mx = c + r;
      break;
    }
    case XB_PRIM_PLANE: {
      const float kHuge = 1e4f;
      F3 n(p[0], p[1], p[2]);
      float off = p[3];
      F3 an(std::abs(n.x), std::abs(n.y), std::abs(n.z));
      b.mn = F3::splat(-kHuge) + n * (off - 0.01f);
      b.mx = F3::splat(kHuge) + n * (off + 0.01f);
      for (int i = 0; i < 3; ++i)
        if (an[i] > 0.9f) { b.mn.at(i) = off - 0.01f; b.mx.at(i) = off + 0.01f; }
      break;
    }
    case XB_PRIM_BOX: {
      F3 c(p[0], p[1], p[2]), h(p[3], p[4], p[5]);
      b.mn = c - h; b.mx = c + h;
      break;
    }
    case XB_PRIM_DISK: {
      F3 c(p[0], p[1], p[2]), n(p[3], p[4], p[5]);
      float r = p[6];
      F3 e(r * std::sqrt(1.f - n.x * n.x), r * std::sqrt(1.f - n.y * n.y),
           r * std::sqrt(1.f - n.z * n.z));
      e = max3(e, F3::splat(0.001f));
      b.mn = c - e; b.mx = c + e;
      break;
    }
    default: {
      F3 o(p[0], p[1], p[2]), u(p[3], p[4], p[5]), v(p[6], p[7], p[8]);
      b.grow(o); b.grow(o + u); b.grow(o + v); b.grow(o + u + v);
      b.mn = b.mn - F3::splat(0.001f);
      b.mx = b.mx + F3::splat(0.001f);
      break;
    }
  }
  return b;
}

// The SAH sweep over the bins of a split (src/geometry/blas.cpp:128-146): prefix and suffix
// counts and areas, cost (A_l N_l + A_r N_r) / A_node per plane, the first minimum.
int sah_best_split(const Bounds* bin_box, const int* bin_cnt, int bins, const Bounds& node_box,
                   float* best_cost) {
  float l_area[16], r_area[16];
  int l_cnt[16], r_cnt[16];
  Bounds acc;
  int run = 0;
  for (int i = 0; i < bins - 1; ++i) {
    run += bin_cnt[i]; l_cnt[i] = run;
    acc.grow(bin_box[i]); l_area[i] = acc.area();
  }
  acc = Bounds();
  run = 0;
  for (int i = bins - 1; i > 0; --i) {
    run += bin_cnt[i]; r_cnt[i - 1] = run;
    acc.grow(bin_box[i]); r_area[i - 1] = acc.area();
  }
  const float parent = node_box.area();
  float best = kInf;
  int best_bin = -1;
  for (int i = 0; i < bins - 1; ++i) {
    const float c = (l_area[i] * l_cnt[i] + r_area[i] * r_cnt[i]) / parent;
    if (c < best) { best = c; best_bin = i; }
  }
  *best_cost = best;
  return best_bin;
}

namespace {

// Binned-SAH BVH build in the reference's node allocation order: root 0, then each split
// allocates its two children as a contiguous pair and recurses left before right.
//
// With par_depth > 0, the two subtrees of a split over at least kParallelItems items are built
// at once (the left one on another thread), each into a node array of its own, down to
// par_depth levels. They work on disjoint ranges of the items and of `order`, and their node
// arrays are then placed where the one-thread build allocates them — the subtree roots in the
// pair, then the left subtree's other nodes, then the right's, child indices shifted — so the
// arrays are the same whatever the thread count.
class BvhBuilder {
 public:
  BvhBuilder(int bins, uint32_t max_leaf, bool leaf_cost, int par_depth = 0)
      : bins_(bins), max_leaf_(max_leaf), leaf_cost_(leaf_cost), par_depth_(par_depth) {}

  void build(std::vector<BuildItem>& items, std::vector<xb_bvh_node>& nodes,
             std::vector<uint32_t>& order) {
    nodes.clear();
    order.assign(items.size(), 0);
    if (items.empty()) return;
    nodes_ = &nodes;
    order_ = &order;
    nodes.reserve(items.size() * 2);
    nodes.emplace_back();
    split(0, 0, (uint32_t)items.size(), items);
  }

 private:
  static constexpr uint32_t kParallelItems = 16384;
  int bins_;
  uint32_t max_leaf_;
  bool leaf_cost_;
  int par_depth_;
  std::vector<xb_bvh_node>* nodes_ = nullptr;
  std::vector<uint32_t>* order_ = nullptr;

  // The subtree over items [lo, hi) into `local`, its root at local index 0.
  void build_subtree(std::vector<xb_bvh_node>& local, uint32_t lo, uint32_t hi, std::vector<BuildItem>& it) {
    nodes_ = &local;
    local.reserve((size_t)(hi - lo) * 2);
    local.emplace_back();
    split(0, lo, hi, it);
  }
  // Local node j >= 1 of a subtree goes to base + j - 1; interior nodes' children move along
  // (a leaf's child is an item offset and stays).
  static xb_bvh_node placed(xb_bvh_node n, uint32_t base) {
    if (n.count == 0) n.child = base + n.child - 1;
    return n;
  }

  void set_box(uint32_t node, const Bounds& b) {
    xb_bvh_node& n = (*nodes_)[node];
    n.mn[0] = b.mn.x; n.mn[1] = b.mn.y; n.mn[2] = b.mn.z;
    n.mx[0] = b.mx.x; n.mx[1] = b.mx.y; n.mx[2] = b.mx.z;
  }
  void leaf(uint32_t node, uint32_t lo, uint32_t hi, const std::vector<BuildItem>& it) {
    (*nodes_)[node].child = lo;
    (*nodes_)[node].count = hi - lo;
    for (uint32_t i = lo; i < hi; ++i) (*order_)[i] = it[i].index;
  }
  int bin_of(const BuildItem& p, int axis, float lo, float scale) const {
    int b = (int)((p.centroid[axis] - lo) * scale);
    return b >= bins_ ? bins_ - 1 : b;
  }

  void split(uint32_t node, uint32_t lo, uint32_t hi, std::vector<BuildItem>& it) {
    Bounds nb;
    for (uint32_t i = lo; i < hi; ++i) nb.grow(it[i].box);
    set_box(node, nb);
    const uint32_t count = hi - lo;
    if (count <= max_leaf_) { leaf(node, lo, hi, it); return; }

    Bounds cb;
    for (uint32_t i = lo; i < hi; ++i) cb.grow(it[i].centroid);
    const int axis = max_axis3(cb.extent());
    const float ext = cb.extent()[axis];
    if (ext == 0.f) { leaf(node, lo, hi, it); return; }

    const float scale = (float)bins_ / ext;
    const float cmin = cb.mn[axis];
    Bounds bin_box[16];
    int bin_cnt[16] = {};
    for (uint32_t i = lo; i < hi; ++i) {
      int b = bin_of(it[i], axis, cmin, scale);
      bin_cnt[b]++;
      bin_box[b].grow(it[i].box);
    }
    float best;
    const int best_bin = sah_best_split(bin_box, bin_cnt, bins_, nb, &best);
    if ((leaf_cost_ && best >= (float)count) || best_bin < 0) { leaf(node, lo, hi, it); return; }

    auto mid_it = std::partition(it.begin() + lo, it.begin() + hi, [&](const BuildItem& p) {
      return bin_of(p, axis, cmin, scale) <= best_bin;
    });
    uint32_t mid = (uint32_t)(mid_it - it.begin());
    if (mid == lo || mid == hi) {
      mid = lo + count / 2;
      std::nth_element(it.begin() + lo, it.begin() + mid, it.begin() + hi,
                       [axis](const BuildItem& a, const BuildItem& b) {
                         return a.centroid[axis] < b.centroid[axis];
                       });
    }
    const uint32_t left = (uint32_t)nodes_->size();
    nodes_->emplace_back();
    nodes_->emplace_back();
    (*nodes_)[node].child = left;
    (*nodes_)[node].count = 0;
    if (par_depth_ > 0 && count >= kParallelItems) {
      std::vector<xb_bvh_node> ln, rn;
      BvhBuilder lb(bins_, max_leaf_, leaf_cost_, par_depth_ - 1), rb(lb);
      lb.order_ = rb.order_ = order_;
      auto done = std::async(std::launch::async, [&] { lb.build_subtree(ln, lo, mid, it); });
      rb.build_subtree(rn, mid, hi, it);
      done.get();
      std::vector<xb_bvh_node>& nodes = *nodes_;
      const uint32_t base_l = (uint32_t)nodes.size(), base_r = base_l + (uint32_t)ln.size() - 1;
      nodes[left] = placed(ln[0], base_l);
      nodes[left + 1] = placed(rn[0], base_r);
      for (size_t j = 1; j < ln.size(); ++j) nodes.push_back(placed(ln[j], base_l));
      for (size_t j = 1; j < rn.size(); ++j) nodes.push_back(placed(rn[j], base_r));
      return;
    }
    split(left, lo, mid, it);
    split(left + 1, mid, hi, it);
  }
};

Bounds node_bounds(const xb_bvh_node& n) {
  Bounds b;
  b.mn = F3(n.mn[0], n.mn[1], n.mn[2]);
  b.mx = F3(n.mx[0], n.mx[1], n.mx[2]);
  return b;
}

}  // namespace

void HostScene::build() {
  // Per-mesh BLAS (BLAS::build, blas.cpp:183-205): meshes on a pool of threads, and the large
  // subtrees of each mesh on threads of their own (BvhBuilder); the arrays do not depend on it.
  const int threads = build_threads > 0 ? build_threads : std::max(1, (int)std::thread::hardware_concurrency());
  int par_depth = 0;
  while (par_depth < 4 && (2 << par_depth) <= threads) ++par_depth;
  auto build_mesh = [&](HostMesh& m) {
    if (build_mode == 2) {   // the items are made on the device too
      build_bvh_device_mesh(m, 12, 2, true, m.nodes, m.prims);
      return;
    }
    std::vector<BuildItem> items(m.num_triangles());
    for (int t = 0; t < m.num_triangles(); ++t) {
      Bounds b;
      b.grow(m.vertex(m.indices[3 * t]));
      b.grow(m.vertex(m.indices[3 * t + 1]));
      b.grow(m.vertex(m.indices[3 * t + 2]));
      items[t] = {b, b.center(), (uint32_t)t};
    }
    if (build_mode == 1) build_bvh_levels(items, 12, 2, true, m.nodes, m.prims);
    else BvhBuilder(12, 2, true, par_depth).build(items, m.nodes, m.prims);
  };
  std::atomic<size_t> next{0};
  std::vector<std::exception_ptr> failed(meshes.size());
  auto worker = [&] {
    for (size_t i = next++; i < meshes.size(); i = next++) {
      try {
        build_mesh(meshes[i]);
      } catch (...) {   // rethrown below, on the calling thread
        failed[i] = std::current_exception();
      }
    }
  };
  std::vector<std::thread> pool;
  const int mesh_threads = build_mode == 2 ? 1 : threads;   // device builds: one mesh at a time
  for (int k = 1; k < std::min<int>(mesh_threads, (int)meshes.size()); ++k) pool.emplace_back(worker);
  worker();
  for (std::thread& t : pool) t.join();
  for (const std::exception_ptr& e : failed)
    if (e) std::rethrow_exception(e);
  // PrimBLAS (prim_blas.cpp:114-134)
  prim_nodes.clear();
  prim_indices.clear();
  if (!prims.empty()) {
    std::vector<BuildItem> items(prims.size());
    for (size_t i = 0; i < prims.size(); ++i) {
      Bounds b = prim_bounds(prims[i]);
      items[i] = {b, b.center(), (uint32_t)i};
    }
    if (build_mode == 2) build_bvh_device(items, 12, 2, true, prim_nodes, prim_indices);
    else if (build_mode == 1) build_bvh_levels(items, 12, 2, true, prim_nodes, prim_indices);
    else BvhBuilder(12, 2, true).build(items, prim_nodes, prim_indices);
  }
  // Instances: explicit ones, or one identity instance per mesh + one for the prim group
  // (Scene::build_acceleration, scene.h:79-121).
  instances.clear();
  if (!explicit_instances.empty()) {
    instances = explicit_instances;
  } else {
    int id = 0;
    for (size_t i = 0; i < meshes.size(); ++i)
      instances.push_back({(int32_t)i, id++, Affine::identity(), Affine::identity()});
    if (!prims.empty()) instances.push_back({XB_GEOM_PRIMS, id++, Affine::identity(), Affine::identity()});
  }
  build_tlas();
  built = true;
}

void HostScene::build_tlas() {
  std::vector<Affine> l2w;
  std::vector<const xb_bvh_node*> roots;
  for (const HostInstance& in : instances) {
    l2w.push_back(in.l2w);
    const xb_bvh_node* root = nullptr;
    if (in.geom >= 0) {
      if (!meshes[in.geom].nodes.empty()) root = &meshes[in.geom].nodes[0];
    } else if (!prim_nodes.empty()) {
      root = &prim_nodes[0];
    }
    roots.push_back(root);
  }
  xb::build_tlas(l2w, roots, tlas_nodes, tlas_inst, build_mode);
}

// TLAS over world AABBs of the 8 transformed root-box corners (tlas.cpp:116-128,
// transform.h:78-89, Instance::rebuild_world_aabb tlas.h:51-53).
void build_tlas(const std::vector<Affine>& l2w, const std::vector<const xb_bvh_node*>& roots,
                std::vector<xb_bvh_node>& nodes, std::vector<uint32_t>& order, int mode) {
  std::vector<BuildItem> items(l2w.size());
  for (size_t i = 0; i < l2w.size(); ++i) {
    Bounds local;
    if (roots[i]) local = node_bounds(*roots[i]);
    Bounds w;
    for (int c = 0; c < 8; ++c)
      w.grow(l2w[i].point(F3((c & 1) ? local.mx.x : local.mn.x, (c & 2) ? local.mx.y : local.mn.y,
                             (c & 4) ? local.mx.z : local.mn.z)));
    items[i] = {w, w.center(), (uint32_t)i};
  }
  if (mode == 2) build_bvh_device(items, 8, 1, false, nodes, order);
  else if (mode == 1) build_bvh_levels(items, 8, 1, false, nodes, order);
  else BvhBuilder(8, 1, false).build(items, nodes, order);
}

void refit_blas(const HostMesh& m, std::vector<xb_bvh_node>& nodes) {
  // the mesh packed as the renderer uploads it (node and slot bases 0), then the device refit's
  // passes run as loops over their thread indices (refit_kernels.h)
  const int32_t nn = (int32_t)nodes.size(), nt = m.num_triangles();
  if (nn == 0) return;
  auto bits = [](uint32_t u) { float f; std::memcpy(&f, &u, sizeof(f)); return f; };
  std::vector<Quad> blas(2 * (size_t)nn), tris(3 * (size_t)nt);
  for (int32_t i = 0; i < nn; ++i) {
    const xb_bvh_node& n = nodes[i];
    blas[2 * i] = Quad{n.mn[0], n.mn[1], n.mn[2], n.mx[0]};
    blas[2 * i + 1] = Quad{n.mx[1], n.mx[2], bits(n.child), bits(n.count)};
  }
  for (int32_t s = 0; s < nt; ++s) tris[3 * s].w = bits(m.prims[s]);
  std::vector<float> pos(3 * (size_t)m.num_vertices());
  for (int v = 0; v < m.num_vertices(); ++v) { pos[3 * v] = m.vx[v]; pos[3 * v + 1] = m.vy[v]; pos[3 * v + 2] = m.vz[v]; }
  std::vector<int32_t> parent(nn, -1);
  std::vector<uint32_t> arrivals(nn, 0);
  int32_t status = 0;
  RefitArgs a;
  a.blas = blas.data();
  a.tris = tris.data();
  a.tri_index = m.indices.data();
  a.pos = pos.data();
  a.parent = parent.data();
  a.arrivals = arrivals.data();
  a.status = &status;
  a.node_base = 0;
  a.slot_base = 0;
  a.num_nodes = nn;
  a.num_tris = nt;
  a.num_verts = m.num_vertices();
  a.tri_offset = 0;
  a.vtx_offset = 0;
  for (int32_t s = 0; s < nt; ++s) refit_tris_at(a, s);
  for (int32_t i = 0; i < nn; ++i) refit_parents_at(a, i);
  for (int32_t i = 0; i < nn; ++i) refit_nodes_at(a, i);
  if (status != 0) throw std::invalid_argument("refit: malformed BLAS");
  for (int32_t i = 0; i < nn; ++i) {
    xb_bvh_node& n = nodes[i];
    n.mn[0] = blas[2 * i].x; n.mn[1] = blas[2 * i].y; n.mn[2] = blas[2 * i].z;
    n.mx[0] = blas[2 * i].w; n.mx[1] = blas[2 * i + 1].x; n.mx[2] = blas[2 * i + 1].y;
  }
}

void HostScene::refit_mesh(int mesh, const float* positions, const float* normals) {
  HostMesh& m = meshes[mesh];
  for (int i = 0; i < m.num_vertices(); ++i) {
    m.vx[i] = positions[3 * i]; m.vy[i] = positions[3 * i + 1]; m.vz[i] = positions[3 * i + 2];
  }
  if (normals) {
    m.nx.resize(m.num_vertices()); m.ny.resize(m.num_vertices()); m.nz.resize(m.num_vertices());
    for (int i = 0; i < m.num_vertices(); ++i) {
      m.nx[i] = normals[3 * i]; m.ny[i] = normals[3 * i + 1]; m.nz[i] = normals[3 * i + 2];
    }
  }
  refit_blas(m, m.nodes);
  const int mode = build_mode;
  build_mode = 0;   // the TLAS over the new root boxes is rebuilt on the host (same arrays)
  build_tlas();
  build_mode = mode;
}

void HostScene::view(xb_scene_view* v) {
  std::memset(v, 0, sizeof(*v));
  mesh_views_.clear();
  for (const HostMesh& m : meshes) {
    xb_mesh_view mv{};
    mv.num_vertices = m.num_vertices();
    mv.num_triangles = m.num_triangles();
    mv.vx = m.vx.data(); mv.vy = m.vy.data(); mv.vz = m.vz.data();
    if (!m.nx.empty()) { mv.nx = m.nx.data(); mv.ny = m.ny.data(); mv.nz = m.nz.data(); }
    mv.indices = m.indices.data();
    mv.mat_ids = m.mat_ids.data();
    mv.blas_nodes = m.nodes.data();
    mv.num_blas_nodes = (int32_t)m.nodes.size();
    mv.blas_prims = m.prims.data();
    mesh_views_.push_back(mv);
  }
  v->num_meshes = (int32_t)mesh_views_.size();
  v->meshes = mesh_views_.data();
  v->num_prims = (int32_t)prims.size();
  v->prims = prims.data();
  v->prim_nodes = prim_nodes.data();
  v->num_prim_nodes = (int32_t)prim_nodes.size();
  v->prim_indices = prim_indices.data();
  inst_views_.clear();
  for (const HostInstance& in : instances) {
    xb_instance_view iv{};
    iv.geom = in.geom;
    iv.instance_id = in.instance_id;
    for (int c = 0; c < 4; ++c) {
      iv.local_to_world[3 * c] = in.l2w.c[c].x; iv.local_to_world[3 * c + 1] = in.l2w.c[c].y;
      iv.local_to_world[3 * c + 2] = in.l2w.c[c].z;
      iv.world_to_local[3 * c] = in.w2l.c[c].x; iv.world_to_local[3 * c + 1] = in.w2l.c[c].y;
      iv.world_to_local[3 * c + 2] = in.w2l.c[c].z;
    }
    inst_views_.push_back(iv);
  }
  v->num_instances = (int32_t)inst_views_.size();
  v->instances = inst_views_.data();
  v->tlas_nodes = tlas_nodes.data();
  v->num_tlas_nodes = (int32_t)tlas_nodes.size();
  v->tlas_inst_indices = tlas_inst.data();
  v->num_materials = (int32_t)materials.size();
  v->materials = materials.data();
  v->num_lights = (int32_t)lights.size();
  v->lights = lights.data();
  v->num_suns = (int32_t)suns.size();
  v->suns = suns.data();
  v->sky = sky;
}

}  // namespace xb

namespace xb {

bool light_geometry(const xb_scene_view& v, const xb_light& l, LightGeom* out) {
  if ((int)l.mesh_id >= v.num_meshes) return false;
  const xb_mesh_view& m = v.meshes[l.mesh_id];
  if ((int)l.tri_idx >= m.num_triangles) return false;
  F3 p[3];
  for (int k = 0; k < 3; ++k) {
    const int i = m.indices[3 * l.tri_idx + k];
    p[k] = F3(m.vx[i], m.vy[i], m.vz[i]);
  }
  F3 n = normalize3(cross3(p[1] - p[0], p[2] - p[0]));
  for (int k = 0; k < 3; ++k) {
    float* dst = k == 0 ? out->p0 : (k == 1 ? out->p1 : out->p2);
    dst[0] = p[k].x; dst[1] = p[k].y; dst[2] = p[k].z;
  }
  out->n[0] = n.x; out->n[1] = n.y; out->n[2] = n.z;
  return true;
}

void multiscatter_constants(const xb_material_derived& d, float* k1, float* k2, float fms[3]) {
  const float a = d.alpha;
  *k1 = 5.0f * std::exp(-2.69f * a);
  *k2 = 1.0f + 22.7f * std::pow(a, 1.5f);
  const float eavg = 1.0f / (1.0f + 0.3037f * a + 0.1218f * a * a);
  const F3 f0(d.f0[0], d.f0[1], d.f0[2]);
  const F3 favg = (F3::splat(1.f) + f0 * 20.f) * (1.f / 21.f);
  float denom = 1.f - favg.x * (1.f - eavg);
  denom = std::max(denom, 1e-4f);
  // F_avg * F_avg * E_avg / Vec3(denom): component products, then component division
  const F3 t = F3(favg.x * favg.x, favg.y * favg.y, favg.z * favg.z) * eavg;
  fms[0] = t.x / denom; fms[1] = t.y / denom; fms[2] = t.z / denom;
}

void sun_emission(const xb_sun& s, float out[3]) {
  F3 e = F3(s.color[0], s.color[1], s.color[2]) * s.intensity;
  out[0] = e.x; out[1] = e.y; out[2] = e.z;
}

}  // namespace xb
