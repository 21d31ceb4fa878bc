// oracle/ref_driver.cpp — headless C API over the reference's own CPU sources.
//
// Test infrastructure only: compiled together with the reference's geometry, material,
// render and scene sources (oracle/Makefile) into oracle/_ref/. It replaces the reference's
// main.cpp + GLFW window (src/main.cpp:54-190) with plain calls:
//   * build a Scene from arrays (meshes, prims, lights, sky) and run its own
//     Scene::build_acceleration (src/scene/scene.h:79-121) or TLAS::build over explicit
//     AffineTransform::from_trs instances (src/geometry/tlas.cpp:116, transform.h:105);
//   * export that Scene as an xb_scene_view (the BVH arrays the reference built);
//   * Scene::intersect / intersects on ray batches (src/scene/scene.h:124-129);
//   * bsdf_eval_for_nee / bsdf_pdf_for_nee / bsdf_sample (src/material/bsdf.h:601-708);
//   * WavefrontRenderer::render_frame_tiled (src/render/cpu_tiled.cpp:13) per sample index, with
//     the per-sample radiance summed in FP64 here.
//
// WavefrontRenderer keeps its accumulator and sample counter private and PrimBLAS keeps its
// node arrays private; this driver opens them (the `private` redefinition below) only to run
// sample k alone and to read the nodes, without changing any reference code.

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <deque>
#include <filesystem>
#include <fstream>
#include <functional>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <thread>
#include <type_traits>
#include <unordered_map>
#include <utility>
#include <variant>
#include <vector>
#include <immintrin.h>

#define private public
#include "render/wavefront.h"
#include "scene/scene_file.h"
#include "material/bsdf.h"
#include "math/image.h"
#undef private

#include "../include/xenon_b200.h"

using namespace xn;

namespace {

struct RefScene {
  Scene scene;
  std::vector<xb_material> mats_pod;       // authoring params as added (for the view)
  struct PendingInst { int geom; Vec3 t; float s; Vec3 rot; int id; };
  std::vector<PendingInst> pending;
  // view storage
  std::vector<xb_mesh_view> mesh_views;
  std::vector<xb_instance_view> inst_views;
  std::vector<xb_prim> prims_pod;
  std::vector<xb_light> lights_pod;
  std::vector<xb_sun> suns_pod;
  bool built = false;
};

Material to_material(const xb_material& p) {
  Material m;
  m.baseColor = Vec3(p.base_color[0], p.base_color[1], p.base_color[2]);
  m.roughness = p.roughness;
  m.metallic = p.metallic;
  m.ior = p.ior;
  m.transmission = p.transmission;
  m.subsurface = p.subsurface;
  m.subsurfaceColor = Vec3(p.subsurface_color[0], p.subsurface_color[1], p.subsurface_color[2]);
  m.subsurfaceMFP = Vec3(p.subsurface_mfp[0], p.subsurface_mfp[1], p.subsurface_mfp[2]);
  m.clearcoat = p.clearcoat;
  m.clearcoatRoughness = p.clearcoat_roughness;
  m.anisotropy = p.anisotropy;
  m.emission = Vec3(p.emission[0], p.emission[1], p.emission[2]);
  m.emissionTemperature = p.emission_temperature;
  material_prepare(m);
  return m;
}

xb_prim prim_to_pod(const PrimVariant& v) {
  xb_prim q{};
  std::visit([&](const auto& p) {
    using T = std::decay_t<decltype(p)>;
    q.mat_id = p.mat_id;
    if constexpr (std::is_same_v<T, Sphere>) {
      q.type = XB_PRIM_SPHERE;
      q.p[0] = p.center.x; q.p[1] = p.center.y; q.p[2] = p.center.z; q.p[3] = p.radius;
    } else if constexpr (std::is_same_v<T, Plane>) {
      q.type = XB_PRIM_PLANE;
      q.p[0] = p.normal.x; q.p[1] = p.normal.y; q.p[2] = p.normal.z; q.p[3] = p.offset;
    } else if constexpr (std::is_same_v<T, Box>) {
      q.type = XB_PRIM_BOX;
      q.p[0] = p.center.x; q.p[1] = p.center.y; q.p[2] = p.center.z;
      q.p[3] = p.half.x; q.p[4] = p.half.y; q.p[5] = p.half.z;
    } else if constexpr (std::is_same_v<T, Disk>) {
      q.type = XB_PRIM_DISK;
      q.p[0] = p.center.x; q.p[1] = p.center.y; q.p[2] = p.center.z;
      q.p[3] = p.normal.x; q.p[4] = p.normal.y; q.p[5] = p.normal.z; q.p[6] = p.radius;
    } else {
      q.type = XB_PRIM_QUAD;
      q.p[0] = p.origin.x; q.p[1] = p.origin.y; q.p[2] = p.origin.z;
      q.p[3] = p.u_vec.x; q.p[4] = p.u_vec.y; q.p[5] = p.u_vec.z;
      q.p[6] = p.v_vec.x; q.p[7] = p.v_vec.y; q.p[8] = p.v_vec.z;
    }
  }, v);
  return q;
}

void mat4x3_to_pod(const Mat4x3& m, float out[12]) {
  for (int c = 0; c < 4; ++c) {
    out[c * 3 + 0] = m.cols[c].x; out[c * 3 + 1] = m.cols[c].y; out[c * 3 + 2] = m.cols[c].z;
  }
}

void fill_hit(const HitRecord& rec, bool hit, xb_hit* h) {
  if (!hit) {
    std::memset(h, 0, sizeof(*h));
    h->t = std::numeric_limits<float>::infinity();
    h->prim_id = -1; h->instance_id = -1; h->mat_id = -1;
    return;
  }
  h->t = rec.t; h->u = rec.u; h->v = rec.v;
  h->prim_id = rec.prim_id; h->instance_id = rec.instance_id; h->mat_id = rec.mat_id;
  h->front_face = rec.front_face ? 1 : 0;
  h->pos[0] = rec.pos.x; h->pos[1] = rec.pos.y; h->pos[2] = rec.pos.z;
  h->normal[0] = rec.normal.x; h->normal[1] = rec.normal.y; h->normal[2] = rec.normal.z;
  h->geo_normal[0] = rec.geo_normal.x; h->geo_normal[1] = rec.geo_normal.y;
  h->geo_normal[2] = rec.geo_normal.z;
}

struct RefRenderer {
  std::unique_ptr<WavefrontRenderer> r;
  std::unique_ptr<TripleSwapchain> sc;
  int w = 0, h = 0;
};

template <class F>
void parallel_rows(int64_t n, F&& fn) {
  unsigned nt = std::max(1u, std::thread::hardware_concurrency());
  std::vector<std::thread> th;
  std::atomic<int64_t> next{0};
  const int64_t chunk = 4096;
  for (unsigned t = 0; t < nt; ++t)
    th.emplace_back([&]() {
      for (;;) {
        int64_t b = next.fetch_add(chunk);
        if (b >= n) break;
        int64_t e = std::min(n, b + chunk);
        for (int64_t i = b; i < e; ++i) fn(i);
      }
    });
  for (auto& t : th) t.join();
}

}  // namespace

extern "C" {

void* xr_scene_new() { return new RefScene(); }
void xr_scene_free(void* s) { delete static_cast<RefScene*>(s); }

int xr_scene_add_material(void* sp, const xb_material* m) {
  auto* s = static_cast<RefScene*>(sp);
  s->scene.materials.push_back(to_material(*m));
  s->mats_pod.push_back(*m);
  return (int)s->scene.materials.size() - 1;
}

// normals: NULL → the reference's own TriangleMesh::compute_smooth_normals (mesh.cpp:13)
int xr_scene_add_mesh(void* sp, int nv, const float* pos, const float* nrm, int nt,
                      const int* idx, const int* mat_ids, int default_mat) {
  auto* s = static_cast<RefScene*>(sp);
  TriangleMesh m;
  m.mat_id = default_mat;
  for (int i = 0; i < nv; ++i) m.add_vertex(Vec3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]));
  for (int t = 0; t < nt; ++t)
    m.add_triangle(idx[3 * t], idx[3 * t + 1], idx[3 * t + 2], mat_ids ? mat_ids[t] : -1);
  if (nrm) {
    for (int i = 0; i < nv; ++i) {
      m.nx[i] = nrm[3 * i]; m.ny[i] = nrm[3 * i + 1]; m.nz[i] = nrm[3 * i + 2];
    }
  } else {
    m.compute_smooth_normals();
  }
  s->scene.meshes.push_back(std::move(m));
  return (int)s->scene.meshes.size() - 1;
}

int xr_scene_transform_mesh(void* sp, int mesh, const float* pos, float scale, const float* rot) {
  auto* s = static_cast<RefScene*>(sp);
  s->scene.meshes[mesh].transform(Vec3(pos[0], pos[1], pos[2]), scale, Vec3(rot[0], rot[1], rot[2]));
  return 0;
}

// Copy of the mesh's vertex/normal arrays (to check transform/smooth-normal parity).
int xr_scene_mesh_arrays(void* sp, int mesh, float* pos, float* nrm) {
  auto* s = static_cast<RefScene*>(sp);
  const TriangleMesh& m = s->scene.meshes[mesh];
  for (int i = 0; i < m.num_vertices(); ++i) {
    pos[3 * i] = m.vx[i]; pos[3 * i + 1] = m.vy[i]; pos[3 * i + 2] = m.vz[i];
    if (nrm) { nrm[3 * i] = m.nx[i]; nrm[3 * i + 1] = m.ny[i]; nrm[3 * i + 2] = m.nz[i]; }
  }
  return m.num_vertices();
}

int xr_scene_add_prim(void* sp, const xb_prim* q) {
  auto* s = static_cast<RefScene*>(sp);
  const float* p = q->p;
  switch (q->type) {
    case XB_PRIM_SPHERE: { Sphere v; v.center = Vec3(p[0], p[1], p[2]); v.radius = p[3]; v.mat_id = q->mat_id; s->scene.all_prims.add(v); break; }
    case XB_PRIM_PLANE:  { Plane v; v.normal = Vec3(p[0], p[1], p[2]); v.offset = p[3]; v.mat_id = q->mat_id; s->scene.all_prims.add(v); break; }
    case XB_PRIM_BOX:    { Box v; v.center = Vec3(p[0], p[1], p[2]); v.half = Vec3(p[3], p[4], p[5]); v.mat_id = q->mat_id; s->scene.all_prims.add(v); break; }
    case XB_PRIM_DISK:   { Disk v; v.center = Vec3(p[0], p[1], p[2]); v.normal = Vec3(p[3], p[4], p[5]); v.radius = p[6]; v.mat_id = q->mat_id; s->scene.all_prims.add(v); break; }
    case XB_PRIM_QUAD:   { Quad v; v.origin = Vec3(p[0], p[1], p[2]); v.u_vec = Vec3(p[3], p[4], p[5]); v.v_vec = Vec3(p[6], p[7], p[8]); v.mat_id = q->mat_id; s->scene.all_prims.add(v); break; }
    default: return -1;
  }
  return s->scene.all_prims.size() - 1;
}

int xr_scene_add_light(void* sp, unsigned mesh_id, unsigned tri, const float* e, float area) {
  auto* s = static_cast<RefScene*>(sp);
  Light l{};
  l.mesh_id = mesh_id; l.tri_idx = tri; l.emission = Vec3(e[0], e[1], e[2]); l.area = area;
  s->scene.lights.push_back(l);
  return (int)s->scene.lights.size() - 1;
}

// Same normalisation as the `sunlight` line of the .xenon loader (scene_file.cpp:127-134).
int xr_scene_add_sun(void* sp, const float* d, const float* c, float intensity) {
  auto* s = static_cast<RefScene*>(sp);
  DirectionalLight dl;
  dl.direction = Vec3(d[0], d[1], d[2]);
  dl.color = Vec3(c[0], c[1], c[2]);
  dl.intensity = intensity;
  float len = dl.direction.length();
  if (len > 1e-6f) dl.direction = dl.direction / len;
  else dl.direction = Vec3(0.f, 1.f, 0.f);
  s->scene.dir_lights.push_back(dl);
  return (int)s->scene.dir_lights.size() - 1;
}

void xr_scene_set_sky(void* sp, const xb_sky* k) {
  auto* s = static_cast<RefScene*>(sp);
  s->scene.sky.zenith_color = Vec3(k->zenith[0], k->zenith[1], k->zenith[2]);
  s->scene.sky.horizon_color = Vec3(k->horizon[0], k->horizon[1], k->horizon[2]);
  s->scene.sky.ground_color = Vec3(k->ground[0], k->ground[1], k->ground[2]);
  s->scene.sky.horizon_sharpness = k->sharpness;
  s->scene.sky.intensity = k->intensity;
}

int xr_scene_add_instance(void* sp, int geom, const float* t, float scale, const float* rot, int id) {
  auto* s = static_cast<RefScene*>(sp);
  s->pending.push_back({geom, Vec3(t[0], t[1], t[2]), scale, Vec3(rot[0], rot[1], rot[2]), id});
  return (int)s->pending.size() - 1;
}

int xr_scene_build(void* sp) {
  auto* s = static_cast<RefScene*>(sp);
  Scene& sc = s->scene;
  if (s->pending.empty()) {
    sc.build_acceleration();
  } else {
    // Same BLAS / PrimBLAS builds as Scene::build_acceleration, then a TLAS over the
    // explicit instances (the reference has no .xenon instancing command).
    sc.blas_list.clear();
    for (auto& m : sc.meshes) {
      auto b = std::make_unique<BLAS>();
      b->build(m);
      sc.blas_list.push_back(std::move(b));
    }
    if (!sc.all_prims.empty()) {
      sc.prim_blas = std::make_unique<PrimBLAS>();
      sc.prim_blas->build(sc.all_prims);
    }
    std::vector<Instance> insts;
    for (auto& p : s->pending) {
      Instance inst;
      if (p.geom >= 0) inst.geom = GeomHandle::from_mesh(sc.blas_list[p.geom].get());
      else inst.geom = GeomHandle::from_prim(sc.prim_blas.get());
      inst.xform = AffineTransform::from_trs(p.t, p.s, p.rot);
      inst.instance_id = p.id;
      inst.rebuild_world_aabb();
      insts.push_back(std::move(inst));
    }
    sc.tlas.build(std::move(insts));
  }
  s->built = true;
  return 0;
}

// Load a .xenon file with the reference loader. cfg: w, h, spp. cam: eye[3], target[3], fov.
int xr_scene_load_xenon(const char* path, void** out, int* cfg, float* cam_out) {
  auto* s = new RefScene();
  Camera cam;
  SceneConfig conf;
  // The loader does not expose eye/target; re-read the camera line for the caller.
  if (!load_scene(path, s->scene, cam, conf)) { delete s; return -1; }
  s->built = true;
  for (auto& m : s->scene.materials) {
    xb_material p{};
    p.base_color[0] = m.baseColor.x; p.base_color[1] = m.baseColor.y; p.base_color[2] = m.baseColor.z;
    p.roughness = m.roughness; p.metallic = m.metallic; p.ior = m.ior; p.transmission = m.transmission;
    p.subsurface = m.subsurface;
    p.subsurface_color[0] = m.subsurfaceColor.x; p.subsurface_color[1] = m.subsurfaceColor.y;
    p.subsurface_color[2] = m.subsurfaceColor.z;
    p.anisotropy = m.anisotropy;
    p.emission[0] = m.emission.x; p.emission[1] = m.emission.y; p.emission[2] = m.emission.z;
    p.subsurface_mfp[0] = m.subsurfaceMFP.x; p.subsurface_mfp[1] = m.subsurfaceMFP.y;
    p.subsurface_mfp[2] = m.subsurfaceMFP.z;
    p.clearcoat = m.clearcoat; p.clearcoat_roughness = m.clearcoatRoughness;
    p.emission_temperature = m.emissionTemperature;
    s->mats_pod.push_back(p);
  }
  cfg[0] = conf.width; cfg[1] = conf.height; cfg[2] = conf.samples;
  Vec3 e = cam.get_eye(), ll = cam.get_lower_left_corner(), hz = cam.get_horizontal(), vt = cam.get_vertical();
  float v[12] = {e.x, e.y, e.z, ll.x, ll.y, ll.z, hz.x, hz.y, hz.z, vt.x, vt.y, vt.z};
  std::memcpy(cam_out, v, sizeof(v));
  *out = s;
  return 0;
}

// Derived material values (material_prepare) for parity of the host restatement.
void xr_material_prepare(const xb_material* p, xb_material_derived* out) {
  Material m = to_material(*p);
  out->alpha = m.alpha; out->alpha_x = m.alpha_x; out->alpha_y = m.alpha_y;
  out->f0[0] = m.F0.x; out->f0[1] = m.F0.y; out->f0[2] = m.F0.z;
  out->flags = (m.isConductor ? XB_MAT_CONDUCTOR : 0) | (m.isTransmissive ? XB_MAT_TRANSMISSIVE : 0) |
               (m.hasSubsurface ? XB_MAT_SUBSURFACE : 0) | (m.isDelta ? XB_MAT_DELTA : 0) |
               (m.isEmissive ? XB_MAT_EMISSIVE : 0);
}

int xr_material_load(const char* path, xb_material* p, char* name, int name_len) {
  Material m = load_material(path);
  p->base_color[0] = m.baseColor.x; p->base_color[1] = m.baseColor.y; p->base_color[2] = m.baseColor.z;
  p->roughness = m.roughness; p->metallic = m.metallic; p->ior = m.ior; p->transmission = m.transmission;
  p->subsurface = m.subsurface;
  p->subsurface_color[0] = m.subsurfaceColor.x; p->subsurface_color[1] = m.subsurfaceColor.y;
  p->subsurface_color[2] = m.subsurfaceColor.z;
  p->anisotropy = m.anisotropy;
  p->emission[0] = m.emission.x; p->emission[1] = m.emission.y; p->emission[2] = m.emission.z;
  p->subsurface_mfp[0] = m.subsurfaceMFP.x; p->subsurface_mfp[1] = m.subsurfaceMFP.y;
  p->subsurface_mfp[2] = m.subsurfaceMFP.z;
  p->clearcoat = m.clearcoat; p->clearcoat_roughness = m.clearcoatRoughness;
  p->emission_temperature = m.emissionTemperature;
  std::snprintf(name, (size_t)name_len, "%s", m.name.c_str());
  return 0;
}

// Export the reference-built scene (its own BVH arrays) as an xb_scene_view.
int xr_scene_view(void* sp, xb_scene_view* v) {
  auto* s = static_cast<RefScene*>(sp);
  if (!s->built) return -1;
  Scene& sc = s->scene;
  std::memset(v, 0, sizeof(*v));
  s->mesh_views.clear();
  for (size_t i = 0; i < sc.meshes.size(); ++i) {
    const TriangleMesh& m = sc.meshes[i];
    xb_mesh_view mv{};
    mv.num_vertices = m.num_vertices();
    mv.num_triangles = m.num_triangles();
    mv.vx = m.vx.data(); mv.vy = m.vy.data(); mv.vz = m.vz.data();
    if (!m.nx.empty()) { mv.nx = m.nx.data(); mv.ny = m.ny.data(); mv.nz = m.nz.data(); }
    mv.indices = m.indices.data();
    mv.mat_ids = m.mat_ids.data();
    const BLAS& b = *sc.blas_list[i];
    mv.blas_nodes = reinterpret_cast<const xb_bvh_node*>(b.nodes().data());
    mv.num_blas_nodes = (int)b.nodes().size();
    mv.blas_prims = b.prims().data();
    s->mesh_views.push_back(mv);
  }
  v->num_meshes = (int)s->mesh_views.size();
  v->meshes = s->mesh_views.data();

  s->prims_pod.clear();
  for (auto& p : sc.all_prims.prims) s->prims_pod.push_back(prim_to_pod(p));
  v->num_prims = (int)s->prims_pod.size();
  v->prims = s->prims_pod.data();
  if (sc.prim_blas) {
    v->prim_nodes = reinterpret_cast<const xb_bvh_node*>(sc.prim_blas->nodes_.data());
    v->num_prim_nodes = (int)sc.prim_blas->nodes_.size();
    v->prim_indices = sc.prim_blas->prims_.data();
  }

  s->inst_views.clear();
  for (const Instance& inst : sc.tlas.instances()) {
    xb_instance_view iv{};
    iv.instance_id = inst.instance_id;
    if (inst.geom.type == GeomHandle::PRIM_BLAS) {
      iv.geom = XB_GEOM_PRIMS;
    } else {
      iv.geom = -2;
      for (size_t k = 0; k < sc.blas_list.size(); ++k)
        if (sc.blas_list[k].get() == inst.geom.mesh) iv.geom = (int)k;
    }
    mat4x3_to_pod(inst.xform.local_to_world, iv.local_to_world);
    mat4x3_to_pod(inst.xform.world_to_local, iv.world_to_local);
    s->inst_views.push_back(iv);
  }
  v->num_instances = (int)s->inst_views.size();
  v->instances = s->inst_views.data();
  v->tlas_nodes = reinterpret_cast<const xb_bvh_node*>(sc.tlas.nodes().data());
  v->num_tlas_nodes = (int)sc.tlas.nodes().size();
  v->tlas_inst_indices = sc.tlas.inst_indices().data();

  v->num_materials = (int)s->mats_pod.size();
  v->materials = s->mats_pod.data();
  s->lights_pod.clear();
  for (auto& l : sc.lights) {
    xb_light q{};
    q.mesh_id = l.mesh_id; q.tri_idx = l.tri_idx;
    q.emission[0] = l.emission.x; q.emission[1] = l.emission.y; q.emission[2] = l.emission.z;
    q.area = l.area;
    s->lights_pod.push_back(q);
  }
  v->num_lights = (int)s->lights_pod.size();
  v->lights = s->lights_pod.data();
  s->suns_pod.clear();
  for (auto& d : sc.dir_lights) {
    xb_sun q{};
    q.direction[0] = d.direction.x; q.direction[1] = d.direction.y; q.direction[2] = d.direction.z;
    q.color[0] = d.color.x; q.color[1] = d.color.y; q.color[2] = d.color.z;
    q.intensity = d.intensity;
    s->suns_pod.push_back(q);
  }
  v->num_suns = (int)s->suns_pod.size();
  v->suns = s->suns_pod.data();
  const Environment& e = sc.sky;
  v->sky.zenith[0] = e.zenith_color.x; v->sky.zenith[1] = e.zenith_color.y; v->sky.zenith[2] = e.zenith_color.z;
  v->sky.horizon[0] = e.horizon_color.x; v->sky.horizon[1] = e.horizon_color.y; v->sky.horizon[2] = e.horizon_color.z;
  v->sky.ground[0] = e.ground_color.x; v->sky.ground[1] = e.ground_color.y; v->sky.ground[2] = e.ground_color.z;
  v->sky.sharpness = e.horizon_sharpness;
  v->sky.intensity = e.intensity;
  return 0;
}

// Scene::intersect (mode 0) or Scene::intersects (mode 1) over a ray batch.
int xr_trace(void* sp, int64_t n, const xb_ray* rays, xb_hit* hits, int mode) {
  auto* s = static_cast<RefScene*>(sp);
  parallel_rows(n, [&](int64_t i) {
    Ray r;
    r.origin = Vec3(rays[i].org[0], rays[i].org[1], rays[i].org[2]);
    r.dir = Vec3(rays[i].dir[0], rays[i].dir[1], rays[i].dir[2]);
    r.tmin = rays[i].tmin;
    r.tmax = rays[i].tmax;
    if (mode == 0) {
      HitRecord rec;
      bool hit = s->scene.intersect(r, rec);
      fill_hit(rec, hit, &hits[i]);
    } else {
      bool occ = s->scene.intersects(r);
      HitRecord rec;
      fill_hit(rec, false, &hits[i]);
      if (occ) hits[i].t = 0.f;
    }
  });
  return 0;
}

void xr_bsdf_eval(const xb_material* mp, int64_t n, const float* wo, const float* wi,
                  float* f, float* pdf) {
  Material m = to_material(*mp);
  for (int64_t i = 0; i < n; ++i) {
    Vec3 o(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]);
    Vec3 w(wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]);
    Vec3 fv = bsdf_eval_for_nee(o, w, m);
    f[3 * i] = fv.x; f[3 * i + 1] = fv.y; f[3 * i + 2] = fv.z;
    pdf[i] = bsdf_pdf_for_nee(o, w, m);
  }
}

void xr_bsdf_sample(const xb_material* mp, int64_t n, const float* wo, uint64_t* state,
                    float* wi, float* f, float* pdf, int* flags) {
  Material m = to_material(*mp);
  for (int64_t i = 0; i < n; ++i) {
    PCGState rng{state[i], 1};
    Vec3 o(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]);
    BSDFSample smp;
    bool ok = bsdf_sample(o, m, rng, smp);
    state[i] = rng.state;
    wi[3 * i] = smp.wi.x; wi[3 * i + 1] = smp.wi.y; wi[3 * i + 2] = smp.wi.z;
    f[3 * i] = smp.f.x; f[3 * i + 1] = smp.f.y; f[3 * i + 2] = smp.f.z;
    pdf[i] = smp.pdf;
    flags[i] = (ok ? 1 : 0) | (smp.is_delta ? 2 : 0);
  }
}

// PCG seeding of the CPU backend (seed_pcg, src/camera/sampler.h:29-35): state after seeding.
uint64_t xr_seed_pcg(uint64_t seed) { return seed_pcg(seed).state; }

// Camera::look_at with up = (0,1,0) (scene_file.cpp:224). out: eye, lower_left, horizontal, vertical.
void xr_camera(const float* eye, const float* target, float fov, float aspect, float* out) {
  Camera c;
  c.look_at(Vec3(eye[0], eye[1], eye[2]), Vec3(target[0], target[1], target[2]), Vec3(0, 1, 0), fov, aspect);
  Vec3 e = c.get_eye(), ll = c.get_lower_left_corner(), hz = c.get_horizontal(), vt = c.get_vertical();
  float v[12] = {e.x, e.y, e.z, ll.x, ll.y, ll.z, hz.x, hz.y, hz.z, vt.x, vt.y, vt.z};
  std::memcpy(out, v, sizeof(v));
}

void* xr_renderer_new(int w, int h, int min_b, int max_b) {
  auto* r = new RefRenderer();
  r->r = std::make_unique<WavefrontRenderer>(w, h);
  r->r->set_bounces(min_b, max_b);
  r->sc = std::make_unique<TripleSwapchain>(w, h);
  r->w = w; r->h = h;
  return r;
}
void xr_renderer_free(void* r) { delete static_cast<RefRenderer*>(r); }

// Render samples [spp_first, spp_first + spp_count) (1-based, the value spp_ takes inside
// render_frame_tiled) one at a time; sum_rgb (double[W*H*3], top-down rows like the CPU
// output) receives the FP64 sum of the per-sample radiance. Returns wall seconds spent in
// render_frame_tiled. `eye_target_fov` = eye[3], target[3], fov.
double xr_render(void* rp, void* sp, const float* eye_target_fov, int spp_first, int spp_count,
                 double* sum_rgb) {
  auto* r = static_cast<RefRenderer*>(rp);
  auto* s = static_cast<RefScene*>(sp);
  Camera cam;
  cam.look_at(Vec3(eye_target_fov[0], eye_target_fov[1], eye_target_fov[2]),
              Vec3(eye_target_fov[3], eye_target_fov[4], eye_target_fov[5]), Vec3(0, 1, 0),
              eye_target_fov[6], (float)r->w / (float)r->h);
  const int W = r->w, H = r->h;
  double secs = 0.0;
  for (int k = 0; k < spp_count; ++k) {
    std::fill(r->r->accumulation_buffer_.begin(), r->r->accumulation_buffer_.end(), Vec3(0.f));
    r->r->spp_ = spp_first + k - 1;               // render_frame_tiled increments first
    auto t0 = std::chrono::steady_clock::now();
    r->r->render_frame_tiled(s->scene, cam, *r->sc);
    auto t1 = std::chrono::steady_clock::now();
    secs += std::chrono::duration<double>(t1 - t0).count();
    if (sum_rgb) {
      for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
          const Vec3& c = r->r->accumulation_buffer_[(size_t)y * W + x];
          size_t d = ((size_t)(H - 1 - y) * W + x) * 3;
          sum_rgb[d] += c.x; sum_rgb[d + 1] += c.y; sum_rgb[d + 2] += c.z;
        }
    }
  }
  return secs;
}

int xr_hardware_threads() { return (int)std::thread::hardware_concurrency(); }

// The reference's output stage (src/main.cpp:24-52). Noise statistics: its own
// ImageNoiseEstimator (src/math/image.h:35-118) on an RGB float image; out receives the ten
// float fields of NoiseStats (meanSquaredScore, rmsScore, meanAbsolute, medianAbsolute,
// p95Absolute, maxAbsolute, avgLuminance, edgeThreshold, epsilon, validPixelRatio), counts the
// valid and interior pixel counts.
void xr_noise_stats(const float* rgb, int w, int h, float* out, int* counts) {
  const xn::NoiseStats s = xn::ImageNoiseEstimator::computeResidualNoiseStats(rgb, w, h);
  const float f[10] = {s.meanSquaredScore, s.rmsScore, s.meanAbsolute, s.medianAbsolute, s.p95Absolute,
                       s.maxAbsolute, s.avgLuminance, s.edgeThreshold, s.epsilon, s.validPixelRatio};
  for (int i = 0; i < 10; ++i) out[i] = f[i];
  counts[0] = s.validPixelCount;
  counts[1] = s.totalInteriorPixelCount;
}

// save_image's 8-bit values (src/main.cpp:27-30 lives in main(), so it is restated here): each
// channel clamped to [0, 1], raised to 1/2.2, times 255.99, truncated; n values, no flip.
void xr_image_rgb8(const float* rgb, int64_t n, uint8_t* out) {
  for (int64_t i = 0; i < n; ++i) out[i] = (uint8_t)(255.99f * std::pow(std::clamp(rgb[i], 0.f, 1.f), 1.f / 2.2f));
}

}  // extern "C"
