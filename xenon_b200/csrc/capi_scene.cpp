// capi_scene.cpp — C ABI of the host scene (xb_scene_*, xb_material_*, xb_camera_look_at).

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <stdexcept>
#include <string>

#include "capi_common.h"
#include "scene_host.h"

struct xb_scene {
  xb::HostScene s;
};

namespace xb {
thread_local std::string g_last_error;

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}
}  // namespace xb

using namespace xb;

extern "C" {

void xb_material_default(xb_material* m) {
  if (m) default_material(m);
}

int xb_material_prepare(const xb_material* m, xb_material_derived* out) {
  if (!m || !out) return fail(XB_E_INVALID, "xb_material_prepare: null argument");
  *out = prepare_material(*m);
  return XB_OK;
}

int xb_material_load(const char* path, xb_material* out, char* name, size_t name_len) {
  if (!path || !out) return fail(XB_E_INVALID, "xb_material_load: null argument");
  std::string n;
  if (!load_mat_file(path, out, &n)) return fail(XB_E_IO, "cannot open material file %s", path);
  if (name && name_len) std::snprintf(name, name_len, "%s", n.c_str());
  return XB_OK;
}

// Camera::look_at (src/camera/camera.h:15-31)
int xb_camera_look_at(const float eye[3], const float target[3], const float up[3], float fov,
                      float aspect, xb_camera* out) {
  if (!eye || !target || !out) return fail(XB_E_INVALID, "xb_camera_look_at: null argument");
  F3 e(eye[0], eye[1], eye[2]), t(target[0], target[1], target[2]);
  F3 u0 = up ? F3(up[0], up[1], up[2]) : F3(0.f, 1.f, 0.f);
  const float theta = fov * kPiF / 180.f;
  const float h = std::tan(theta / 2.f);
  const float vh = 2.f * h;
  const float vw = aspect * vh;
  F3 w = normalize3(e - t);
  F3 u = normalize3(cross3(u0, w));
  F3 v = cross3(w, u);
  F3 hor = vw * u, ver = vh * v;
  F3 ll = e - hor * 0.5f - ver * 0.5f - w;
  const F3 vals[4] = {e, ll, hor, ver};
  float* dst[4] = {out->eye, out->lower_left, out->horizontal, out->vertical};
  for (int i = 0; i < 4; ++i) { dst[i][0] = vals[i].x; dst[i][1] = vals[i].y; dst[i][2] = vals[i].z; }
  return XB_OK;
}

int xb_scene_create(xb_scene** out) {
  if (!out) return fail(XB_E_INVALID, "xb_scene_create: null argument");
  *out = new (std::nothrow) xb_scene();
  return *out ? XB_OK : fail(XB_E_OOM, "xb_scene_create: out of memory");
}

void xb_scene_destroy(xb_scene* s) { delete s; }

#define SCENE_CHECK(s)                                                          \
  do {                                                                          \
    if (!(s)) return fail(XB_E_INVALID, "%s: null scene", __func__);            \
  } while (0)
#define SCENE_MUTABLE(s)                                                        \
  do {                                                                          \
    SCENE_CHECK(s);                                                             \
    (s)->s.built = false;                                                       \
  } while (0)

int xb_scene_add_material(xb_scene* s, const char* name, const xb_material* m) {
  SCENE_MUTABLE(s);
  if (!m) return fail(XB_E_INVALID, "xb_scene_add_material: null material");
  s->s.materials.push_back(*m);
  s->s.material_names.push_back(name ? name : "default");
  return (int)s->s.materials.size() - 1;
}

int xb_scene_add_mesh(xb_scene* s, int32_t nv, const float* positions, const float* normals,
                      int32_t nt, const int32_t* indices, const int32_t* mat_ids, int32_t default_mat) {
  SCENE_MUTABLE(s);
  if (nv < 0 || nt < 0 || (nv && !positions) || (nt && !indices))
    return fail(XB_E_INVALID, "xb_scene_add_mesh: bad sizes or null arrays");
  HostMesh m;
  m.default_mat = default_mat;
  m.vx.resize(nv); m.vy.resize(nv); m.vz.resize(nv);
  for (int32_t i = 0; i < nv; ++i) {
    m.vx[i] = positions[3 * i]; m.vy[i] = positions[3 * i + 1]; m.vz[i] = positions[3 * i + 2];
  }
  m.indices.assign(indices, indices + 3 * (size_t)nt);
  for (int32_t i = 0; i < 3 * nt; ++i)
    if (m.indices[i] < 0 || m.indices[i] >= nv)
      return fail(XB_E_INVALID, "xb_scene_add_mesh: index %d out of range", m.indices[i]);
  m.mat_ids.resize(nt);
  for (int32_t t = 0; t < nt; ++t) m.mat_ids[t] = (mat_ids && mat_ids[t] >= 0) ? mat_ids[t] : default_mat;
  if (normals) {
    m.nx.resize(nv); m.ny.resize(nv); m.nz.resize(nv);
    for (int32_t i = 0; i < nv; ++i) {
      m.nx[i] = normals[3 * i]; m.ny[i] = normals[3 * i + 1]; m.nz[i] = normals[3 * i + 2];
    }
  } else {
    m.compute_smooth_normals();
  }
  s->s.meshes.push_back(std::move(m));
  return (int)s->s.meshes.size() - 1;
}

int xb_scene_transform_mesh(xb_scene* s, int32_t mesh, const float pos[3], float scale,
                            const float rot[3]) {
  SCENE_MUTABLE(s);
  if (mesh < 0 || mesh >= (int)s->s.meshes.size() || !pos || !rot)
    return fail(XB_E_INVALID, "xb_scene_transform_mesh: bad mesh %d", mesh);
  s->s.meshes[mesh].transform(F3(pos[0], pos[1], pos[2]), scale, F3(rot[0], rot[1], rot[2]));
  return XB_OK;
}

int xb_scene_add_prim(xb_scene* s, const xb_prim* p) {
  SCENE_MUTABLE(s);
  if (!p || p->type < XB_PRIM_SPHERE || p->type > XB_PRIM_QUAD)
    return fail(XB_E_INVALID, "xb_scene_add_prim: bad prim");
  s->s.prims.push_back(*p);
  return (int)s->s.prims.size() - 1;
}

int xb_scene_add_light(xb_scene* s, uint32_t mesh_id, uint32_t tri, const float e[3], float area) {
  SCENE_MUTABLE(s);
  if (!e) return fail(XB_E_INVALID, "xb_scene_add_light: null emission");
  s->s.lights.push_back(xb_light{mesh_id, tri, {e[0], e[1], e[2]}, area});
  return (int)s->s.lights.size() - 1;
}

// direction normalised as the `sunlight` line does (src/scene/scene_file.cpp:127-134)
int xb_scene_add_sun(xb_scene* s, const float d[3], const float c[3], float intensity) {
  SCENE_MUTABLE(s);
  if (!d || !c) return fail(XB_E_INVALID, "xb_scene_add_sun: null argument");
  F3 dir(d[0], d[1], d[2]);
  float len = len3(dir);
  dir = len > 1e-6f ? div_scalar(dir, len) : F3(0.f, 1.f, 0.f);
  s->s.suns.push_back(xb_sun{{dir.x, dir.y, dir.z}, {c[0], c[1], c[2]}, intensity});
  return (int)s->s.suns.size() - 1;
}

int xb_scene_set_sky(xb_scene* s, const xb_sky* k) {
  SCENE_MUTABLE(s);
  if (!k) return fail(XB_E_INVALID, "xb_scene_set_sky: null sky");
  s->s.sky = *k;
  return XB_OK;
}

int xb_scene_add_instance(xb_scene* s, int32_t geom, const float t[3], float scale,
                          const float rot[3], int32_t instance_id) {
  SCENE_MUTABLE(s);
  if (!t || !rot || scale == 0.f) return fail(XB_E_INVALID, "xb_scene_add_instance: bad transform");
  if (geom != XB_GEOM_PRIMS && (geom < 0 || geom >= (int)s->s.meshes.size()))
    return fail(XB_E_INVALID, "xb_scene_add_instance: bad geometry %d", geom);
  HostInstance in;
  in.geom = geom;
  in.instance_id = instance_id;
  in.l2w = affine_from_trs(F3(t[0], t[1], t[2]), scale, F3(rot[0], rot[1], rot[2]), &in.w2l);
  s->s.explicit_instances.push_back(in);
  return (int)s->s.explicit_instances.size() - 1;
}

int xb_scene_set_build_threads(xb_scene* s, int32_t threads) {
  SCENE_MUTABLE(s);
  if (threads < 0) return fail(XB_E_INVALID, "xb_scene_set_build_threads: %d threads", threads);
  s->s.build_threads = threads;
  return XB_OK;
}

int xb_scene_set_build_mode(xb_scene* s, int32_t mode) {
  SCENE_MUTABLE(s);
  if (mode != XB_BUILD_RECURSIVE && mode != XB_BUILD_LEVELS && mode != XB_BUILD_DEVICE)
    return fail(XB_E_INVALID, "xb_scene_set_build_mode: unknown mode %d", mode);
  s->s.build_mode = mode;
  return XB_OK;
}

int xb_scene_build(xb_scene* s) {
  SCENE_CHECK(s);
  for (const auto& l : s->s.lights)
    if (l.mesh_id >= s->s.meshes.size() || (int)l.tri_idx >= s->s.meshes[l.mesh_id].num_triangles())
      return fail(XB_E_INVALID, "light refers to mesh %u triangle %u which does not exist", l.mesh_id, l.tri_idx);
  try {
    s->s.build();
  } catch (const std::bad_alloc&) {
    return fail(XB_E_OOM, "xb_scene_build: out of host memory");
  } catch (const std::invalid_argument& e) {
    return fail(XB_E_INVALID, "xb_scene_build: %s", e.what());
  } catch (const std::runtime_error& e) {   // the device build's CUDA errors
    return fail(XB_E_CUDA, "xb_scene_build: %s", e.what());
  }
  return XB_OK;
}

int xb_scene_refit_mesh(xb_scene* s, int32_t mesh, const float* positions, const float* normals) {
  SCENE_CHECK(s);
  if (!s->s.built) return fail(XB_E_STATE, "xb_scene_refit_mesh: call xb_scene_build first");
  if (mesh < 0 || mesh >= (int)s->s.meshes.size() || !positions)
    return fail(XB_E_INVALID, "xb_scene_refit_mesh: bad mesh %d or null positions", mesh);
  const int nv = s->s.meshes[mesh].num_vertices();
  for (int i = 0; i < 3 * nv; ++i)
    if (!std::isfinite(positions[i]) || (normals && !std::isfinite(normals[i])))
      return fail(XB_E_INVALID, "xb_scene_refit_mesh: non-finite value at %d", i);
  try {
    s->s.refit_mesh(mesh, positions, normals);
  } catch (const std::bad_alloc&) {
    return fail(XB_E_OOM, "xb_scene_refit_mesh: out of host memory");
  } catch (const std::exception& e) {
    return fail(XB_E_INVALID, "xb_scene_refit_mesh: %s", e.what());
  }
  return XB_OK;
}

int xb_scene_get_view(const xb_scene* s, xb_scene_view* out) {
  SCENE_CHECK(s);
  if (!out) return fail(XB_E_INVALID, "xb_scene_get_view: null output");
  if (!s->s.built) return fail(XB_E_STATE, "xb_scene_get_view: call xb_scene_build first");
  const_cast<xb_scene*>(s)->s.view(out);
  return XB_OK;
}

int xb_scene_load(const char* path, xb_scene** out, xb_scene_config* cfg, xb_camera_desc* cam) {
  if (!path || !out) return fail(XB_E_INVALID, "xb_scene_load: null argument");
  auto* s = new (std::nothrow) xb_scene();
  if (!s) return fail(XB_E_OOM, "xb_scene_load: out of memory");
  xb_scene_config c;
  xb_camera_desc d;
  std::string err;
  if (!load_xenon(path, s->s, &c, &d, &err)) {
    delete s;
    return fail(XB_E_IO, "%s", err.c_str());
  }
  if (cfg) *cfg = c;
  if (cam) *cam = d;
  *out = s;
  return XB_OK;
}

}  // extern "C"
