// loaders.cpp — the reference's scene file formats, read into a HostScene.
//
//   .mat   key/value material files        (src/material/material.cpp:31-104)
//   .obj   v / vn / f / usemtl, fan faces   (src/geometry/mesh.cpp:42-150)
//   .xenon scene description               (src/scene/scene_file.cpp:49-231), plus one
//                                           command of this library's: `instance` (below)
//
// The parser is the source of truth for the syntax (docs/MAT_FORMAT.md disagrees with it in
// places: `anisotropic` / `transmissionRoughness` are not keys the reference reads).

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <map>
#include <sstream>
#include <unordered_map>

#include "scene_host.h"

namespace xb {

namespace {

std::string unquote(const std::string& s) {
  if (s.size() >= 2 && s.front() == '"' && s.back() == '"') return s.substr(1, s.size() - 2);
  return s;
}

// A relative path is tried as given, then next to the scene file (scene_file.cpp:13-20).
std::string resolve_near(const std::string& scene_path, const std::string& rel) {
  namespace fs = std::filesystem;
  std::error_code ec;
  if (fs::exists(rel, ec)) return rel;
  fs::path p = fs::path(scene_path).parent_path() / rel;
  if (fs::exists(p, ec)) return p.string();
  return rel;
}

}  // namespace

bool load_mat_file(const std::string& path, xb_material* m, std::string* name) {
  default_material(m);
  *name = "default";
  std::ifstream f(path);
  if (!f.is_open()) return false;
  std::string line;
  while (std::getline(f, line)) {
    size_t first = line.find_first_not_of(" \t");
    if (first == std::string::npos || line[first] == '#') continue;
    std::istringstream ss(line);
    std::string key;
    ss >> key;
    if (key == "name") { std::string v; ss >> v; *name = unquote(v); }
    else if (key == "type") { std::string v; ss >> v; }
    else if (key == "baseColor") ss >> m->base_color[0] >> m->base_color[1] >> m->base_color[2];
    else if (key == "roughness") ss >> m->roughness;
    else if (key == "metallic") ss >> m->metallic;
    else if (key == "ior") ss >> m->ior;
    else if (key == "transmission") ss >> m->transmission;
    else if (key == "subsurface") ss >> m->subsurface;
    else if (key == "subsurfaceColor") ss >> m->subsurface_color[0] >> m->subsurface_color[1] >> m->subsurface_color[2];
    else if (key == "subsurfaceMFP") ss >> m->subsurface_mfp[0] >> m->subsurface_mfp[1] >> m->subsurface_mfp[2];
    else if (key == "clearcoat") ss >> m->clearcoat;
    else if (key == "clearcoatRoughness") ss >> m->clearcoat_roughness;
    else if (key == "anisotropy") ss >> m->anisotropy;
    else if (key == "emission") ss >> m->emission[0] >> m->emission[1] >> m->emission[2];
    else if (key == "emissionTemperature") ss >> m->emission_temperature;
    else std::fprintf(stderr, "[xenon_b200] %s: unknown material key '%s'\n", path.c_str(), key.c_str());
  }
  return true;
}

bool load_obj(const std::string& path, HostMesh& mesh, const std::vector<std::string>& mat_names,
              int default_mat, std::string* err) {
  std::ifstream f(path);
  if (!f.is_open()) { *err = "cannot open mesh " + path; return false; }
  std::vector<F3> pos, nrm;
  std::unordered_map<int64_t, int32_t> cache;
  bool has_normals = false;
  int cur_mat = default_mat;
  mesh.default_mat = default_mat;
  auto vert = [&](int pi, int ni) -> int32_t {
    const int64_t key = ((int64_t)pi << 32) | (uint32_t)ni;
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    const int32_t id = (int32_t)mesh.vx.size();
    const F3 p = pos[pi];
    mesh.vx.push_back(p.x); mesh.vy.push_back(p.y); mesh.vz.push_back(p.z);
    if (ni >= 0 && ni < (int)nrm.size()) {
      mesh.nx.push_back(nrm[ni].x); mesh.ny.push_back(nrm[ni].y); mesh.nz.push_back(nrm[ni].z);
    } else {
      mesh.nx.push_back(0.f); mesh.ny.push_back(0.f); mesh.nz.push_back(0.f);
    }
    cache[key] = id;
    return id;
  };
  std::string line;
  while (std::getline(f, line)) {
    if (line.empty() || line[0] == '#') continue;
    char type[8] = {};
    if (std::sscanf(line.c_str(), "%7s", type) < 1) continue;
    const char* p = line.c_str() + std::strlen(type);
    if (!std::strcmp(type, "v")) {
      float x, y, z;
      if (std::sscanf(p, " %f %f %f", &x, &y, &z) == 3) pos.push_back(F3(x, y, z));
    } else if (!std::strcmp(type, "vn")) {
      float x, y, z;
      if (std::sscanf(p, " %f %f %f", &x, &y, &z) == 3) { nrm.push_back(normalize3(F3(x, y, z))); has_normals = true; }
    } else if (!std::strcmp(type, "usemtl")) {
      char mname[128];
      if (std::sscanf(p, " %127s", mname) == 1) {
        for (size_t i = 0; i < mat_names.size(); ++i)
          if (mat_names[i] == mname) cur_mat = (int)i;   // last material of that name wins
      }
    } else if (!std::strcmp(type, "f")) {
      std::vector<int32_t> fv;
      const char* q = p;
      while (*q) {
        while (*q == ' ' || *q == '\t') ++q;
        if (!*q || *q == '\n' || *q == '\r') break;
        int pi = -1, ti = -1, ni = -1, used = 0;
        if (std::sscanf(q, "%d/%d/%d%n", &pi, &ti, &ni, &used) >= 3) {}
        else if (std::sscanf(q, "%d//%d%n", &pi, &ni, &used) >= 2) {}
        else if (std::sscanf(q, "%d/%d%n", &pi, &ti, &used) >= 2) {}
        else if (std::sscanf(q, "%d%n", &pi, &used) >= 1) {}
        else break;
        if (pi > 0) {
          --pi;
          ni = ni > 0 ? ni - 1 : -1;
          if (pi >= (int)pos.size()) { *err = "face index out of range in " + path; return false; }
          fv.push_back(vert(pi, ni));
        }
        q += used;
      }
      for (int i = 1; i + 1 < (int)fv.size(); ++i) {
        mesh.indices.push_back(fv[0]); mesh.indices.push_back(fv[i]); mesh.indices.push_back(fv[i + 1]);
        mesh.mat_ids.push_back(cur_mat);
      }
    }
  }
  if (!has_normals) mesh.compute_smooth_normals();
  return true;
}

bool load_xenon(const std::string& path, HostScene& sc, xb_scene_config* cfg, xb_camera_desc* cam,
                std::string* err) {
  std::ifstream f(path);
  if (!f.is_open()) { *err = "cannot open scene " + path; return false; }
  cfg->width = 800; cfg->height = 600; cfg->samples = 64;     // SceneConfig defaults
  cfg->min_bounces = 3; cfg->max_bounces = 8;
  F3 eye(0, 5, 20), target(0, 5, 0);
  float fov = 40.f;
  std::map<std::string, int> mat_map;
  auto mat_of = [&](const std::string& n) {
    auto it = mat_map.find(n);
    if (it == mat_map.end()) {
      std::fprintf(stderr, "[xenon_b200] unknown material '%s', using 0\n", n.c_str());
      return 0;
    }
    return it->second;
  };
  std::string line;
  while (std::getline(f, line)) {
    std::stringstream ss(line);
    std::string cmd;
    ss >> cmd;
    if (cmd.empty() || cmd[0] == '#') continue;
    if (cmd == "config") {
      ss >> cfg->width >> cfg->height >> cfg->samples;
    } else if (cmd == "camera") {
      ss >> eye.x >> eye.y >> eye.z >> target.x >> target.y >> target.z >> fov;
    } else if (cmd == "matfile") {
      std::string mp;
      ss >> mp;
      mp = "materials/" + unquote(mp);
      xb_material m;
      std::string name;
      if (!load_mat_file(resolve_near(path, mp), &m, &name))
        std::fprintf(stderr, "[xenon_b200] cannot open material %s, using defaults\n", mp.c_str());
      mat_map[name] = (int)sc.materials.size();
      sc.materials.push_back(m);
      sc.material_names.push_back(name);
    } else if (cmd == "material") {
      // material_from_legacy (src/material/material.cpp:134-152)
      std::string name;
      xb_material m;
      default_material(&m);
      ss >> name >> m.base_color[0] >> m.base_color[1] >> m.base_color[2] >> m.metallic >> m.roughness;
      float spec = 0.5f, ior = 1.5f, trans = 0.f, trans_rough = -1.f;
      ss >> spec >> ior >> trans >> trans_rough;
      m.ior = ior;
      m.transmission = trans;
      if (trans_rough >= 0.f && trans > 0.01f) m.roughness = trans_rough;
      mat_map[name] = (int)sc.materials.size();
      sc.materials.push_back(m);
      sc.material_names.push_back(name);
    } else if (cmd == "mesh") {
      std::string obj;
      ss >> obj;
      HostMesh m;
      std::string e;
      if (!load_obj(obj, m, sc.material_names, 0, &e)) {
        std::fprintf(stderr, "[xenon_b200] %s\n", e.c_str());
        continue;
      }
      F3 pos(0, 0, 0), rot(0, 0, 0);
      float scale = 1.f;
      if (ss >> pos.x >> pos.y >> pos.z >> scale >> rot.x >> rot.y >> rot.z) m.transform(pos, scale, rot);
      sc.meshes.push_back(std::move(m));
    } else if (cmd == "light") {
      xb_light l{};
      ss >> l.mesh_id >> l.tri_idx >> l.emission[0] >> l.emission[1] >> l.emission[2] >> l.area;
      sc.lights.push_back(l);
    } else if (cmd == "sunlight") {
      F3 d(0, 1, 0), c(1.0f, 0.95f, 0.8f);
      float inten = 5.f;
      ss >> d.x >> d.y >> d.z >> c.x >> c.y >> c.z >> inten;
      float len = len3(d);
      d = len > 1e-6f ? div_scalar(d, len) : F3(0.f, 1.f, 0.f);
      sc.suns.push_back(xb_sun{{d.x, d.y, d.z}, {c.x, c.y, c.z}, inten});
    } else if (cmd == "sky") {
      xb_sky& k = sc.sky;
      ss >> k.zenith[0] >> k.zenith[1] >> k.zenith[2] >> k.horizon[0] >> k.horizon[1] >> k.horizon[2];
      float g[3] = {0.1f, 0.08f, 0.05f};
      float inten = 1.f, sharp = 3.f;
      if (ss >> g[0] >> g[1] >> g[2]) {
        k.ground[0] = g[0]; k.ground[1] = g[1]; k.ground[2] = g[2];
        ss >> inten >> sharp;
        k.intensity = inten;
        k.sharpness = sharp;
      }
    } else if (cmd == "instance") {
      // Not a reference command (its parser has no instancing; a `mesh` line bakes its transform
      // into the vertices): `instance <mesh> tx ty tz scale rx ry rz [id]` places the mesh of
      // the <mesh>-th loaded `mesh` line (0-based), or the analytic primitives (`prims`), with
      // a mesh line's transform convention (rotations in degrees). Once a file has one, the
      // TLAS holds exactly the instances listed. The id defaults to the mesh's index (the
      // number of meshes for `prims`), which keeps `light` entries matching their meshes.
      std::string what;
      ss >> what;
      F3 t(0, 0, 0), rot(0, 0, 0);
      float scale = 1.f;
      if (!(ss >> t.x >> t.y >> t.z >> scale >> rot.x >> rot.y >> rot.z) || scale == 0.f) {
        std::fprintf(stderr, "[xenon_b200] instance: needs tx ty tz scale rx ry rz, scale not 0 (skipped)\n");
        continue;
      }
      HostInstance in;
      if (what == "prims") {
        in.geom = XB_GEOM_PRIMS;
        in.instance_id = (int32_t)sc.meshes.size();
      } else {
        char* end = nullptr;
        const long g = std::strtol(what.c_str(), &end, 10);
        if (what.empty() || *end != '\0' || g < 0 || g >= (long)sc.meshes.size()) {
          std::fprintf(stderr, "[xenon_b200] instance: no mesh '%s' (skipped)\n", what.c_str());
          continue;
        }
        in.geom = (int32_t)g;
        in.instance_id = (int32_t)g;
      }
      int32_t id;
      if (ss >> id) in.instance_id = id;
      in.l2w = affine_from_trs(t, scale, rot, &in.w2l);
      sc.explicit_instances.push_back(in);
    } else if (cmd == "sphere" || cmd == "box" || cmd == "disk" || cmd == "quad" || cmd == "plane") {
      xb_prim q{};
      std::string mname;
      float* p = q.p;
      if (cmd == "sphere") { q.type = XB_PRIM_SPHERE; ss >> p[0] >> p[1] >> p[2] >> p[3] >> mname; }
      else if (cmd == "box") { q.type = XB_PRIM_BOX; ss >> p[0] >> p[1] >> p[2] >> p[3] >> p[4] >> p[5] >> mname; }
      else if (cmd == "disk") { q.type = XB_PRIM_DISK; ss >> p[0] >> p[1] >> p[2] >> p[3] >> p[4] >> p[5] >> p[6] >> mname; }
      else if (cmd == "quad") { q.type = XB_PRIM_QUAD; ss >> p[0] >> p[1] >> p[2] >> p[3] >> p[4] >> p[5] >> p[6] >> p[7] >> p[8] >> mname; }
      else { q.type = XB_PRIM_PLANE; ss >> p[0] >> p[1] >> p[2] >> p[3] >> mname; }
      if (q.type == XB_PRIM_DISK || q.type == XB_PRIM_PLANE) {
        float* n = (q.type == XB_PRIM_DISK) ? p + 3 : p;
        F3 nv(n[0], n[1], n[2]);
        float len = len3(nv);
        if (len > 1e-6f) { nv = div_scalar(nv, len); n[0] = nv.x; n[1] = nv.y; n[2] = nv.z; }
      }
      q.mat_id = mat_of(mname);
      sc.prims.push_back(q);
    }
  }
  cam->eye[0] = eye.x; cam->eye[1] = eye.y; cam->eye[2] = eye.z;
  cam->target[0] = target.x; cam->target[1] = target.y; cam->target[2] = target.z;
  cam->fov_y_deg = fov;
  sc.build();
  return true;
}

}  // namespace xb
