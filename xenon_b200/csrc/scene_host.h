// scene_host.h — host-side scene: meshes, analytic prims, materials, lights, sky, instances
// and their TLAS/BLAS, built on the CPU and flattened into an xb_scene_view for upload.
#pragma once

#include <string>
#include <vector>

#include "../../include/xenon_b200.h"
#include "host_math.h"

namespace xb {

struct HostMesh {
  std::vector<float> vx, vy, vz;
  std::vector<float> nx, ny, nz;      // empty → geometric normal
  std::vector<int32_t> indices;
  std::vector<int32_t> mat_ids;
  int32_t default_mat = 0;
  std::vector<xb_bvh_node> nodes;     // BLAS
  std::vector<uint32_t> prims;
  int num_vertices() const { return (int)vx.size(); }
  int num_triangles() const { return (int)indices.size() / 3; }
  F3 vertex(int i) const { return {vx[i], vy[i], vz[i]}; }
  void compute_smooth_normals();
  void transform(F3 pos, float scale, F3 rot_deg);
};

struct HostInstance {
  int32_t geom;
  int32_t instance_id;
  Affine l2w, w2l;
};

class HostScene {
 public:
  std::vector<xb_material> materials;
  std::vector<std::string> material_names;
  std::vector<HostMesh> meshes;
  std::vector<xb_prim> prims;
  std::vector<xb_bvh_node> prim_nodes;
  std::vector<uint32_t> prim_indices;
  std::vector<xb_light> lights;
  std::vector<xb_sun> suns;
  xb_sky sky;
  std::vector<HostInstance> explicit_instances;
  std::vector<HostInstance> instances;   // after build
  std::vector<xb_bvh_node> tlas_nodes;
  std::vector<uint32_t> tlas_inst;
  bool built = false;
  int build_threads = 0;   // BVH build threads (0: the machine's hardware threads, 1: one)
  int build_mode = 0;      // 0: recursive, 1: level-synchronous, 2: on the device (same arrays)

  HostScene();
  void build();
  void view(xb_scene_view* out);
  // Moves the vertices of a built mesh (positions: float[3 * num_vertices]; normals the same,
  // or null to keep them), refits its BLAS with the topology kept (bvh_refit.h) and rebuilds
  // the TLAS over the instances' new world boxes.
  void refit_mesh(int mesh, const float* positions, const float* normals);

 private:
  void build_tlas();
  std::vector<xb_mesh_view> mesh_views_;
  std::vector<xb_instance_view> inst_views_;
};

Bounds prim_bounds(const xb_prim& p);
// The TLAS build (8 bins, one instance per leaf) over instances placed by l2w, each over the
// box of its root node (null: an empty box), as HostScene::build makes it.
void build_tlas(const std::vector<Affine>& l2w, const std::vector<const xb_bvh_node*>& roots,
                std::vector<xb_bvh_node>& nodes, std::vector<uint32_t>& order, int mode = 0);
// Node boxes of a mesh's BLAS recomputed from its current vertices (bvh_refit.h).
void refit_blas(const HostMesh& m, std::vector<xb_bvh_node>& nodes);
Affine affine_from_trs(F3 t, float s, F3 rot_deg, Affine* inverse);
xb_material_derived prepare_material(const xb_material& m);
void default_material(xb_material* m);
bool load_mat_file(const std::string& path, xb_material* m, std::string* name);
bool load_obj(const std::string& path, HostMesh& mesh,
              const std::vector<std::string>& mat_names, int default_mat, std::string* err);
bool load_xenon(const std::string& path, HostScene& scene, xb_scene_config* cfg,
                xb_camera_desc* cam, std::string* err);

}  // namespace xb

namespace xb {
// Emitter data the device needs, computed with the reference's float operations:
// light vertices + Mesh::geo_normal (src/geometry/mesh.h:37-62), sun emission() (scene.h:48).
struct LightGeom {
  float p0[3], p1[3], p2[3], n[3];
};
bool light_geometry(const xb_scene_view& v, const xb_light& l, LightGeom* out);
// Per-material terms of the multiple-scattering factor (src/material/bsdf.h:212-249) that do not
// depend on directions: k1 = 5 exp(-2.69 a), k2 = 1 + 22.7 a^1.5 and F_ms = F_avg^2 E_avg / denom,
// computed once with the host libm the reference itself uses.
void multiscatter_constants(const xb_material_derived& d, float* k1, float* k2, float fms[3]);
void sun_emission(const xb_sun& s, float out[3]);
}  // namespace xb
