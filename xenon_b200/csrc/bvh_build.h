// bvh_build.h — the binned-SAH builds of the host scene (internal to the library).
//
// Three forms give the same node and order arrays:
//   * the recursive build in scene_host.cpp (BvhBuilder), which follows the reference's
//     BLAS::build / PrimBLAS::build / TLAS::build step for step;
//   * build_bvh_levels (bvh_levels.cpp), the level-synchronous form: every node of a depth is
//     split at once, and each step is an ordered reduction, a prefix sum or a per-node scan.
//     build_bvh_device (bvh_device.cu) runs this form on the device.
#pragma once

#include <cstdint>
#include <vector>

#include "../../include/xenon_b200.h"
#include "bvh_refit.h"
#include "host_math.h"

namespace xb {

struct BuildItem {
  Bounds box;
  F3 centroid;
  uint32_t index;
};

// The SAH sweep of one split over its bins (at most 16): the best plane (bins [0, plane] go
// left), -1 if none, and its cost in *best_cost. Both builds use it.
int sah_best_split(const Bounds* bin_box, const int* bin_cnt, int bins, const Bounds& node_box,
                   float* best_cost);

// bins: SAH bins per split (12 for a BLAS or the PrimBLAS, 8 for the TLAS); max_leaf: largest
// leaf; leaf_cost: make a leaf when the best split costs no less than the node's count. Items are
// reordered in place; order receives each leaf slot's item index.
struct LevelItem;
std::vector<LevelItem> to_level_items(const std::vector<BuildItem>& items);
// The items back, in their built order, and each slot's item index in order.
void from_level_items(const std::vector<LevelItem>& it, std::vector<BuildItem>& items, std::vector<uint32_t>& order);

// A node of the level-synchronous builds, in level order: items [lo, hi), the level-order
// index of its left child (the right child follows it; -1 for a leaf) and its box.
struct LevelNodeRecord {
  uint32_t lo, hi;
  int32_t left;
  RefitBox box;
};
// The node array in the recursive build's depth-first allocation order, from level-order nodes.
void place_level_nodes(const std::vector<LevelNodeRecord>& all, std::vector<xb_bvh_node>& nodes);

void build_bvh_levels(std::vector<BuildItem>& items, int bins, uint32_t max_leaf, bool leaf_cost,
                      std::vector<xb_bvh_node>& nodes, std::vector<uint32_t>& order);
// The same build run by the device (bvh_device.cu) on the current CUDA device: the same node
// and order arrays; the host items are left in their input order (the reordered items stay on
// the device). Throws std::runtime_error on a CUDA error, std::invalid_argument on bad arguments.
void build_bvh_device(const std::vector<BuildItem>& items, int bins, uint32_t max_leaf, bool leaf_cost,
                      std::vector<xb_bvh_node>& nodes, std::vector<uint32_t>& order);
// The device build of a triangle mesh's BLAS, its build items (each triangle's box in vertex
// order and its centroid, as HostScene::build makes them) made on the device from the mesh's
// vertices and indices: the same arrays as build_bvh_device over the host-made items.
struct HostMesh;
void build_bvh_device_mesh(const HostMesh& m, int bins, uint32_t max_leaf, bool leaf_cost,
                           std::vector<xb_bvh_node>& nodes, std::vector<uint32_t>& order);

}  // namespace xb
