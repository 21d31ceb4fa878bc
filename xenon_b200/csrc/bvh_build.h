// bvh_build.h — the binned-SAH builds of the host scene (internal to the library).
//
// Two forms give the same node and order arrays:
//   * the recursive build in scene_host.cpp (BvhBuilder), which follows the reference's
//     BLAS::build / PrimBLAS::build / TLAS::build step for step;
//   * build_bvh_levels (bvh_levels.cpp), the level-synchronous form: every node of a depth is
//     split at once, and each step is an ordered reduction, a prefix sum or a per-node scan.
//     This is the form a device build takes.
#pragma once

#include <cstdint>
#include <vector>

#include "../../include/xenon_b200.h"
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
void build_bvh_levels(std::vector<BuildItem>& items, int bins, uint32_t max_leaf, bool leaf_cost,
                      std::vector<xb_bvh_node>& nodes, std::vector<uint32_t>& order);

}  // namespace xb
