// bvh_level_steps.h — the per-thread steps of the level-synchronous BVH build, shared by its
// host form (bvh_levels.cpp) and its device form (bvh_device.cu), so that the CPU tests of the
// host form check the arithmetic the device runs.
//
// A level holds the nodes being split at one depth. A node covers items [lo, hi). Its items are
// cut into chunks of kLevelChunk (the last one shorter), and a chunk is one device thread's range.
// Every fold keeps the first of equal values (bvh_refit.h), so folding chunks and then the chunk
// results in chunk order gives the sequential fold of the recursive build exactly.
//
// All arithmetic is the recursive build's, operation for operation (scene_host.cpp BvhBuilder,
// after the reference's src/geometry/blas.cpp:100-205). The device file is compiled with
// -fmad=false and the host files with -ffp-contract=off, so no product is fused into a sum.
#pragma once

#include <cstdint>

#include "bvh_refit.h"

namespace xb {

constexpr uint32_t kLevelChunk = 64;
constexpr int kLevelMaxBins = 16;

// One build item: its box, its centroid and the index it stands for (a triangle, a primitive
// or an instance).
struct LevelItem {
  float mn[3], mx[3];
  float c[3];
  uint32_t index;
};

// Bounds of the items' boxes and of their centroids over [b, e).
XB_HD void level_chunk_bounds(const LevelItem* it, uint32_t b, uint32_t e, RefitBox& box, RefitBox& cbox) {
  refit_empty(box);
  refit_empty(cbox);
  for (uint32_t i = b; i < e; ++i) {
    RefitBox ib;
    for (int k = 0; k < 3; ++k) { ib.mn[k] = it[i].mn[k]; ib.mx[k] = it[i].mx[k]; }
    refit_grow(box, ib);
    refit_grow(cbox, it[i].c[0], it[i].c[1], it[i].c[2]);
  }
}

// The split axis (largest centroid extent, x before y before z on ties only when strictly
// larger, as max_axis3), its lowest centroid and the bin scale. False when the centroids
// coincide along that axis: the node becomes a leaf.
XB_HD bool level_plane(const RefitBox& cb, int bins, int* axis, float* cmin, float* scale) {
  const float ex = cb.mx[0] - cb.mn[0], ey = cb.mx[1] - cb.mn[1], ez = cb.mx[2] - cb.mn[2];
  const int a = (ex > ey && ex > ez) ? 0 : (ey > ez ? 1 : 2);
  const float ext = a == 0 ? ex : (a == 1 ? ey : ez);
  if (ext == 0.f) return false;
  *axis = a;
  *scale = (float)bins / ext;
  *cmin = cb.mn[a];
  return true;
}

XB_HD int level_bin(const LevelItem& p, int axis, float cmin, float scale, int bins) {
  const int b = (int)((p.c[axis] - cmin) * scale);
  return b >= bins ? bins - 1 : b;
}

// Per-bin counts and boxes of the items in [b, e).
XB_HD void level_chunk_bins(const LevelItem* it, uint32_t b, uint32_t e, int axis, float cmin, float scale,
                            int bins, RefitBox* bin_box, int* bin_cnt) {
  for (int k = 0; k < bins; ++k) { refit_empty(bin_box[k]); bin_cnt[k] = 0; }
  for (uint32_t i = b; i < e; ++i) {
    const int k = level_bin(it[i], axis, cmin, scale, bins);
    RefitBox ib;
    for (int d = 0; d < 3; ++d) { ib.mn[d] = it[i].mn[d]; ib.mx[d] = it[i].mx[d]; }
    bin_cnt[k]++;
    refit_grow(bin_box[k], ib);
  }
}

// Surface area 2 (e.x e.y + e.y e.z + e.z e.x), the extent e = mx - mn (Bounds::area).
XB_HD float level_area(const RefitBox& b) {
  const float ex = b.mx[0] - b.mn[0], ey = b.mx[1] - b.mn[1], ez = b.mx[2] - b.mn[2];
  return 2.f * (ex * ey + ey * ez + ez * ex);
}

// The SAH sweep (sah_best_split in scene_host.cpp): the best plane, -1 if none, and its cost.
XB_HD int level_sah(const RefitBox* bin_box, const int* bin_cnt, int bins, const RefitBox& node_box,
                    float* best_cost) {
  float l_area[kLevelMaxBins], r_area[kLevelMaxBins];
  int l_cnt[kLevelMaxBins], r_cnt[kLevelMaxBins];
  RefitBox acc;
  refit_empty(acc);
  int run = 0;
  for (int i = 0; i < bins - 1; ++i) {
    run += bin_cnt[i]; l_cnt[i] = run;
    refit_grow(acc, bin_box[i]); l_area[i] = level_area(acc);
  }
  refit_empty(acc);
  run = 0;
  for (int i = bins - 1; i > 0; --i) {
    run += bin_cnt[i]; r_cnt[i - 1] = run;
    refit_grow(acc, bin_box[i]); r_area[i - 1] = level_area(acc);
  }
  const float parent = level_area(node_box);
  float best = __builtin_huge_valf();
  int best_bin = -1;
  for (int i = 0; i < bins - 1; ++i) {
    const float c = (l_area[i] * l_cnt[i] + r_area[i] * r_cnt[i]) / parent;
    if (c < best) { best = c; best_bin = i; }
  }
  *best_cost = best;
  return best_bin;
}

// Whether an item goes left of the chosen plane.
XB_HD bool level_pass(const LevelItem& p, int axis, float cmin, float scale, int bins, int best_bin) {
  return level_bin(p, axis, cmin, scale, bins) <= best_bin;
}

// The partition, as std::partition's two-pointer exchange leaves it. With m of the node's items
// passing, an item at offset i (from lo) that passed_before items before it passed:
//   * fails and i < m: it is the k-th failing item left of the split point, k = i - passed_before;
//   * passes and i >= m: it is the k-th passing item right of it counted from the right,
//     k = m - passed_before - 1;
//   * otherwise it stays.
// The k-th of the first kind and the k-th of the second trade places. Returns k, or -1 for an
// item that stays.
XB_HD int64_t level_exchange_rank(uint32_t i, bool pass, uint32_t passed_before, uint32_t m) {
  if (!pass && i < m) return (int64_t)i - passed_before;
  if (pass && i >= m) return (int64_t)m - passed_before - 1;
  return -1;
}

}  // namespace xb
