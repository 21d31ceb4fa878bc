// bvh_level_kernels.h — the passes of the level-synchronous BVH build and the loop that drives
// them, shared by the host form (bvh_levels.cpp) and the device form (bvh_device.cu).
//
// Each pass is a function of one thread index (a chunk, a node or an item slot). The device runs
// a pass as one kernel launch over all indices; the host runs it as a loop over the same
// indices. No pass reads what another thread of the same pass writes, except lvl_exchange, whose
// threads swap disjoint pairs. So both orders give the same arrays, and the CPU tests of the
// host form run the device's pass code. The loop (run_level_build) is the same for both; an
// executor supplies the memory and runs the passes.
//
// One depth (nodes of more than kLevelChunk items; lvl_small_at splits each smaller node whole,
// in one thread, with the same steps):
//   1. lvl_bounds_at:   per chunk, the items' box and centroid bounds;
//   2. lvl_plane_at:    per node, the chunk bounds folded in chunk order; a leaf, or the axis;
//   3. lvl_bins_at:     per chunk of a splitting node, its bin counts and boxes;
//   4. lvl_sah_at:      per node, the bins folded in chunk order and the SAH sweep;
//   5. lvl_pass_at:     per chunk, how many items go left;
//   6. lvl_prefix_at:   per node, the exclusive prefix of those counts and their total m;
//   7. lvl_rank_at:     per chunk, each moving item's exchange rank, into the rank tables;
//   8. lvl_exchange_at: per rank slot, the pair it names swapped.
// Then the loop reads every node's outcome, runs the rare median split (a partition leaving a
// side empty) through the executor, and lists the next depth's nodes.
#pragma once

#include <algorithm>
#include <cstdint>
#include <stdexcept>
#include <vector>

#include "bvh_build.h"
#include "bvh_level_steps.h"

namespace xb {

struct LevelTask {
  uint32_t lo, hi;
  uint32_t chunk0, nchunks;   // the node's chunks in the depth's chunk list
};

struct ChunkRef {
  uint32_t node, b, e;        // items [b, e) of the depth's node `node`
};

struct NodeOut {
  RefitBox box;
  int32_t state;              // 0 a leaf, 1 a split, 2 a split by the median (host)
  uint32_t m;                 // items going left
  int32_t axis, best_bin;
  float cmin, scale;
};

struct LevelArgs {
  LevelItem* items;
  const LevelTask* tasks;
  const ChunkRef* chunks;
  NodeOut* out;
  RefitBox* chunk_box;
  RefitBox* chunk_cbox;
  RefitBox* chunk_bins;       // `bins` per chunk
  int32_t* chunk_cnt;         // `bins` per chunk
  uint32_t* chunk_pass;
  uint32_t* chunk_before;
  int64_t* left_of;           // per item slot lo + rank: the failing item's index (-1: none);
  int64_t* right_of;          // the passing item's. All -1 between depths (lvl_exchange_at)
  int32_t* error;             // 0; 1 a rank outside the tables; 2 a rank with one side only
  uint32_t ntasks, nchunks, nitems, max_leaf;
  int32_t bins, leaf_cost;
};

XB_HD void level_error(int32_t* error, int32_t code) {
#ifdef __CUDA_ARCH__
  atomicExch(error, code);
#else
  *error = code;
#endif
}

// Chunks of a node of `size` items: none for a node that one thread splits whole (lvl_small_at).
XB_HD uint32_t level_node_chunks(uint32_t size) {
  return size > kLevelChunk ? (size + kLevelChunk - 1) / kLevelChunk : 0u;
}

XB_HD void lvl_bounds_at(const LevelArgs& a, uint32_t c) {
  const ChunkRef r = a.chunks[c];
  level_chunk_bounds(a.items, r.b, r.e, a.chunk_box[c], a.chunk_cbox[c]);
}

// A node's box and split plane from its folded chunk bounds (box: the items', cb: their
// centroids').
XB_HD void lvl_plane_finish(const LevelArgs& a, uint32_t x, const RefitBox& box, const RefitBox& cb) {
  const LevelTask t = a.tasks[x];
  NodeOut o;
  o.box = box;
  o.state = 0;
  o.m = 0;
  o.axis = 0;
  o.best_bin = -1;
  o.cmin = 0.f;
  o.scale = 0.f;
  if (t.hi - t.lo > a.max_leaf && level_plane(cb, a.bins, &o.axis, &o.cmin, &o.scale)) o.state = 1;
  a.out[x] = o;
}

XB_HD void lvl_plane_at(const LevelArgs& a, uint32_t x) {
  const LevelTask t = a.tasks[x];
  if (t.nchunks == 0) return;
  RefitBox box, cb;
  refit_empty(box);
  refit_empty(cb);
  for (uint32_t c = t.chunk0; c < t.chunk0 + t.nchunks; ++c) {
    refit_grow(box, a.chunk_box[c]);
    refit_grow(cb, a.chunk_cbox[c]);
  }
  lvl_plane_finish(a, x, box, cb);
}

XB_HD void lvl_bins_at(const LevelArgs& a, uint32_t c) {
  const ChunkRef r = a.chunks[c];
  const NodeOut& o = a.out[r.node];
  if (o.state != 1) return;
  RefitBox box[kLevelMaxBins];
  int cnt[kLevelMaxBins];
  level_chunk_bins(a.items, r.b, r.e, o.axis, o.cmin, o.scale, a.bins, box, cnt);
  for (int k = 0; k < a.bins; ++k) {
    a.chunk_bins[(size_t)c * a.bins + k] = box[k];
    a.chunk_cnt[(size_t)c * a.bins + k] = cnt[k];
  }
}

// A splitting node's SAH sweep over its folded bins: the plane, or a leaf.
XB_HD void lvl_sah_finish(const LevelArgs& a, uint32_t x, const RefitBox* bin_box, const int* bin_cnt) {
  NodeOut& o = a.out[x];
  const LevelTask t = a.tasks[x];
  float best;
  const int best_bin = level_sah(bin_box, bin_cnt, a.bins, o.box, &best);
  if ((a.leaf_cost && best >= (float)(t.hi - t.lo)) || best_bin < 0) o.state = 0;
  else o.best_bin = best_bin;
}

XB_HD void lvl_sah_at(const LevelArgs& a, uint32_t x) {
  const LevelTask t = a.tasks[x];
  if (t.nchunks == 0 || a.out[x].state != 1) return;
  RefitBox bin_box[kLevelMaxBins];
  int bin_cnt[kLevelMaxBins];
  for (int k = 0; k < a.bins; ++k) { refit_empty(bin_box[k]); bin_cnt[k] = 0; }
  for (uint32_t c = t.chunk0; c < t.chunk0 + t.nchunks; ++c)
    for (int k = 0; k < a.bins; ++k) {
      bin_cnt[k] += a.chunk_cnt[(size_t)c * a.bins + k];
      refit_grow(bin_box[k], a.chunk_bins[(size_t)c * a.bins + k]);
    }
  lvl_sah_finish(a, x, bin_box, bin_cnt);
}

XB_HD void lvl_pass_at(const LevelArgs& a, uint32_t c) {
  const ChunkRef r = a.chunks[c];
  const NodeOut& o = a.out[r.node];
  if (o.state != 1) return;
  uint32_t n = 0;
  for (uint32_t i = r.b; i < r.e; ++i) n += level_pass(a.items[i], o.axis, o.cmin, o.scale, a.bins, o.best_bin);
  a.chunk_pass[c] = n;
}

// m items of a splitting node go left; a partition leaving a side empty goes to the median.
XB_HD void lvl_prefix_finish(const LevelArgs& a, uint32_t x, uint32_t m) {
  NodeOut& o = a.out[x];
  const LevelTask t = a.tasks[x];
  o.m = m;
  if (m == 0 || m == t.hi - t.lo) o.state = 2;
}

XB_HD void lvl_prefix_at(const LevelArgs& a, uint32_t x) {
  const LevelTask t = a.tasks[x];
  if (t.nchunks == 0 || a.out[x].state != 1) return;
  uint32_t m = 0;
  for (uint32_t c = t.chunk0; c < t.chunk0 + t.nchunks; ++c) {
    a.chunk_before[c] = m;
    m += a.chunk_pass[c];
  }
  lvl_prefix_finish(a, x, m);
}

XB_HD void lvl_rank_at(const LevelArgs& a, uint32_t c) {
  const ChunkRef r = a.chunks[c];
  const NodeOut& o = a.out[r.node];
  if (o.state != 1) return;
  const uint32_t lo = a.tasks[r.node].lo;
  uint32_t before = a.chunk_before[c];
  for (uint32_t i = r.b; i < r.e; ++i) {
    const bool pass = level_pass(a.items[i], o.axis, o.cmin, o.scale, a.bins, o.best_bin);
    const int64_t k = level_exchange_rank(i - lo, pass, before, o.m);
    if (k >= 0) {
      if (lo + k >= a.nitems) { level_error(a.error, 1); return; }
      (i - lo < o.m ? a.left_of : a.right_of)[lo + k] = i;
    }
    before += pass;
  }
}

// The bidirectional std::partition of libstdc++ over items [first, last) by level_pass: from the
// left, stop at an item that fails; from the right, at one that passes; swap; until they meet.
XB_HD void level_partition(LevelItem* it, uint32_t first, uint32_t last, const NodeOut& o, int bins) {
  for (;;) {
    for (;;) {
      if (first == last) return;
      if (level_pass(it[first], o.axis, o.cmin, o.scale, bins, o.best_bin)) ++first;
      else break;
    }
    --last;
    for (;;) {
      if (first == last) return;
      if (!level_pass(it[last], o.axis, o.cmin, o.scale, bins, o.best_bin)) --last;
      else break;
    }
    const LevelItem t = it[first];
    it[first] = it[last];
    it[last] = t;
    ++first;
  }
}

// A node of at most kLevelChunk items, split whole: its bounds, plane, bins, SAH sweep and
// partition are the chunked passes' for a node of one chunk (a fold over one chunk is that
// chunk's own result), and the partition is the one the exchange ranks reproduce.
XB_HD void lvl_small_at(const LevelArgs& a, uint32_t x) {
  const LevelTask t = a.tasks[x];
  if (t.nchunks != 0) return;
  RefitBox box, cb;
  level_chunk_bounds(a.items, t.lo, t.hi, box, cb);
  lvl_plane_finish(a, x, box, cb);
  NodeOut& o = a.out[x];
  if (o.state != 1) return;
  RefitBox bin_box[kLevelMaxBins];
  int bin_cnt[kLevelMaxBins];
  level_chunk_bins(a.items, t.lo, t.hi, o.axis, o.cmin, o.scale, a.bins, bin_box, bin_cnt);
  lvl_sah_finish(a, x, bin_box, bin_cnt);
  if (o.state != 1) return;
  uint32_t m = 0;
  for (uint32_t i = t.lo; i < t.hi; ++i) m += level_pass(a.items[i], o.axis, o.cmin, o.scale, a.bins, o.best_bin);
  lvl_prefix_finish(a, x, m);
  if (o.state != 1) return;
  level_partition(a.items, t.lo, t.hi, o, a.bins);
}

// Swaps the pair slot s names and clears the slot, so the tables are all -1 again for the next
// depth (they start so).
XB_HD void lvl_exchange_at(const LevelArgs& a, uint32_t s) {
  const int64_t l = a.left_of[s];
  if (l < 0) return;
  const int64_t r = a.right_of[s];
  if (r < 0 || r >= a.nitems || l >= a.nitems) { level_error(a.error, 2); return; }
  const LevelItem t = a.items[l];
  a.items[l] = a.items[r];
  a.items[r] = t;
  a.left_of[s] = -1;
  a.right_of[s] = -1;
}

// The level loop over n items (already in the executor's memory). Exec provides
//   void run_depth(LevelArgs& a, const std::vector<LevelTask>&, const std::vector<ChunkRef>&,
//                  std::vector<NodeOut>& out, int32_t* error)
//       sets a's memory, runs lvl_small_at and the eight passes and reads back every node's
//       outcome and the error;
//   void median_split(uint32_t lo, uint32_t mid, uint32_t hi, int axis)
//       std::nth_element of items [lo, hi) at mid by centroid[axis].
template <class Exec>
void run_level_build(Exec& ex, uint32_t n, int bins, uint32_t max_leaf, bool leaf_cost,
                     std::vector<LevelNodeRecord>& all) {
  all.clear();
  if (n == 0) return;
  all.push_back(LevelNodeRecord{0u, n, -1, RefitBox()});
  std::vector<LevelTask> tasks;
  std::vector<ChunkRef> chunks;
  std::vector<NodeOut> out;
  for (size_t begin = 0; begin < all.size();) {
    const size_t end = all.size();
    tasks.clear();
    chunks.clear();
    for (size_t x = begin; x < end; ++x) {
      const uint32_t lo = all[x].lo, hi = all[x].hi;
      LevelTask t{lo, hi, (uint32_t)chunks.size(), level_node_chunks(hi - lo)};
      for (uint32_t k = 0; k < t.nchunks; ++k) {
        const uint32_t c = lo + k * kLevelChunk;
        chunks.push_back(ChunkRef{(uint32_t)(x - begin), c, std::min(hi, c + kLevelChunk)});
      }
      tasks.push_back(t);
    }
    LevelArgs a{};
    a.ntasks = (uint32_t)tasks.size();
    a.nchunks = (uint32_t)chunks.size();
    a.nitems = n;
    a.max_leaf = max_leaf;
    a.bins = bins;
    a.leaf_cost = leaf_cost ? 1 : 0;
    int32_t error = 0;
    ex.run_depth(a, tasks, chunks, out, &error);
    if (error) throw std::runtime_error("level BVH build: exchange ranks disagree");
    for (size_t x = begin; x < end; ++x) {
      const NodeOut& o = out[x - begin];
      const uint32_t lo = all[x].lo, hi = all[x].hi;
      all[x].box = o.box;
      if (o.state == 0) continue;
      uint32_t mid = lo + o.m;
      if (o.state == 2) {
        mid = lo + (hi - lo) / 2;
        ex.median_split(lo, mid, hi, o.axis);
      }
      all[x].left = (int32_t)all.size();
      all.push_back(LevelNodeRecord{lo, mid, -1, RefitBox()});
      all.push_back(LevelNodeRecord{mid, hi, -1, RefitBox()});
    }
    begin = end;
  }
}

// std::nth_element of the recursive build's median split, on host items.
inline void level_median_split(LevelItem* items, uint32_t lo, uint32_t mid, uint32_t hi, int axis) {
  std::nth_element(items + lo, items + mid, items + hi,
                   [axis](const LevelItem& p, const LevelItem& q) { return p.c[axis] < q.c[axis]; });
}

}  // namespace xb
