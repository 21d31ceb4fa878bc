// bvh_levels.cpp — the level-synchronous form of the binned-SAH build (bvh_build.h).
//
// The recursive build (BvhBuilder in scene_host.cpp, after the reference's BLAS::build,
// src/geometry/blas.cpp:100-205) splits depth first, one node at a time. Here every node of a
// depth is split in the same pass, and each step has the data-parallel form a device build
// uses, chosen so that the node and order arrays come out identical to the recursive build's.
// Its passes and its depth loop are those of bvh_level_kernels.h, which the device build
// (bvh_device.cu) runs too; here each pass is a loop over its thread indices:
//
//   * Bounds (of the item boxes, of their centroids, of each bin) are folds that keep the first
//     of equal values (std::min / std::max). Such a fold is associative, so folding fixed-size
//     chunks and then the chunk results in chunk order gives the sequential fold, ties between
//     +0 and -0 included. kLevelChunk items stand for one device thread's range.
//   * The partition is the permutation of the bidirectional std::partition of libstdc++ (the
//     library the reference is built with): a pointer from the left stops at each item that
//     fails the predicate, one from the right at each item that passes, and the two are
//     swapped until the pointers cross. With m items passing, the k-th failing item in the
//     first m positions trades places with the k-th passing item, counted from the right, in
//     the rest; nothing else moves. Both ranks are prefix sums of the predicate.
//   * A split whose partition leaves one side empty falls back to std::nth_element, as the
//     recursive build does (rare: a device build hands such a node to the host).
//   * Node indices follow the recursive build's depth-first allocation. A split allocates its
//     children as a pair. A left child's own pair comes right after its parent's pair. A right
//     child's comes after its left sibling's whole subtree: two nodes per interior node there.
#include <algorithm>
#include <stdexcept>

#include "bvh_build.h"
#include "bvh_level_kernels.h"

namespace xb {
namespace {

// Runs the passes of a depth as loops over their thread indices, in host memory.
struct HostLevelExec {
  std::vector<LevelItem>& items;
  std::vector<LevelTask> tasks;
  std::vector<ChunkRef> chunks;
  std::vector<NodeOut> out;
  std::vector<RefitBox> chunk_box, chunk_cbox, chunk_bins;
  std::vector<int32_t> chunk_cnt;
  std::vector<uint32_t> chunk_pass, chunk_before;
  std::vector<int64_t> left_of, right_of;

  explicit HostLevelExec(std::vector<LevelItem>& it)
      : items(it), left_of(it.size(), -1), right_of(it.size(), -1) {}

  void run_depth(LevelArgs& a, const std::vector<LevelTask>& t, const std::vector<ChunkRef>& c,
                 std::vector<NodeOut>& result, int32_t* error) {
    tasks = t;
    chunks = c;
    out.assign(t.size(), NodeOut());
    chunk_box.assign(c.size(), RefitBox());
    chunk_cbox.assign(c.size(), RefitBox());
    chunk_bins.assign(c.size() * a.bins, RefitBox());
    chunk_cnt.assign(c.size() * a.bins, 0);
    chunk_pass.assign(c.size(), 0);
    chunk_before.assign(c.size(), 0);
    a.items = items.data();
    a.tasks = tasks.data();
    a.chunks = chunks.data();
    a.out = out.data();
    a.chunk_box = chunk_box.data();
    a.chunk_cbox = chunk_cbox.data();
    a.chunk_bins = chunk_bins.data();
    a.chunk_cnt = chunk_cnt.data();
    a.chunk_pass = chunk_pass.data();
    a.chunk_before = chunk_before.data();
    a.left_of = left_of.data();
    a.right_of = right_of.data();
    a.error = error;
    for (uint32_t i = 0; i < a.ntasks; ++i) lvl_small_at(a, i);
    for (uint32_t i = 0; i < a.nchunks; ++i) lvl_bounds_at(a, i);
    for (uint32_t i = 0; i < a.ntasks; ++i) lvl_plane_at(a, i);
    for (uint32_t i = 0; i < a.nchunks; ++i) lvl_bins_at(a, i);
    for (uint32_t i = 0; i < a.ntasks; ++i) lvl_sah_at(a, i);
    for (uint32_t i = 0; i < a.nchunks; ++i) lvl_pass_at(a, i);
    for (uint32_t i = 0; i < a.ntasks; ++i) lvl_prefix_at(a, i);
    for (uint32_t i = 0; i < a.nchunks; ++i) lvl_rank_at(a, i);
    for (uint32_t i = 0; i < a.nitems; ++i) lvl_exchange_at(a, i);
    result = out;
  }

  void median_split(uint32_t lo, uint32_t mid, uint32_t hi, int axis) {
    level_median_split(items.data(), lo, mid, hi, axis);
  }
};

}  // namespace

// Node x of the level order goes to index pos[x]. Its child pair, if it has one, starts at
// pair[x]. internal[x] counts the interior nodes of x's subtree.
void place_level_nodes(const std::vector<LevelNodeRecord>& all, std::vector<xb_bvh_node>& nodes) {
  const size_t n = all.size();
  std::vector<uint32_t> internal(n, 0), pos(n, 0), pair(n, 0);
  for (size_t x = n; x-- > 0;)
    if (all[x].left >= 0) internal[x] = 1 + internal[all[x].left] + internal[all[x].left + 1];
  nodes.assign(1 + 2 * (size_t)internal[0], xb_bvh_node{});
  pair[0] = 1;
  for (size_t x = 0; x < n; ++x) {
    const LevelNodeRecord& d = all[x];
    xb_bvh_node& out = nodes[pos[x]];
    for (int k = 0; k < 3; ++k) { out.mn[k] = d.box.mn[k]; out.mx[k] = d.box.mx[k]; }
    if (d.left < 0) {
      out.child = d.lo;
      out.count = d.hi - d.lo;
      continue;
    }
    out.child = pair[x];
    out.count = 0;
    const int32_t l = d.left, r = d.left + 1;
    pos[l] = pair[x];
    pos[r] = pair[x] + 1;
    pair[l] = pair[x] + 2;
    pair[r] = pair[x] + 2 + 2 * internal[l];
  }
}

void from_level_items(const std::vector<LevelItem>& it, std::vector<BuildItem>& items, std::vector<uint32_t>& order) {
  order.resize(it.size());
  for (size_t i = 0; i < it.size(); ++i) {
    const LevelItem& l = it[i];
    order[i] = l.index;
    items[i].box.mn = F3(l.mn[0], l.mn[1], l.mn[2]);
    items[i].box.mx = F3(l.mx[0], l.mx[1], l.mx[2]);
    items[i].centroid = F3(l.c[0], l.c[1], l.c[2]);
    items[i].index = l.index;
  }
}

std::vector<LevelItem> to_level_items(const std::vector<BuildItem>& items) {
  std::vector<LevelItem> out(items.size());
  for (size_t i = 0; i < items.size(); ++i) {
    const BuildItem& b = items[i];
    out[i] = LevelItem{{b.box.mn.x, b.box.mn.y, b.box.mn.z}, {b.box.mx.x, b.box.mx.y, b.box.mx.z},
                       {b.centroid.x, b.centroid.y, b.centroid.z}, b.index};
  }
  return out;
}

void build_bvh_levels(std::vector<BuildItem>& items, int bins, uint32_t max_leaf, bool leaf_cost,
                      std::vector<xb_bvh_node>& nodes, std::vector<uint32_t>& order) {
  if (bins < 2 || bins > kLevelMaxBins) throw std::invalid_argument("build_bvh_levels: bins");
  if (items.size() >= (1u << 31)) throw std::invalid_argument("build_bvh_levels: too many items");
  std::vector<LevelItem> it = to_level_items(items);
  HostLevelExec ex(it);
  std::vector<LevelNodeRecord> all;
  run_level_build(ex, (uint32_t)it.size(), bins, max_leaf, leaf_cost, all);
  nodes.clear();
  if (!all.empty()) place_level_nodes(all, nodes);
  from_level_items(it, items, order);
}

}  // namespace xb
