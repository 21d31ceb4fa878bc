// bvh_levels.cpp — the level-synchronous form of the binned-SAH build (bvh_build.h).
//
// The recursive build (BvhBuilder in scene_host.cpp, after the reference's BLAS::build,
// src/geometry/blas.cpp:100-205) splits depth first, one node at a time. Here every node of a
// depth is split in the same pass, and each step has the data-parallel form a device build
// uses, chosen so that the node and order arrays come out identical to the recursive build's.
// The per-thread steps are those of bvh_level_steps.h, which the device build runs too:
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
#include "bvh_level_steps.h"

namespace xb {
namespace {

class LevelBuilder {
 public:
  LevelBuilder(std::vector<LevelItem>& items, int bins, uint32_t max_leaf, bool leaf_cost)
      : it_(items), bins_(bins), max_leaf_(max_leaf), leaf_cost_(leaf_cost) {}

  void build(std::vector<xb_bvh_node>& nodes) {
    nodes.clear();
    if (it_.empty()) return;
    all_.clear();
    all_.push_back(LevelNodeRecord{0u, (uint32_t)it_.size(), -1, RefitBox()});
    // one pass per depth: the nodes of the depth, in the order their parents were split
    for (size_t begin = 0; begin < all_.size();) {
      const size_t end = all_.size();
      for (size_t x = begin; x < end; ++x) split(x);
      begin = end;
    }
    place_level_nodes(all_, nodes);
  }

 private:
  std::vector<LevelItem>& it_;
  int bins_;
  uint32_t max_leaf_;
  bool leaf_cost_;
  std::vector<LevelNodeRecord> all_;   // every node, in level order

  void split(size_t x) {
    const uint32_t lo = all_[x].lo, hi = all_[x].hi, count = hi - lo;
    // node box and centroid bounds: chunk partials, folded in chunk order
    RefitBox nb, cb;
    refit_empty(nb);
    refit_empty(cb);
    for (uint32_t c = lo; c < hi; c += kLevelChunk) {
      RefitBox pb, pc;
      level_chunk_bounds(it_.data(), c, std::min(hi, c + kLevelChunk), pb, pc);
      refit_grow(nb, pb);
      refit_grow(cb, pc);
    }
    all_[x].box = nb;
    if (count <= max_leaf_) return;
    int axis;
    float cmin, scale;
    if (!level_plane(cb, bins_, &axis, &cmin, &scale)) return;
    // bins: chunk partials, folded in chunk order
    RefitBox bin_box[kLevelMaxBins];
    int bin_cnt[kLevelMaxBins] = {};
    for (int k = 0; k < bins_; ++k) refit_empty(bin_box[k]);
    for (uint32_t c = lo; c < hi; c += kLevelChunk) {
      RefitBox pbox[kLevelMaxBins];
      int pcnt[kLevelMaxBins];
      level_chunk_bins(it_.data(), c, std::min(hi, c + kLevelChunk), axis, cmin, scale, bins_, pbox, pcnt);
      for (int k = 0; k < bins_; ++k) {
        bin_cnt[k] += pcnt[k];
        refit_grow(bin_box[k], pbox[k]);
      }
    }
    float best;
    const int best_bin = level_sah(bin_box, bin_cnt, bins_, nb, &best);
    if ((leaf_cost_ && best >= (float)count) || best_bin < 0) return;
    // passing items per chunk, their prefix over the node, and the total m
    std::vector<uint32_t> chunk_before;
    uint32_t m = 0;
    for (uint32_t c = lo; c < hi; c += kLevelChunk) {
      chunk_before.push_back(m);
      for (uint32_t i = c; i < std::min(hi, c + kLevelChunk); ++i)
        m += level_pass(it_[i], axis, cmin, scale, bins_, best_bin);
    }
    uint32_t mid;
    if (m == 0 || m == count) {
      mid = lo + count / 2;
      std::nth_element(it_.begin() + lo, it_.begin() + mid, it_.begin() + hi,
                       [axis](const LevelItem& a, const LevelItem& b) { return a.c[axis] < b.c[axis]; });
    } else {
      mid = lo + m;
      // each moving item's exchange rank, then the exchange
      const uint32_t moves = count - m;   // an upper bound on the exchanges
      std::vector<int64_t> left_of(moves, -1), right_of(moves, -1);
      for (uint32_t c = lo, ci = 0; c < hi; c += kLevelChunk, ++ci) {
        uint32_t before = chunk_before[ci];
        for (uint32_t i = c; i < std::min(hi, c + kLevelChunk); ++i) {
          const bool pass = level_pass(it_[i], axis, cmin, scale, bins_, best_bin);
          const int64_t k = level_exchange_rank(i - lo, pass, before, m);
          if (k >= 0) (i - lo < m ? left_of : right_of)[k] = i;
          before += pass;
        }
      }
      for (uint32_t k = 0; k < moves && left_of[k] >= 0; ++k) {
        if (right_of[k] < 0) throw std::logic_error("build_bvh_levels: exchange ranks disagree");
        std::swap(it_[left_of[k]], it_[right_of[k]]);
      }
    }
    all_[x].left = (int32_t)all_.size();
    all_.push_back(LevelNodeRecord{lo, mid, -1, RefitBox()});
    all_.push_back(LevelNodeRecord{mid, hi, -1, RefitBox()});
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
  std::vector<LevelItem> it = to_level_items(items);
  LevelBuilder(it, bins, max_leaf, leaf_cost).build(nodes);
  order.resize(it.size());
  for (size_t i = 0; i < it.size(); ++i) {
    order[i] = it[i].index;
    const LevelItem& l = it[i];
    items[i] = BuildItem{Bounds(), F3(l.c[0], l.c[1], l.c[2]), l.index};
    items[i].box.mn = F3(l.mn[0], l.mn[1], l.mn[2]);
    items[i].box.mx = F3(l.mx[0], l.mx[1], l.mx[2]);
  }
}

}  // namespace xb
