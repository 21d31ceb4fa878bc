// bvh_levels.cpp — the level-synchronous form of the binned-SAH build (bvh_build.h).
//
// The recursive build (BvhBuilder in scene_host.cpp, after the reference's BLAS::build,
// src/geometry/blas.cpp:100-205) splits depth first, one node at a time. Here every node of a
// depth is split in the same pass, and each step has the data-parallel form a device build
// uses, chosen so that the node and order arrays come out identical to the recursive build's:
//
//   * Bounds (of the item boxes, of their centroids, of each bin) are folds that keep the first
//     of equal values (std::min / std::max). Such a fold is associative, so folding fixed-size
//     chunks and then the chunk results in chunk order gives the sequential fold, ties between
//     +0 and -0 included. kChunk items stand for one device thread's range.
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

namespace xb {
namespace {

constexpr uint32_t kChunk = 64;

struct LevelNode {
  uint32_t lo, hi;
  int32_t left;   // level-order index of the left child (the right child is left + 1); -1: a leaf
  Bounds box;
  LevelNode(uint32_t l, uint32_t h) : lo(l), hi(h), left(-1) {}
};

int bin_of(const BuildItem& p, int axis, float lo, float scale, int bins) {
  const int b = (int)((p.centroid[axis] - lo) * scale);
  return b >= bins ? bins - 1 : b;
}

// Bounds of f(items[i]) over [lo, hi), folded per chunk and then chunk by chunk.
template <class F>
Bounds chunked_bounds(uint32_t lo, uint32_t hi, F f) {
  Bounds total;
  for (uint32_t c = lo; c < hi; c += kChunk) {
    Bounds part;
    const uint32_t end = std::min(hi, c + kChunk);
    for (uint32_t i = c; i < end; ++i) f(part, i);
    total.grow(part);
  }
  return total;
}

class LevelBuilder {
 public:
  LevelBuilder(std::vector<BuildItem>& items, int bins, uint32_t max_leaf, bool leaf_cost)
      : it_(items), bins_(bins), max_leaf_(max_leaf), leaf_cost_(leaf_cost) {}

  void build(std::vector<xb_bvh_node>& nodes, std::vector<uint32_t>& order) {
    nodes.clear();
    order.assign(it_.size(), 0);
    if (it_.empty()) return;
    all_.clear();
    all_.emplace_back(0u, (uint32_t)it_.size());
    // one pass per depth: the nodes of the depth, in the order their parents were split
    for (size_t begin = 0; begin < all_.size();) {
      const size_t end = all_.size();
      for (size_t x = begin; x < end; ++x) split(x);
      begin = end;
    }
    place(nodes);
    for (size_t i = 0; i < it_.size(); ++i) order[i] = it_[i].index;
  }

 private:
  std::vector<BuildItem>& it_;
  int bins_;
  uint32_t max_leaf_;
  bool leaf_cost_;
  std::vector<LevelNode> all_;   // every node, in level order

  void split(size_t x) {
    const uint32_t lo = all_[x].lo, hi = all_[x].hi, count = hi - lo;
    const Bounds nb = chunked_bounds(lo, hi, [&](Bounds& b, uint32_t i) { b.grow(it_[i].box); });
    all_[x].box = nb;
    if (count <= max_leaf_) return;
    const Bounds cb = chunked_bounds(lo, hi, [&](Bounds& b, uint32_t i) { b.grow(it_[i].centroid); });
    const int axis = max_axis3(cb.extent());
    const float ext = cb.extent()[axis];
    if (ext == 0.f) return;
    const float scale = (float)bins_ / ext;
    const float cmin = cb.mn[axis];
    // bins: per-chunk counts and boxes, combined in chunk order
    Bounds bin_box[16];
    int bin_cnt[16] = {};
    for (uint32_t c = lo; c < hi; c += kChunk) {
      Bounds part_box[16];
      int part_cnt[16] = {};
      const uint32_t end = std::min(hi, c + kChunk);
      for (uint32_t i = c; i < end; ++i) {
        const int b = bin_of(it_[i], axis, cmin, scale, bins_);
        part_cnt[b]++;
        part_box[b].grow(it_[i].box);
      }
      for (int b = 0; b < bins_; ++b) {
        bin_cnt[b] += part_cnt[b];
        bin_box[b].grow(part_box[b]);
      }
    }
    float best;
    const int best_bin = sah_best_split(bin_box, bin_cnt, bins_, nb, &best);
    if ((leaf_cost_ && best >= (float)count) || best_bin < 0) return;
    // partition: ranks of the failing items left of the split point and of the passing items
    // right of it (counted from the right), then the pairwise exchange std::partition makes
    std::vector<uint8_t> pass(count);
    uint32_t m = 0;
    for (uint32_t i = 0; i < count; ++i) {
      pass[i] = bin_of(it_[lo + i], axis, cmin, scale, bins_) <= best_bin;
      m += pass[i];
    }
    uint32_t mid;
    if (m == 0 || m == count) {
      mid = lo + count / 2;
      std::nth_element(it_.begin() + lo, it_.begin() + mid, it_.begin() + hi,
                       [axis](const BuildItem& a, const BuildItem& b) {
                         return a.centroid[axis] < b.centroid[axis];
                       });
    } else {
      mid = lo + m;
      // k -> position of the k-th passing item, counted from the right
      std::vector<uint32_t> right_by_rank(count - m);
      uint32_t swaps = 0;
      for (uint32_t i = count; i-- > m;)
        if (pass[i]) right_by_rank[swaps++] = i;
      uint32_t k = 0;
      for (uint32_t i = 0; i < m; ++i)
        if (!pass[i]) std::swap(it_[lo + i], it_[lo + right_by_rank[k++]]);
      if (k != swaps) throw std::logic_error("build_bvh_levels: partition ranks disagree");
    }
    all_[x].left = (int32_t)all_.size();
    all_.emplace_back(lo, mid);
    all_.emplace_back(mid, hi);
  }

  // Node x of the level order goes to index pos[x]. Its child pair, if it has one, starts at
  // pair[x]. internal[x] counts the interior nodes of x's subtree.
  void place(std::vector<xb_bvh_node>& nodes) {
    const size_t n = all_.size();
    std::vector<uint32_t> internal(n, 0), pos(n, 0), pair(n, 0);
    for (size_t x = n; x-- > 0;)
      if (all_[x].left >= 0) internal[x] = 1 + internal[all_[x].left] + internal[all_[x].left + 1];
    nodes.assign(1 + 2 * (size_t)internal[0], xb_bvh_node{});
    pair[0] = 1;
    for (size_t x = 0; x < n; ++x) {
      const LevelNode& d = all_[x];
      xb_bvh_node& out = nodes[pos[x]];
      out.mn[0] = d.box.mn.x; out.mn[1] = d.box.mn.y; out.mn[2] = d.box.mn.z;
      out.mx[0] = d.box.mx.x; out.mx[1] = d.box.mx.y; out.mx[2] = d.box.mx.z;
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
};

}  // namespace

void build_bvh_levels(std::vector<BuildItem>& items, int bins, uint32_t max_leaf, bool leaf_cost,
                      std::vector<xb_bvh_node>& nodes, std::vector<uint32_t>& order) {
  LevelBuilder(items, bins, max_leaf, leaf_cost).build(nodes, order);
}

}  // namespace xb
