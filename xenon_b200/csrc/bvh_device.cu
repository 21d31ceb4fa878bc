// bvh_device.cu — the level-synchronous BVH build on the device (XB_BUILD_DEVICE).
//
// The host form of this build (bvh_levels.cpp) and this one run the same per-thread steps
// (bvh_level_steps.h), so their node and order arrays equal the recursive build's, and so the
// reference's. The host drives one pass per depth:
//   1. lvl_bounds:   per chunk, the items' box and centroid bounds;
//   2. lvl_plane:    per node, the chunk bounds folded in chunk order; leaf or split axis;
//   3. lvl_bins:     per chunk of a splitting node, bin counts and boxes;
//   4. lvl_sah:      per node, the bins folded in chunk order and the SAH sweep;
//   5. lvl_pass:     per chunk, how many items go left;
//   6. lvl_prefix:   per node, the exclusive prefix of those counts and the total m;
//   7. lvl_rank:     per chunk, each moving item's exchange rank, written to the rank tables;
//   8. lvl_exchange: per rank slot, the pair swapped in place (pairs are disjoint).
// The host reads each node's outcome back, makes the next depth's node list and, for the rare
// split whose partition leaves a side empty, runs std::nth_element on those items itself. Node
// indices are placed on the host from subtree sizes (place_level_nodes). The build runs on the
// calling thread's current CUDA device, on the default stream; no kernel waits on another.
#include <cuda_runtime.h>

#include <algorithm>
#include <stdexcept>
#include <string>
#include <vector>

#include "bvh_build.h"
#include "bvh_level_steps.h"

namespace xb {
namespace {

struct LevelTask {
  uint32_t lo, hi;
  uint32_t chunk0, nchunks;   // the node's chunks in the level's chunk list
};

struct ChunkRef {
  uint32_t node, b, e;        // items [b, e) of level node `node`
};

struct NodeOut {
  RefitBox box;
  int32_t state;              // 0 a leaf, 1 a split, 2 a split the host partitions
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
  RefitBox* chunk_bins;       // bins per chunk
  int32_t* chunk_cnt;         // bins per chunk
  uint32_t* chunk_pass;
  uint32_t* chunk_before;
  int64_t* left_of;           // per item slot: lo + rank -> item index (-1: none)
  int64_t* right_of;
  int32_t* error;
  uint32_t ntasks, nchunks, nitems, max_leaf;
  int32_t bins, leaf_cost;
};

__global__ void lvl_bounds(LevelArgs a) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.nchunks) return;
  const ChunkRef r = a.chunks[c];
  level_chunk_bounds(a.items, r.b, r.e, a.chunk_box[c], a.chunk_cbox[c]);
}

__global__ void lvl_plane(LevelArgs a) {
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= a.ntasks) return;
  const LevelTask t = a.tasks[x];
  RefitBox box, cb;
  refit_empty(box);
  refit_empty(cb);
  for (uint32_t c = t.chunk0; c < t.chunk0 + t.nchunks; ++c) {
    refit_grow(box, a.chunk_box[c]);
    refit_grow(cb, a.chunk_cbox[c]);
  }
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

__global__ void lvl_bins(LevelArgs a) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.nchunks) return;
  const ChunkRef r = a.chunks[c];
  const NodeOut& o = a.out[r.node];
  if (o.state != 1) return;
  level_chunk_bins(a.items, r.b, r.e, o.axis, o.cmin, o.scale, a.bins, a.chunk_bins + (size_t)c * a.bins,
                   a.chunk_cnt + (size_t)c * a.bins);
}

__global__ void lvl_sah(LevelArgs a) {
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= a.ntasks) return;
  NodeOut& o = a.out[x];
  if (o.state != 1) return;
  const LevelTask t = a.tasks[x];
  RefitBox bin_box[kLevelMaxBins];
  int bin_cnt[kLevelMaxBins];
  for (int k = 0; k < a.bins; ++k) { refit_empty(bin_box[k]); bin_cnt[k] = 0; }
  for (uint32_t c = t.chunk0; c < t.chunk0 + t.nchunks; ++c)
    for (int k = 0; k < a.bins; ++k) {
      bin_cnt[k] += a.chunk_cnt[(size_t)c * a.bins + k];
      refit_grow(bin_box[k], a.chunk_bins[(size_t)c * a.bins + k]);
    }
  float best;
  const int best_bin = level_sah(bin_box, bin_cnt, a.bins, o.box, &best);
  if ((a.leaf_cost && best >= (float)(t.hi - t.lo)) || best_bin < 0) o.state = 0;
  else o.best_bin = best_bin;
}

__global__ void lvl_pass(LevelArgs a) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.nchunks) return;
  const ChunkRef r = a.chunks[c];
  const NodeOut& o = a.out[r.node];
  if (o.state != 1) return;
  uint32_t n = 0;
  for (uint32_t i = r.b; i < r.e; ++i) n += level_pass(a.items[i], o.axis, o.cmin, o.scale, a.bins, o.best_bin);
  a.chunk_pass[c] = n;
}

__global__ void lvl_prefix(LevelArgs a) {
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= a.ntasks) return;
  NodeOut& o = a.out[x];
  if (o.state != 1) return;
  const LevelTask t = a.tasks[x];
  uint32_t m = 0;
  for (uint32_t c = t.chunk0; c < t.chunk0 + t.nchunks; ++c) {
    a.chunk_before[c] = m;
    m += a.chunk_pass[c];
  }
  o.m = m;
  if (m == 0 || m == t.hi - t.lo) o.state = 2;
}

__global__ void lvl_rank(LevelArgs a) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.nchunks) return;
  const ChunkRef r = a.chunks[c];
  const NodeOut& o = a.out[r.node];
  if (o.state != 1) return;
  const uint32_t lo = a.tasks[r.node].lo;
  uint32_t before = a.chunk_before[c];
  for (uint32_t i = r.b; i < r.e; ++i) {
    const bool pass = level_pass(a.items[i], o.axis, o.cmin, o.scale, a.bins, o.best_bin);
    const int64_t k = level_exchange_rank(i - lo, pass, before, o.m);
    if (k >= 0) {
      if (lo + k >= a.nitems) { atomicExch(a.error, 1); return; }
      (i - lo < o.m ? a.left_of : a.right_of)[lo + k] = i;
    }
    before += pass;
  }
}

__global__ void lvl_exchange(LevelArgs a) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= a.nitems) return;
  const int64_t l = a.left_of[s];
  if (l < 0) return;
  const int64_t r = a.right_of[s];
  if (r < 0 || r >= a.nitems || l >= a.nitems) { atomicExch(a.error, 2); return; }
  const LevelItem t = a.items[l];
  a.items[l] = a.items[r];
  a.items[r] = t;
}

void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string("device BVH build: ") + what + ": " + cudaGetErrorString(e));
}

// A device array that grows to the largest size asked of it and frees itself.
template <class T>
struct DevArray {
  T* p = nullptr;
  size_t cap = 0;
  ~DevArray() { if (p) cudaFree(p); }
  T* need(size_t n, const char* what) {
    if (n <= cap) return p;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    ck(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)), what);
    cap = std::max<size_t>(n, 1);
    return p;
  }
};

unsigned blocks(size_t n) { return (unsigned)((n + 127) / 128); }

}  // namespace

void build_bvh_device(std::vector<BuildItem>& items, int bins, uint32_t max_leaf, bool leaf_cost,
                      std::vector<xb_bvh_node>& nodes, std::vector<uint32_t>& order) {
  if (bins < 2 || bins > kLevelMaxBins) throw std::invalid_argument("build_bvh_device: bins");
  nodes.clear();
  order.assign(items.size(), 0);
  if (items.empty()) return;
  if (items.size() >= (1u << 31)) throw std::invalid_argument("build_bvh_device: too many items");
  std::vector<LevelItem> host_items = to_level_items(items);
  const uint32_t n = (uint32_t)host_items.size();
  DevArray<LevelItem> d_items;
  DevArray<LevelTask> d_tasks;
  DevArray<ChunkRef> d_chunks;
  DevArray<NodeOut> d_out;
  DevArray<RefitBox> d_box, d_cbox, d_bins;
  DevArray<int32_t> d_cnt, d_error;
  DevArray<uint32_t> d_pass, d_before;
  DevArray<int64_t> d_left, d_right;
  ck(cudaMemcpy(d_items.need(n, "items"), host_items.data(), n * sizeof(LevelItem), cudaMemcpyHostToDevice),
     "upload items");
  d_left.need(n, "rank tables");
  d_right.need(n, "rank tables");
  ck(cudaMemset(d_error.need(1, "status"), 0, sizeof(int32_t)), "clear status");

  std::vector<LevelNodeRecord> all;
  all.push_back(LevelNodeRecord{0, n, -1, RefitBox()});
  std::vector<LevelTask> tasks;
  std::vector<ChunkRef> chunks;
  std::vector<NodeOut> out;
  for (size_t begin = 0; begin < all.size();) {
    const size_t end = all.size();
    tasks.clear();
    chunks.clear();
    for (size_t x = begin; x < end; ++x) {
      const uint32_t lo = all[x].lo, hi = all[x].hi;
      LevelTask t{lo, hi, (uint32_t)chunks.size(), 0};
      for (uint32_t c = lo; c < hi; c += kLevelChunk) {
        chunks.push_back(ChunkRef{(uint32_t)(x - begin), c, std::min(hi, c + kLevelChunk)});
        ++t.nchunks;
      }
      tasks.push_back(t);
    }
    LevelArgs a;
    a.items = d_items.p;
    a.ntasks = (uint32_t)tasks.size();
    a.nchunks = (uint32_t)chunks.size();
    a.nitems = n;
    a.max_leaf = max_leaf;
    a.bins = bins;
    a.leaf_cost = leaf_cost ? 1 : 0;
    a.tasks = d_tasks.need(tasks.size(), "tasks");
    a.chunks = d_chunks.need(chunks.size(), "chunks");
    a.out = d_out.need(tasks.size(), "node outcomes");
    a.chunk_box = d_box.need(chunks.size(), "chunk bounds");
    a.chunk_cbox = d_cbox.need(chunks.size(), "chunk bounds");
    a.chunk_bins = d_bins.need(chunks.size() * bins, "chunk bins");
    a.chunk_cnt = d_cnt.need(chunks.size() * bins, "chunk bins");
    a.chunk_pass = d_pass.need(chunks.size(), "chunk counts");
    a.chunk_before = d_before.need(chunks.size(), "chunk counts");
    a.left_of = d_left.p;
    a.right_of = d_right.p;
    a.error = d_error.p;
    ck(cudaMemcpy(d_tasks.p, tasks.data(), tasks.size() * sizeof(LevelTask), cudaMemcpyHostToDevice), "upload tasks");
    ck(cudaMemcpy(d_chunks.p, chunks.data(), chunks.size() * sizeof(ChunkRef), cudaMemcpyHostToDevice),
       "upload chunks");
    ck(cudaMemset(d_left.p, 0xff, (size_t)n * sizeof(int64_t)), "clear rank tables");
    ck(cudaMemset(d_right.p, 0xff, (size_t)n * sizeof(int64_t)), "clear rank tables");
    lvl_bounds<<<blocks(a.nchunks), 128>>>(a);
    lvl_plane<<<blocks(a.ntasks), 128>>>(a);
    lvl_bins<<<blocks(a.nchunks), 128>>>(a);
    lvl_sah<<<blocks(a.ntasks), 128>>>(a);
    lvl_pass<<<blocks(a.nchunks), 128>>>(a);
    lvl_prefix<<<blocks(a.ntasks), 128>>>(a);
    lvl_rank<<<blocks(a.nchunks), 128>>>(a);
    lvl_exchange<<<blocks(n), 128>>>(a);
    ck(cudaGetLastError(), "launch");
    out.resize(tasks.size());
    ck(cudaMemcpy(out.data(), d_out.p, out.size() * sizeof(NodeOut), cudaMemcpyDeviceToHost), "read outcomes");
    int32_t error = 0;
    ck(cudaMemcpy(&error, d_error.p, sizeof(error), cudaMemcpyDeviceToHost), "read status");
    if (error) throw std::runtime_error("device BVH build: exchange ranks disagree");
    for (size_t x = begin; x < end; ++x) {
      const NodeOut& o = out[x - begin];
      const uint32_t lo = all[x].lo, hi = all[x].hi;
      all[x].box = o.box;
      if (o.state == 0) continue;
      uint32_t mid;
      if (o.state == 2) {
        // one side empty: the recursive build's median split, on the host
        mid = lo + (hi - lo) / 2;
        std::vector<LevelItem> part(hi - lo);
        ck(cudaMemcpy(part.data(), d_items.p + lo, part.size() * sizeof(LevelItem), cudaMemcpyDeviceToHost),
           "read a median split");
        const int axis = o.axis;
        std::nth_element(part.begin(), part.begin() + (mid - lo), part.end(),
                         [axis](const LevelItem& p, const LevelItem& q) { return p.c[axis] < q.c[axis]; });
        ck(cudaMemcpy(d_items.p + lo, part.data(), part.size() * sizeof(LevelItem), cudaMemcpyHostToDevice),
           "write a median split");
      } else {
        mid = lo + o.m;
      }
      all[x].left = (int32_t)all.size();
      all.push_back(LevelNodeRecord{lo, mid, -1, RefitBox()});
      all.push_back(LevelNodeRecord{mid, hi, -1, RefitBox()});
    }
    begin = end;
  }
  ck(cudaMemcpy(host_items.data(), d_items.p, n * sizeof(LevelItem), cudaMemcpyDeviceToHost), "read items");
  place_level_nodes(all, nodes);
  for (uint32_t i = 0; i < n; ++i) {
    order[i] = host_items[i].index;
    const LevelItem& l = host_items[i];
    items[i].box.mn = F3(l.mn[0], l.mn[1], l.mn[2]);
    items[i].box.mx = F3(l.mx[0], l.mx[1], l.mx[2]);
    items[i].centroid = F3(l.c[0], l.c[1], l.c[2]);
    items[i].index = l.index;
  }
}

}  // namespace xb
