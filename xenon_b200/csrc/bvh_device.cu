// bvh_device.cu — the level-synchronous BVH build on the device (XB_BUILD_DEVICE).
//
// The passes are those of bvh_level_kernels.h, which the host form (bvh_levels.cpp,
// XB_BUILD_LEVELS) runs as loops, so the CPU tests of the host form run this build's pass code
// too. Here the whole depth loop stays on the device: the node list, each depth's node and chunk
// lists (prefix sums over the nodes' chunk counts), the eight passes, the children of each split
// (a prefix sum over the splits, so they are listed in the order the host loop appends them) and
// finally the node placement (subtree sizes bottom-up, positions top-down, one launch per depth).
// The folds over a node's chunks run one warp per node: each lane folds a contiguous run of
// chunks and the lanes' results are combined left to right, which is the sequential fold because
// every fold keeps the first of equal values and is therefore associative.
//
// The host reads back two small totals per depth (the chunk count, to size the passes; the
// children and median-split counts with the error flag). The rare median split
// (std::nth_element, a partition that leaves a side empty) runs on the host on that node's items.
// The build runs on the calling thread's current CUDA device, on the default stream; no kernel
// waits on another.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <stdexcept>
#include <string>
#include <vector>

#include "bvh_build.h"
#include "bvh_level_kernels.h"
#include "scene_host.h"

namespace xb {
namespace {

static_assert(sizeof(BuildItem) == sizeof(LevelItem) && offsetof(BuildItem, centroid) == offsetof(LevelItem, c) &&
                  offsetof(BuildItem, index) == offsetof(LevelItem, index),
              "BuildItem and LevelItem share one layout (box min, box max, centroid, index)");

// A node of the build: items [lo, hi), its first child (-1: none yet or a leaf) and its box.
struct DevRec {
  uint32_t lo, hi;
  int32_t left;
  RefitBox box;
};

// What the host reads after a depth.
struct DepthTotals {
  uint32_t chunks;     // chunks of the depth's nodes
  uint32_t children;   // nodes of the next depth
  uint32_t medians;    // nodes split by the median (listed in med_list)
  uint32_t big;        // nodes of more than kBlockNodeChunks chunks (listed in big_list)
  int32_t error;       // LevelArgs::error; 3 a child past the node array, 4 a node placed past it
};

constexpr unsigned kFull = 0xffffffffu;
constexpr uint32_t kBlockNodeChunks = 256;   // larger nodes fold their chunks with a block

// ── per-chunk and per-item passes: one thread each ──────────────────────────────────────────
__global__ void lvl_bounds(LevelArgs a) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < a.nchunks) lvl_bounds_at(a, i);
}
__global__ void lvl_bins(LevelArgs a) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < a.nchunks) lvl_bins_at(a, i);
}
__global__ void lvl_pass(LevelArgs a) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < a.nchunks) lvl_pass_at(a, i);
}
__global__ void lvl_rank(LevelArgs a) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < a.nchunks) lvl_rank_at(a, i);
}
__global__ void lvl_small(LevelArgs a) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < a.ntasks) lvl_small_at(a, i);
}
__global__ void lvl_exchange(LevelArgs a) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < a.nitems) lvl_exchange_at(a, i);
}

// ── per-node passes: one warp each ────────────────────────────────────────────────────────
// Lane `lane`'s contiguous run [b, e) of a node's n chunks.
__device__ __forceinline__ void lane_run(uint32_t n, uint32_t lane, uint32_t& b, uint32_t& e) {
  const uint32_t per = (n + 31) / 32;
  b = min(n, lane * per);
  e = min(n, b + per);
}

// Folds the lanes' boxes left to right into lane 0: at each step a lane that holds the fold of
// lanes [L, L + off) takes in the fold of [L + off, L + 2 off) as the right operand.
__device__ __forceinline__ void warp_fold(RefitBox& acc, uint32_t lane) {
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    RefitBox o;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      o.mn[k] = __shfl_down_sync(kFull, acc.mn[k], off);
      o.mx[k] = __shfl_down_sync(kFull, acc.mx[k], off);
    }
    if ((lane & (2 * off - 1)) == 0) refit_grow(acc, o);
  }
}

__device__ __forceinline__ int warp_sum(int v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(kFull, v, off);
  return v;
}

__global__ void lvl_plane_w(LevelArgs a) {
  const uint32_t x = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (x >= a.ntasks) return;   // the whole warp
  const LevelTask t = a.tasks[x];
  if (t.nchunks == 0 || t.nchunks > kBlockNodeChunks) return;   // lvl_small / lvl_plane_blk
  RefitBox box, cb;
  refit_empty(box);
  refit_empty(cb);
  uint32_t b, e;
  lane_run(t.nchunks, lane, b, e);
  for (uint32_t c = t.chunk0 + b; c < t.chunk0 + e; ++c) {
    refit_grow(box, a.chunk_box[c]);
    refit_grow(cb, a.chunk_cbox[c]);
  }
  warp_fold(box, lane);
  warp_fold(cb, lane);
  if (lane == 0) lvl_plane_finish(a, x, box, cb);
}

__global__ void lvl_sah_w(LevelArgs a) {
  const uint32_t x = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (x >= a.ntasks) return;   // the whole warp
  const LevelTask t = a.tasks[x];
  if (t.nchunks == 0 || t.nchunks > kBlockNodeChunks || a.out[x].state != 1) return;   // lvl_sah_blk
  RefitBox bin_box[kLevelMaxBins];
  int bin_cnt[kLevelMaxBins];
  for (int k = 0; k < a.bins; ++k) { refit_empty(bin_box[k]); bin_cnt[k] = 0; }
  uint32_t b, e;
  lane_run(t.nchunks, lane, b, e);
  for (uint32_t c = t.chunk0 + b; c < t.chunk0 + e; ++c)
    for (int k = 0; k < a.bins; ++k) {
      bin_cnt[k] += a.chunk_cnt[(size_t)c * a.bins + k];
      refit_grow(bin_box[k], a.chunk_bins[(size_t)c * a.bins + k]);
    }
  for (int k = 0; k < a.bins; ++k) {
    warp_fold(bin_box[k], lane);
    bin_cnt[k] = warp_sum(bin_cnt[k]);
  }
  if (lane == 0) lvl_sah_finish(a, x, bin_box, bin_cnt);
}

__global__ void lvl_prefix_w(LevelArgs a) {
  const uint32_t x = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (x >= a.ntasks) return;   // the whole warp
  const LevelTask t = a.tasks[x];
  if (t.nchunks == 0 || a.out[x].state != 1) return;
  uint32_t b, e;
  lane_run(t.nchunks, lane, b, e);
  uint32_t s = 0;
  for (uint32_t c = t.chunk0 + b; c < t.chunk0 + e; ++c) s += a.chunk_pass[c];
  uint32_t incl = s;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const uint32_t v = __shfl_up_sync(kFull, incl, off);
    if ((int)lane >= off) incl += v;
  }
  const uint32_t m = __shfl_sync(kFull, incl, 31);
  uint32_t run = incl - s;
  for (uint32_t c = t.chunk0 + b; c < t.chunk0 + e; ++c) {
    a.chunk_before[c] = run;
    run += a.chunk_pass[c];
  }
  if (lane == 0) lvl_prefix_finish(a, x, m);
}

// ── per-node folds of the largest nodes: one block each ─────────────────────────────────────
// A node of more than kBlockNodeChunks chunks (the top levels: the root has n / 64) would leave a
// warp folding hundreds of chunks per lane; these nodes, listed as the depth's chunk counts are
// made, take a block of kFoldThreads instead. Thread t folds a contiguous run of chunks, each warp
// folds its lanes left to right, and warp 0 folds the warps' results left to right: the
// sequential fold again.
constexpr int kFoldThreads = 256, kFoldWarps = kFoldThreads / 32;

__global__ void __launch_bounds__(kFoldThreads) lvl_plane_blk(LevelArgs a, const uint32_t* big_list,
                                                              const DepthTotals* tot) {
  __shared__ RefitBox sbox[kFoldWarps], scb[kFoldWarps];
  const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (uint32_t i = blockIdx.x; i < tot->big; i += gridDim.x) {
    const uint32_t x = big_list[i];
    const LevelTask t = a.tasks[x];
    const uint32_t per = (t.nchunks + kFoldThreads - 1) / kFoldThreads;
    const uint32_t b = min(t.nchunks, threadIdx.x * per), e = min(t.nchunks, b + per);
    RefitBox box, cb;
    refit_empty(box);
    refit_empty(cb);
    for (uint32_t c = t.chunk0 + b; c < t.chunk0 + e; ++c) {
      refit_grow(box, a.chunk_box[c]);
      refit_grow(cb, a.chunk_cbox[c]);
    }
    warp_fold(box, lane);
    warp_fold(cb, lane);
    if (lane == 0) { sbox[w] = box; scb[w] = cb; }
    __syncthreads();
    if (w == 0) {
      if (lane < kFoldWarps) { box = sbox[lane]; cb = scb[lane]; }
      else { refit_empty(box); refit_empty(cb); }
      warp_fold(box, lane);
      warp_fold(cb, lane);
      if (lane == 0) lvl_plane_finish(a, x, box, cb);
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kFoldThreads) lvl_sah_blk(LevelArgs a, const uint32_t* big_list,
                                                            const DepthTotals* tot) {
  __shared__ RefitBox sbox[kFoldWarps][kLevelMaxBins];
  __shared__ int scnt[kFoldWarps][kLevelMaxBins];
  const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (uint32_t i = blockIdx.x; i < tot->big; i += gridDim.x) {
    const uint32_t x = big_list[i];
    if (a.out[x].state != 1) continue;   // the whole block
    const LevelTask t = a.tasks[x];
    const uint32_t per = (t.nchunks + kFoldThreads - 1) / kFoldThreads;
    const uint32_t b = min(t.nchunks, threadIdx.x * per), e = min(t.nchunks, b + per);
    RefitBox bin_box[kLevelMaxBins];
    int bin_cnt[kLevelMaxBins];
    for (int k = 0; k < a.bins; ++k) { refit_empty(bin_box[k]); bin_cnt[k] = 0; }
    for (uint32_t c = t.chunk0 + b; c < t.chunk0 + e; ++c)
      for (int k = 0; k < a.bins; ++k) {
        bin_cnt[k] += a.chunk_cnt[(size_t)c * a.bins + k];
        refit_grow(bin_box[k], a.chunk_bins[(size_t)c * a.bins + k]);
      }
    for (int k = 0; k < a.bins; ++k) {
      warp_fold(bin_box[k], lane);
      bin_cnt[k] = warp_sum(bin_cnt[k]);
      if (lane == 0) { sbox[w][k] = bin_box[k]; scnt[w][k] = bin_cnt[k]; }
    }
    __syncthreads();
    if (w == 0) {
      for (int k = 0; k < a.bins; ++k) {
        RefitBox v;
        int n = 0;
        if (lane < kFoldWarps) { v = sbox[lane][k]; n = scnt[lane][k]; }
        else refit_empty(v);
        warp_fold(v, lane);
        n = warp_sum(n);
        bin_box[k] = v;
        bin_cnt[k] = n;
      }
      if (lane == 0) lvl_sah_finish(a, x, bin_box, bin_cnt);
    }
    __syncthreads();
  }
}

// ── exclusive prefix sums of uint32 counts (three launches) ────────────────────────────────
constexpr int kScanThreads = 256, kScanPer = 4, kScanTile = kScanThreads * kScanPer;

// The exclusive prefix of v over the block (blockDim.x a multiple of 32); *total: the block's sum.
__device__ uint32_t block_exclusive(uint32_t v, uint32_t* total) {
  __shared__ uint32_t warp_incl[32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  uint32_t incl = v;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const uint32_t u = __shfl_up_sync(kFull, incl, off);
    if (lane >= off) incl += u;
  }
  if (lane == 31) warp_incl[w] = incl;
  __syncthreads();
  if (w == 0) {
    uint32_t s = lane < nw ? warp_incl[lane] : 0u;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t u = __shfl_up_sync(kFull, s, off);
      if (lane >= off) s += u;
    }
    warp_incl[lane] = s;
  }
  __syncthreads();
  const uint32_t out = incl - v + (w > 0 ? warp_incl[w - 1] : 0u);
  *total = warp_incl[nw - 1];
  __syncthreads();
  return out;
}

__global__ void __launch_bounds__(kScanThreads) scan_tiles(const uint32_t* in, uint32_t* out, uint32_t n,
                                                          uint32_t* tile_sums) {
  const size_t base = (size_t)blockIdx.x * kScanTile + (size_t)threadIdx.x * kScanPer;
  uint32_t v[kScanPer], s = 0;
#pragma unroll
  for (int j = 0; j < kScanPer; ++j) {
    v[j] = base + j < n ? in[base + j] : 0u;
    s += v[j];
  }
  uint32_t total;
  uint32_t run = block_exclusive(s, &total);
#pragma unroll
  for (int j = 0; j < kScanPer; ++j) {
    if (base + j < n) out[base + j] = run;
    run += v[j];
  }
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

// One block: the tile sums become their exclusive prefix; *total the sum of all.
__global__ void __launch_bounds__(1024) scan_tile_sums(uint32_t* tile_sums, uint32_t ntiles, uint32_t* total) {
  const uint32_t per = (ntiles + blockDim.x - 1) / blockDim.x;
  const uint32_t b = min(ntiles, threadIdx.x * per), e = min(ntiles, b + per);
  uint32_t s = 0;
  for (uint32_t i = b; i < e; ++i) s += tile_sums[i];
  uint32_t all;
  uint32_t run = block_exclusive(s, &all);
  for (uint32_t i = b; i < e; ++i) {
    const uint32_t v = tile_sums[i];
    tile_sums[i] = run;
    run += v;
  }
  if (threadIdx.x == 0) *total = all;
}

__global__ void scan_add(uint32_t* out, uint32_t n, const uint32_t* tile_sums) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] += tile_sums[i / kScanTile];
}

// ── the depth loop's own steps ─────────────────────────────────────────────────────────────
__global__ void node_chunk_counts(const DevRec* recs, uint32_t begin, uint32_t ntasks, uint32_t* nch,
                                  uint32_t* big_list, DepthTotals* tot) {
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= ntasks) return;
  const DevRec r = recs[begin + x];
  const uint32_t c = level_node_chunks(r.hi - r.lo);
  nch[x] = c;
  if (c > kBlockNodeChunks) big_list[atomicAdd(&tot->big, 1u)] = x;
}

__global__ void node_tasks(const DevRec* recs, uint32_t begin, uint32_t ntasks, const uint32_t* nch,
                           const uint32_t* chunk0, LevelTask* tasks) {
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= ntasks) return;
  const DevRec r = recs[begin + x];
  tasks[x] = LevelTask{r.lo, r.hi, chunk0[x], nch[x]};
}

// Chunk c belongs to the last node whose first chunk is at most c (nodes without chunks share
// their first chunk index with the next node, so the last such node is the one that has c).
__global__ void node_chunks(const LevelTask* tasks, uint32_t ntasks, uint32_t nchunks, ChunkRef* chunks) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nchunks) return;
  uint32_t lo = 0, hi = ntasks;   // the first node with chunk0 > c lies in (lo, hi]
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) / 2;
    if (tasks[mid].chunk0 <= c) lo = mid;
    else hi = mid;
  }
  const LevelTask t = tasks[lo];
  const uint32_t b = t.lo + (c - t.chunk0) * kLevelChunk;
  chunks[c] = ChunkRef{lo, b, min(t.hi, b + kLevelChunk)};
}

// A node's box, and its children's count (2 for a split, 0 for a leaf); median splits listed.
__global__ void node_outcomes(DevRec* recs, uint32_t begin, uint32_t ntasks, const NodeOut* out, uint32_t* nchild,
                              uint32_t* med_list, DepthTotals* tot) {
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= ntasks) return;
  const NodeOut o = out[x];
  recs[begin + x].box = o.box;
  nchild[x] = o.state != 0 ? 2u : 0u;
  if (o.state == 2) med_list[atomicAdd(&tot->medians, 1u)] = x;
}

// The children of each split, at end + (the splits before it) * 2: the host loop's order.
// Every child holds one or more items, so there are at most 2n - 1 nodes (max_recs = 2n): a
// child beyond that is an error, not a write.
__global__ void node_children(DevRec* recs, uint32_t begin, uint32_t end, uint32_t ntasks, const NodeOut* out,
                              const uint32_t* child_off, size_t max_recs, int32_t* error) {
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= ntasks) return;
  const NodeOut o = out[x];
  if (o.state == 0) return;
  DevRec& r = recs[begin + x];
  const uint32_t mid = o.state == 2 ? r.lo + (r.hi - r.lo) / 2 : r.lo + o.m;
  const uint32_t l = end + child_off[x];
  if ((size_t)l + 2 > max_recs) { level_error(error, 3); return; }
  r.left = (int32_t)l;
  RefitBox empty;
  refit_empty(empty);
  recs[l] = DevRec{r.lo, mid, -1, empty};
  recs[l + 1] = DevRec{mid, r.hi, -1, empty};
}

// Interior nodes of each subtree, bottom-up one depth at a time (place_level_nodes).
__global__ void node_internal(const DevRec* recs, uint32_t begin, uint32_t end, uint32_t* internal) {
  const uint32_t x = begin + blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= end) return;
  const int32_t l = recs[x].left;
  internal[x] = l < 0 ? 0u : 1u + internal[l] + internal[l + 1];
}

// Node x goes to pos[x]; its child pair, if any, starts at pair[x] (place_level_nodes).
__global__ void node_place(const DevRec* recs, uint32_t begin, uint32_t end, const uint32_t* internal,
                           uint32_t* pos, uint32_t* pair, xb_bvh_node* nodes, uint32_t nn, int32_t* error) {
  const uint32_t x = begin + blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= end) return;
  const DevRec d = recs[x];
  xb_bvh_node n;
  for (int k = 0; k < 3; ++k) { n.mn[k] = d.box.mn[k]; n.mx[k] = d.box.mx[k]; }
  if (d.left < 0) {
    n.child = d.lo;
    n.count = d.hi - d.lo;
  } else {
    const uint32_t p = pair[x];
    n.child = p;
    n.count = 0;
    pos[d.left] = p;
    pos[d.left + 1] = p + 1;
    pair[d.left] = p + 2;
    pair[d.left + 1] = p + 2 + 2 * internal[d.left];
  }
  if (pos[x] >= nn) { level_error(error, 4); return; }
  nodes[pos[x]] = n;
}

__global__ void item_order(const LevelItem* items, uint32_t n, uint32_t* order) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) order[i] = items[i].index;
}

// Triangle t's build item, as the host makes it (HostScene::build): the box of its three vertices
// folded in index order with std::min / std::max semantics, and the centroid (mn + mx) * 0.5
// (this file is compiled without fused multiply-add, so the arithmetic is the host's).
__global__ void mesh_items(const float* vx, const float* vy, const float* vz, const int32_t* idx, uint32_t ntris,
                           LevelItem* items) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ntris) return;
  RefitBox b;
  refit_empty(b);
  for (int k = 0; k < 3; ++k) {
    const int32_t v = idx[3 * (size_t)t + k];
    refit_grow(b, vx[v], vy[v], vz[v]);
  }
  LevelItem it;
  for (int k = 0; k < 3; ++k) {
    it.mn[k] = b.mn[k];
    it.mx[k] = b.mx[k];
    it.c[k] = (b.mn[k] + b.mx[k]) * 0.5f;
  }
  it.index = t;
  items[t] = it;
}

__global__ void place_root(uint32_t* pos, uint32_t* pair) {
  pos[0] = 0;
  pair[0] = 1;
}

void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess)
    throw std::runtime_error(std::string("device BVH build: ") + what + ": " + cudaGetErrorString(e));
}

// One device allocation carved into the build's arrays, each 256-byte aligned; freed with it.
struct Arena {
  char* base = nullptr;
  size_t used = 0;
  Arena() = default;
  Arena(const Arena&) = delete;
  Arena& operator=(const Arena&) = delete;
  ~Arena() { if (base) cudaFree(base); }
  template <class T>
  void plan(T*& p, size_t count) {   // first pass: offsets only
    p = reinterpret_cast<T*>(used);
    used += (std::max<size_t>(count, 1) * sizeof(T) + 255) & ~(size_t)255;
  }
  template <class T>
  void place(T*& p) { p = reinterpret_cast<T*>(base + reinterpret_cast<size_t>(p)); }
};

unsigned blocks(size_t n, unsigned per = 128) { return (unsigned)((n + per - 1) / per); }

constexpr unsigned kBigBlocks = 148;   // blocks of lvl_*_blk, each taking listed nodes in turn

struct DeviceLevelBuild {
  uint32_t n = 0;
  int bins = 12;
  uint32_t max_leaf = 2;
  bool leaf_cost = true;
  Arena arena;
  // Sizes from n alone: at most 2n - 1 nodes (every child holds an item), at most n nodes in a
  // depth, and at most n / 64 + n / 65 chunks in a depth (only nodes of more than 64 items have
  // chunks, ceil(size / 64) <= size / 64 + 1 each).
  size_t max_recs = 0, max_tasks = 0, max_chunks = 0;
  LevelItem* items;
  DevRec* recs;
  LevelTask* tasks;
  ChunkRef* chunks;
  NodeOut* out;
  RefitBox *box, *cbox, *bin_box;
  int32_t* bin_cnt;
  uint32_t *pass, *before, *counts, *offsets, *tile_sums, *med_list, *big_list, *internal, *pos, *pair, *order;
  int64_t *left, *right;
  DepthTotals* tot;
  xb_bvh_node* dnodes;
  std::vector<std::pair<uint32_t, uint32_t>> depths;   // [begin, end) of each depth's records

  void allocate() {
    max_recs = 2 * (size_t)n;
    max_tasks = n;
    max_chunks = n / kLevelChunk + n / (kLevelChunk + 1) + 2;
    Arena& A = arena;
    A.plan(items, n);
    A.plan(recs, max_recs);
    A.plan(tasks, max_tasks);
    A.plan(out, max_tasks);
    A.plan(counts, max_tasks);
    A.plan(offsets, max_tasks);
    A.plan(med_list, max_tasks);
    A.plan(big_list, n / (kLevelChunk * kBlockNodeChunks) + 2);
    A.plan(tile_sums, blocks(max_tasks, kScanTile));
    A.plan(chunks, max_chunks);
    A.plan(box, max_chunks);
    A.plan(cbox, max_chunks);
    A.plan(bin_box, max_chunks * bins);
    A.plan(bin_cnt, max_chunks * bins);
    A.plan(pass, max_chunks);
    A.plan(before, max_chunks);
    A.plan(left, n);
    A.plan(right, n);
    A.plan(tot, 1);
    A.plan(internal, max_recs);
    A.plan(pos, max_recs);
    A.plan(pair, max_recs);
    A.plan(dnodes, max_recs);
    A.plan(order, n);
    ck(cudaMalloc(&A.base, A.used), "allocate the build's arrays");
    A.place(items); A.place(recs); A.place(tasks); A.place(out); A.place(counts); A.place(offsets);
    A.place(med_list); A.place(big_list); A.place(tile_sums); A.place(chunks); A.place(box); A.place(cbox); A.place(bin_box);
    A.place(bin_cnt); A.place(pass); A.place(before); A.place(left); A.place(right); A.place(tot);
    A.place(internal); A.place(pos); A.place(pair); A.place(dnodes); A.place(order);
  }

  // Exclusive prefix of in[0, count) into out; the sum into *total (device).
  void scan(const uint32_t* in, uint32_t* out_, uint32_t count, uint32_t* total) {
    const unsigned tiles = blocks(count, kScanTile);
    scan_tiles<<<tiles, kScanThreads>>>(in, out_, count, tile_sums);
    scan_tile_sums<<<1, 1024>>>(tile_sums, tiles, total);
    scan_add<<<blocks(count), 128>>>(out_, count, tile_sums);
  }

  DepthTotals read_totals() {
    DepthTotals t;
    ck(cudaMemcpy(&t, tot, sizeof(t), cudaMemcpyDeviceToHost), "read depth totals");
    return t;
  }

  void median_split(uint32_t x) {
    LevelTask t;
    NodeOut o;
    ck(cudaMemcpy(&t, tasks + x, sizeof(t), cudaMemcpyDeviceToHost), "read a median split");
    ck(cudaMemcpy(&o, out + x, sizeof(o), cudaMemcpyDeviceToHost), "read a median split");
    std::vector<LevelItem> part(t.hi - t.lo);
    ck(cudaMemcpy(part.data(), items + t.lo, part.size() * sizeof(LevelItem), cudaMemcpyDeviceToHost),
       "read a median split");
    level_median_split(part.data(), 0, (t.hi - t.lo) / 2, t.hi - t.lo, o.axis);
    ck(cudaMemcpy(items + t.lo, part.data(), part.size() * sizeof(LevelItem), cudaMemcpyHostToDevice),
       "write a median split");
  }

  // One depth over records [begin, end); returns the next depth's record count.
  uint32_t run_depth(uint32_t begin, uint32_t end) {
    const uint32_t ntasks = end - begin;
    if (ntasks > max_tasks) throw std::runtime_error("device BVH build: depth out of range");
    ck(cudaMemset(&tot->big, 0, sizeof(uint32_t)), "clear depth totals");
    node_chunk_counts<<<blocks(ntasks), 128>>>(recs, begin, ntasks, counts, big_list, tot);
    scan(counts, offsets, ntasks, &tot->chunks);
    const uint32_t nchunks = read_totals().chunks;
    if (nchunks > max_chunks) throw std::runtime_error("device BVH build: chunk count out of range");
    LevelArgs a{};
    a.items = items;
    a.tasks = tasks;
    a.chunks = chunks;
    a.out = out;
    a.chunk_box = box;
    a.chunk_cbox = cbox;
    a.chunk_bins = bin_box;
    a.chunk_cnt = bin_cnt;
    a.chunk_pass = pass;
    a.chunk_before = before;
    a.left_of = left;
    a.right_of = right;
    a.error = &tot->error;
    a.ntasks = ntasks;
    a.nchunks = nchunks;
    a.nitems = n;
    a.max_leaf = max_leaf;
    a.bins = bins;
    a.leaf_cost = leaf_cost ? 1 : 0;
    node_tasks<<<blocks(ntasks), 128>>>(recs, begin, ntasks, counts, offsets, tasks);
    lvl_small<<<blocks(ntasks), 128>>>(a);
    if (nchunks > 0) {   // nodes of more than kLevelChunk items
      const unsigned warps = blocks((size_t)ntasks * 32);
      node_chunks<<<blocks(nchunks), 128>>>(tasks, ntasks, nchunks, chunks);
      lvl_bounds<<<blocks(nchunks), 128>>>(a);
      lvl_plane_w<<<warps, 128>>>(a);
      lvl_plane_blk<<<kBigBlocks, kFoldThreads>>>(a, big_list, tot);
      lvl_bins<<<blocks(nchunks), 128>>>(a);
      lvl_sah_w<<<warps, 128>>>(a);
      lvl_sah_blk<<<kBigBlocks, kFoldThreads>>>(a, big_list, tot);
      lvl_pass<<<blocks(nchunks), 128>>>(a);
      lvl_prefix_w<<<warps, 128>>>(a);
      lvl_rank<<<blocks(nchunks), 128>>>(a);
      lvl_exchange<<<blocks(n), 128>>>(a);
    }
    ck(cudaMemset(&tot->medians, 0, sizeof(uint32_t)), "clear depth totals");
    node_outcomes<<<blocks(ntasks), 128>>>(recs, begin, ntasks, out, counts, med_list, tot);
    scan(counts, offsets, ntasks, &tot->children);
    node_children<<<blocks(ntasks), 128>>>(recs, begin, end, ntasks, out, offsets, max_recs, &tot->error);
    ck(cudaGetLastError(), "launch");
    const DepthTotals t = read_totals();
    if (t.error) throw std::runtime_error("device BVH build: inconsistent split (" + std::to_string(t.error) + ")");
    if (t.medians) {
      std::vector<uint32_t> xs(t.medians);
      ck(cudaMemcpy(xs.data(), med_list, xs.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost),
         "read median splits");
      for (uint32_t x : xs) median_split(x);
    }
    return t.children;
  }

  // The node and order arrays; the host items are left as they are.
  void build(const std::vector<BuildItem>& host_items, std::vector<xb_bvh_node>& nodes,
             std::vector<uint32_t>& order_out) {
    n = (uint32_t)host_items.size();
    allocate();
    ck(cudaMemcpy(items, host_items.data(), (size_t)n * sizeof(LevelItem), cudaMemcpyHostToDevice), "upload items");
    run(nodes, order_out);
  }

  // The same from a triangle mesh: its vertices and indices go up, the items are made on the
  // device (the positions and indices are about half the bytes of the items).
  void build(const HostMesh& m, std::vector<xb_bvh_node>& nodes, std::vector<uint32_t>& order_out) {
    n = (uint32_t)m.num_triangles();
    allocate();
    const size_t nv = (size_t)m.num_vertices();
    float* dv = nullptr;
    int32_t* di = nullptr;
    ck(cudaMalloc(&dv, std::max<size_t>(nv, 1) * 3 * sizeof(float)), "allocate the mesh");
    cudaError_t e = cudaMalloc(&di, (size_t)n * 3 * sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMemcpy(dv, m.vx.data(), nv * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dv + nv, m.vy.data(), nv * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dv + 2 * nv, m.vz.data(), nv * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(di, m.indices.data(), (size_t)n * 3 * sizeof(int32_t), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
      mesh_items<<<blocks(n), 128>>>(dv, dv + nv, dv + 2 * nv, di, n, items);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    cudaFree(dv);
    cudaFree(di);
    ck(e, "build items from the mesh");
    run(nodes, order_out);
  }

  void run(std::vector<xb_bvh_node>& nodes, std::vector<uint32_t>& order_out) {
    ck(cudaMemset(left, 0xff, (size_t)n * sizeof(int64_t)), "clear rank tables");
    ck(cudaMemset(right, 0xff, (size_t)n * sizeof(int64_t)), "clear rank tables");
    ck(cudaMemset(tot, 0, sizeof(DepthTotals)), "clear depth totals");
    DevRec root{0u, n, -1, RefitBox{}};
    refit_empty(root.box);
    ck(cudaMemcpy(recs, &root, sizeof(root), cudaMemcpyHostToDevice), "upload root");
    depths.clear();
    for (uint32_t begin = 0, end = 1; begin < end;) {
      const uint32_t next = run_depth(begin, end);
      depths.emplace_back(begin, end);
      if ((size_t)end + next > max_recs) throw std::runtime_error("device BVH build: node count out of range");
      begin = end;
      end += next;
    }
    const uint32_t nrec = depths.back().second;
    for (size_t d = depths.size(); d-- > 0;)
      node_internal<<<blocks(depths[d].second - depths[d].first), 128>>>(recs, depths[d].first, depths[d].second,
                                                                         internal);
    uint32_t root_internal = 0;
    ck(cudaMemcpy(&root_internal, internal, sizeof(uint32_t), cudaMemcpyDeviceToHost), "read the node count");
    const size_t nn = 1 + 2 * (size_t)root_internal;
    if (nn != nrec) throw std::runtime_error("device BVH build: node count disagrees");
    place_root<<<1, 1>>>(pos, pair);
    for (const auto& d : depths)
      node_place<<<blocks(d.second - d.first), 128>>>(recs, d.first, d.second, internal, pos, pair, dnodes,
                                                      (uint32_t)nn, &tot->error);
    item_order<<<blocks(n), 128>>>(items, n, order);
    ck(cudaGetLastError(), "launch");
    if (read_totals().error) throw std::runtime_error("device BVH build: inconsistent node placement");
    nodes.resize(nn);
    ck(cudaMemcpy(nodes.data(), dnodes, nn * sizeof(xb_bvh_node), cudaMemcpyDeviceToHost), "read nodes");
    order_out.resize(n);
    ck(cudaMemcpy(order_out.data(), order, (size_t)n * sizeof(uint32_t), cudaMemcpyDeviceToHost), "read order");
  }
};

}  // namespace

void build_bvh_device(const std::vector<BuildItem>& items, int bins, uint32_t max_leaf, bool leaf_cost,
                      std::vector<xb_bvh_node>& nodes, std::vector<uint32_t>& order) {
  if (bins < 2 || bins > kLevelMaxBins) throw std::invalid_argument("build_bvh_device: bins");
  if (items.size() >= (1u << 31)) throw std::invalid_argument("build_bvh_device: too many items");
  nodes.clear();
  order.clear();
  if (items.empty()) return;
  DeviceLevelBuild b;
  b.bins = bins;
  b.max_leaf = max_leaf;
  b.leaf_cost = leaf_cost;
  b.build(items, nodes, order);
}

void build_bvh_device_mesh(const HostMesh& m, int bins, uint32_t max_leaf, bool leaf_cost,
                           std::vector<xb_bvh_node>& nodes, std::vector<uint32_t>& order) {
  if (bins < 2 || bins > kLevelMaxBins) throw std::invalid_argument("build_bvh_device_mesh: bins");
  if ((size_t)m.num_triangles() >= (1u << 31)) throw std::invalid_argument("build_bvh_device_mesh: too many triangles");
  for (int32_t v : m.indices)
    if (v < 0 || v >= m.num_vertices()) throw std::invalid_argument("build_bvh_device_mesh: index out of range");
  nodes.clear();
  order.clear();
  if (m.num_triangles() == 0) return;
  DeviceLevelBuild b;
  b.bins = bins;
  b.max_leaf = max_leaf;
  b.leaf_cost = leaf_cost;
  b.build(m, nodes, order);
}

}  // namespace xb
