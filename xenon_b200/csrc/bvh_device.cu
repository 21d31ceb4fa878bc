// bvh_device.cu — the level-synchronous BVH build on the device (XB_BUILD_DEVICE).
//
// The passes and the depth loop are those of bvh_level_kernels.h, which the host form
// (bvh_levels.cpp, XB_BUILD_LEVELS) runs as loops, so the CPU tests of the host form run this
// build's pass code too. Here each pass is one kernel launch over its thread indices. The
// executor keeps the items and scratch in device memory, reads each depth's node outcomes back
// for the loop, and does the rare median split (std::nth_element) on the host. Node indices are
// placed on the host from subtree sizes (place_level_nodes). The build runs on the calling
// thread's current CUDA device, on the default stream; no kernel waits on another.
#include <cuda_runtime.h>

#include <algorithm>
#include <stdexcept>
#include <string>
#include <vector>

#include "bvh_build.h"
#include "bvh_level_kernels.h"

namespace xb {
namespace {

__global__ void lvl_bounds(LevelArgs a) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < a.nchunks) lvl_bounds_at(a, i);
}
__global__ void lvl_plane(LevelArgs a) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < a.ntasks) lvl_plane_at(a, i);
}
__global__ void lvl_bins(LevelArgs a) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < a.nchunks) lvl_bins_at(a, i);
}
__global__ void lvl_sah(LevelArgs a) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < a.ntasks) lvl_sah_at(a, i);
}
__global__ void lvl_pass(LevelArgs a) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < a.nchunks) lvl_pass_at(a, i);
}
__global__ void lvl_prefix(LevelArgs a) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < a.ntasks) lvl_prefix_at(a, i);
}
__global__ void lvl_rank(LevelArgs a) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < a.nchunks) lvl_rank_at(a, i);
}
__global__ void lvl_exchange(LevelArgs a) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < a.nitems) lvl_exchange_at(a, i);
}

void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess)
    throw std::runtime_error(std::string("device BVH build: ") + what + ": " + cudaGetErrorString(e));
}

// A device array that grows to the largest size asked of it and frees itself.
template <class T>
struct DevArray {
  T* p = nullptr;
  size_t cap = 0;
  DevArray() = default;
  DevArray(const DevArray&) = delete;
  DevArray& operator=(const DevArray&) = delete;
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

struct DeviceLevelExec {
  uint32_t n = 0;
  DevArray<LevelItem> items;
  DevArray<LevelTask> tasks;
  DevArray<ChunkRef> chunks;
  DevArray<NodeOut> out;
  DevArray<RefitBox> box, cbox, bins;
  DevArray<int32_t> cnt, error;
  DevArray<uint32_t> pass, before;
  DevArray<int64_t> left, right;

  void upload(const std::vector<LevelItem>& it) {
    n = (uint32_t)it.size();
    ck(cudaMemcpy(items.need(n, "items"), it.data(), (size_t)n * sizeof(LevelItem), cudaMemcpyHostToDevice),
       "upload items");
    ck(cudaMemset(left.need(n, "rank tables"), 0xff, (size_t)n * sizeof(int64_t)), "clear rank tables");
    ck(cudaMemset(right.need(n, "rank tables"), 0xff, (size_t)n * sizeof(int64_t)), "clear rank tables");
    error.need(1, "status");
  }

  void download(std::vector<LevelItem>& it) {
    ck(cudaMemcpy(it.data(), items.p, (size_t)n * sizeof(LevelItem), cudaMemcpyDeviceToHost), "read items");
  }

  void run_depth(LevelArgs& a, const std::vector<LevelTask>& t, const std::vector<ChunkRef>& c,
                 std::vector<NodeOut>& result, int32_t* err) {
    a.items = items.p;
    a.tasks = tasks.need(t.size(), "tasks");
    a.chunks = chunks.need(c.size(), "chunks");
    a.out = out.need(t.size(), "node outcomes");
    a.chunk_box = box.need(c.size(), "chunk bounds");
    a.chunk_cbox = cbox.need(c.size(), "chunk bounds");
    a.chunk_bins = bins.need(c.size() * a.bins, "chunk bins");
    a.chunk_cnt = cnt.need(c.size() * a.bins, "chunk bins");
    a.chunk_pass = pass.need(c.size(), "chunk counts");
    a.chunk_before = before.need(c.size(), "chunk counts");
    a.left_of = left.p;
    a.right_of = right.p;
    a.error = error.p;
    ck(cudaMemcpy(tasks.p, t.data(), t.size() * sizeof(LevelTask), cudaMemcpyHostToDevice), "upload tasks");
    ck(cudaMemcpy(chunks.p, c.data(), c.size() * sizeof(ChunkRef), cudaMemcpyHostToDevice), "upload chunks");
    ck(cudaMemset(error.p, 0, sizeof(int32_t)), "clear status");
    lvl_bounds<<<blocks(a.nchunks), 128>>>(a);
    lvl_plane<<<blocks(a.ntasks), 128>>>(a);
    lvl_bins<<<blocks(a.nchunks), 128>>>(a);
    lvl_sah<<<blocks(a.ntasks), 128>>>(a);
    lvl_pass<<<blocks(a.nchunks), 128>>>(a);
    lvl_prefix<<<blocks(a.ntasks), 128>>>(a);
    lvl_rank<<<blocks(a.nchunks), 128>>>(a);
    lvl_exchange<<<blocks(a.nitems), 128>>>(a);
    ck(cudaGetLastError(), "launch");
    result.resize(t.size());
    ck(cudaMemcpy(result.data(), out.p, t.size() * sizeof(NodeOut), cudaMemcpyDeviceToHost), "read outcomes");
    ck(cudaMemcpy(err, error.p, sizeof(int32_t), cudaMemcpyDeviceToHost), "read status");
  }

  void median_split(uint32_t lo, uint32_t mid, uint32_t hi, int axis) {
    std::vector<LevelItem> part(hi - lo);
    ck(cudaMemcpy(part.data(), items.p + lo, part.size() * sizeof(LevelItem), cudaMemcpyDeviceToHost),
       "read a median split");
    level_median_split(part.data(), 0, mid - lo, hi - lo, axis);
    ck(cudaMemcpy(items.p + lo, part.data(), part.size() * sizeof(LevelItem), cudaMemcpyHostToDevice),
       "write a median split");
  }
};

}  // namespace

void build_bvh_device(std::vector<BuildItem>& items, int bins, uint32_t max_leaf, bool leaf_cost,
                      std::vector<xb_bvh_node>& nodes, std::vector<uint32_t>& order) {
  if (bins < 2 || bins > kLevelMaxBins) throw std::invalid_argument("build_bvh_device: bins");
  if (items.size() >= (1u << 31)) throw std::invalid_argument("build_bvh_device: too many items");
  nodes.clear();
  order.clear();
  if (items.empty()) return;
  std::vector<LevelItem> it = to_level_items(items);
  DeviceLevelExec ex;
  ex.upload(it);
  std::vector<LevelNodeRecord> all;
  run_level_build(ex, (uint32_t)it.size(), bins, max_leaf, leaf_cost, all);
  ex.download(it);
  place_level_nodes(all, nodes);
  from_level_items(it, items, order);
}

}  // namespace xb
