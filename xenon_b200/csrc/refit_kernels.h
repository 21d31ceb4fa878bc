// refit_kernels.h — the three passes of a BLAS refit, over the renderer's packed arrays, shared
// by the device refit (xb_refit_mesh, renderer.cu: one kernel per pass) and the host refit
// (HostScene::refit_mesh: the same passes as loops over their thread indices, on one mesh packed
// the same way). The CPU tests of the host refit therefore run the device refit's pass code.
//
// Packed arrays (as xb_upload_scene lays them out):
//   blas: two quads per node, {mn.x, mn.y, mn.z, mx.x} and {mx.y, mx.z, child, count} with child
//     and count as bit patterns. An interior node (count 0) has its children at global node
//     indices child and child + 1; a leaf covers global triangle slots [child, child + count).
//   tris: three quads per triangle slot, the vertices, with the triangle's index within its mesh
//     in the first quad's w.
//   tri_index: three global vertex ids per global triangle.
// Passes:
//   1. refit_tris_at(s):    slot s takes its vertices from the new positions;
//   2. refit_parents_at(i): interior node i names itself its children's parent; arrivals = 0;
//   3. refit_nodes_at(i):   from leaf i up: the leaf's box from its triangles, then at each
//      parent the second child to arrive folds both children's boxes and goes on. The first
//      stops, so every box is written once and no thread waits for another. Run as a loop, the
//      leaves arrive in index order, and the same boxes result.
#pragma once

#include <cstdint>

#include "bvh_refit.h"

namespace xb {

struct alignas(16) Quad {
  float x, y, z, w;
};

struct RefitArgs {
  Quad* blas;
  Quad* tris;
  const int32_t* tri_index;
  const float* pos;           // the mesh's new positions, float[3 * num_verts]
  int32_t* parent;            // per node of the mesh: its parent (-1: the root); all -1 at first
  uint32_t* arrivals;         // per node of the mesh: children whose walk reached it
  int32_t* status;            // 0 ok; 1 an index out of range; 2 a walk longer than the node count
  int64_t node_base, slot_base;
  int32_t num_nodes, num_tris, num_verts, tri_offset, vtx_offset;
};

XB_HD uint32_t quad_bits(float f) {
#ifdef __CUDA_ARCH__
  return __float_as_uint(f);
#else
  union { float f; uint32_t u; } c;
  c.f = f;
  return c.u;
#endif
}

XB_HD void refit_status(int32_t* status, int32_t code) {
#ifdef __CUDA_ARCH__
  atomicExch(status, code);
#else
  *status = code;
#endif
}

// Boxes written during the walk by other threads are read and written through L2 on the device.
XB_HD RefitBox refit_load_box(const Quad* blas, int64_t n) {
#ifdef __CUDA_ARCH__
  const float4 lo = __ldcg(reinterpret_cast<const float4*>(blas) + 2 * n);
  const float4 hi = __ldcg(reinterpret_cast<const float4*>(blas) + 2 * n + 1);
#else
  const Quad lo = blas[2 * n], hi = blas[2 * n + 1];
#endif
  RefitBox b;
  b.mn[0] = lo.x; b.mn[1] = lo.y; b.mn[2] = lo.z;
  b.mx[0] = lo.w; b.mx[1] = hi.x; b.mx[2] = hi.y;
  return b;
}

XB_HD void refit_store_box(Quad* blas, int64_t n, const RefitBox& b, const Quad& hi) {
#ifdef __CUDA_ARCH__
  float4* p = reinterpret_cast<float4*>(blas) + 2 * n;
  __stcg(p, make_float4(b.mn[0], b.mn[1], b.mn[2], b.mx[0]));
  __stcg(p + 1, make_float4(b.mx[1], b.mx[2], hi.z, hi.w));
#else
  blas[2 * n] = Quad{b.mn[0], b.mn[1], b.mn[2], b.mx[0]};
  blas[2 * n + 1] = Quad{b.mx[1], b.mx[2], hi.z, hi.w};
#endif
}

// Makes this thread's stores visible to the other threads before what follows.
XB_HD void refit_fence() {
#ifdef __CUDA_ARCH__
  __threadfence();
#endif
}

XB_HD uint32_t refit_arrive(uint32_t* arrivals, int32_t node) {
#ifdef __CUDA_ARCH__
  return atomicAdd(arrivals + node, 1u);
#else
  return arrivals[node]++;
#endif
}

XB_HD void refit_tris_at(const RefitArgs& a, int32_t s) {
  Quad* T = a.tris + 3 * (a.slot_base + s);
  const int32_t t = (int32_t)quad_bits(T[0].w);   // the triangle's index within its mesh
  if (t < 0 || t >= a.num_tris) { refit_status(a.status, 1); return; }
  int32_t v[3];
  for (int k = 0; k < 3; ++k) {
    v[k] = a.tri_index[3 * (int64_t)(a.tri_offset + t) + k] - a.vtx_offset;
    if (v[k] < 0 || v[k] >= a.num_verts) { refit_status(a.status, 1); return; }
  }
  for (int k = 0; k < 3; ++k) {
    const float* p = a.pos + 3 * (int64_t)v[k];
    T[k] = Quad{p[0], p[1], p[2], T[k].w};
  }
}

XB_HD void refit_parents_at(const RefitArgs& a, int32_t i) {
  a.arrivals[i] = 0u;
  const Quad hi = a.blas[2 * (a.node_base + i) + 1];
  if (quad_bits(hi.w) != 0u) return;   // a leaf
  const int64_t c = (int64_t)quad_bits(hi.z) - a.node_base;
  if (c < 1 || c + 1 >= a.num_nodes) { refit_status(a.status, 1); return; }
  a.parent[c] = i;
  a.parent[c + 1] = i;
}

XB_HD void refit_nodes_at(const RefitArgs& a, int32_t i) {
  const Quad hi = a.blas[2 * (a.node_base + i) + 1];
  const uint32_t count = quad_bits(hi.w);
  if (count == 0u) return;
  const int64_t first = quad_bits(hi.z);
  if (first < a.slot_base || first + count > a.slot_base + a.num_tris) { refit_status(a.status, 1); return; }
  const Quad* tris = a.tris;
  auto vertex = [tris](uint32_t slot, int k, float* p) {
    const Quad q = tris[3 * (int64_t)slot + k];
    p[0] = q.x; p[1] = q.y; p[2] = q.z;
  };
  refit_store_box(a.blas, a.node_base + i, refit_leaf((uint32_t)first, count, vertex), hi);
  for (int32_t steps = 0; steps < a.num_nodes; ++steps) {
    const int32_t p = a.parent[i];
    if (p < 0) return;
    refit_fence();                                    // this child's box before its arrival
    if (refit_arrive(a.arrivals, p) != 1u) return;    // the first arrival (or a malformed third)
    refit_fence();
    const Quad ph = a.blas[2 * (a.node_base + p) + 1];
    const int64_t c = quad_bits(ph.z);
    refit_store_box(a.blas, a.node_base + p, refit_interior(refit_load_box(a.blas, c), refit_load_box(a.blas, c + 1)),
                    ph);
    i = p;
  }
  refit_status(a.status, 2);
}

}  // namespace xb
