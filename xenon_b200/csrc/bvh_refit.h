// bvh_refit.h — BLAS refit: node boxes recomputed from moved vertices, tree topology kept.
//
// The box folds of the refit passes (refit_kernels.h), which the host (HostScene::refit_mesh)
// and the device (xb_refit_mesh in renderer.cu) both run. The folds are the build's: a box starts
// empty (+inf / -inf) and grows with std::min / std::max semantics, so the first of two equal
// values is kept (Bounds::grow in host_math.h, AABB::expand in the reference's
// src/geometry/aabb.h). A triangle's box is its three vertices folded in index order. A leaf's
// box is its triangles' boxes in slot order, which is the build's order for a leaf. An interior
// node's box is its left child's box, then its right child's.
//
// With the vertices unchanged, a refit gives the build's boxes value for value. Interior boxes
// also match bit for bit unless a coordinate extreme is reached by both +0 and -0. The build
// folds an interior node over its triangles in the order they had before that node's split,
// and the refit folds children; a zero of either sign compares equal, so the two can keep
// different signs. Traversal reads +0 and -0 alike.
#pragma once

#include <cstdint>

#ifdef __CUDACC__
#define XB_HD __host__ __device__ __forceinline__
#else
#define XB_HD inline
#endif

namespace xb {

struct RefitBox {
  float mn[3], mx[3];
};

XB_HD void refit_empty(RefitBox& b) {
  const float inf = __builtin_huge_valf();
  b.mn[0] = b.mn[1] = b.mn[2] = inf;
  b.mx[0] = b.mx[1] = b.mx[2] = -inf;
}

// min(a, b) = (b < a) ? b : a and max(a, b) = (a < b) ? b : a, as std::min / std::max
XB_HD void refit_grow(RefitBox& b, float x, float y, float z) {
  b.mn[0] = x < b.mn[0] ? x : b.mn[0];
  b.mn[1] = y < b.mn[1] ? y : b.mn[1];
  b.mn[2] = z < b.mn[2] ? z : b.mn[2];
  b.mx[0] = b.mx[0] < x ? x : b.mx[0];
  b.mx[1] = b.mx[1] < y ? y : b.mx[1];
  b.mx[2] = b.mx[2] < z ? z : b.mx[2];
}

XB_HD void refit_grow(RefitBox& b, const RefitBox& c) {
  for (int k = 0; k < 3; ++k) {
    b.mn[k] = c.mn[k] < b.mn[k] ? c.mn[k] : b.mn[k];
    b.mx[k] = b.mx[k] < c.mx[k] ? c.mx[k] : b.mx[k];
  }
}

// The box of a leaf over triangle slots [first, first + count). vertex(slot, k, xyz) writes
// vertex k of the triangle in that slot.
template <class Vertex>
XB_HD RefitBox refit_leaf(uint32_t first, uint32_t count, const Vertex& vertex) {
  RefitBox box;
  refit_empty(box);
  for (uint32_t s = first; s < first + count; ++s) {
    RefitBox tb;
    refit_empty(tb);
    for (int k = 0; k < 3; ++k) {
      float p[3];
      vertex(s, k, p);
      refit_grow(tb, p[0], p[1], p[2]);
    }
    refit_grow(box, tb);
  }
  return box;
}

XB_HD RefitBox refit_interior(const RefitBox& left, const RefitBox& right) {
  RefitBox box;
  refit_empty(box);
  refit_grow(box, left);
  refit_grow(box, right);
  return box;
}

}  // namespace xb
