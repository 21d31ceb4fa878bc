// trace_persistent.cuh — persistent-warp traversal of a ray queue with per-lane refill.
//
// A warp holds 32 rays. Each outer iteration: lanes without a ray take new ones from the queue
// (one atomic per warp for all idle lanes), then the warp steps its rays: in each step every
// lane with a ray does one unit of work — a TLAS node, an instance entry, a BLAS interior node,
// or a BLAS leaf's triangles — and a lane that finishes writes its result and becomes idle. The
// warp leaves the step loop to refill as soon as `refill` lanes are idle, so a long ray no longer
// holds finished lanes hostage (the one-ray-per-thread kernel averages 7-16 of 32 lanes active).
// An earlier form deferred the leaves to a warp-wide phase after the interior work ("while-while")
// and refilled only once every lane had a leaf pending or was done; this one was faster on every
// workload measured (config 3 renders 13.2 -> 11.3 ms per sample; trace queries 1.3-1.8x).
//
// Per ray, nodes and triangles are visited in exactly the order of the reference's recursive
// loops (tlas.cpp:172-245, blas.cpp:211-265): closest-hit results, including which of two
// equal-t triangles wins, are the reference's. Any-hit rays (kAny) only need *whether* some
// triangle lies in [tmin, tmax], which does not depend on order, so they descend nearest child
// first to find occluders sooner.
#pragma once

#include "dev_scene.cuh"

namespace xbd {

struct TraceQueue {
  const float4* ray_o;      // org xyz, w = tmin (closest) / tmax (any-hit shadow items)
  const float4* ray_d;      // dir xyz, w = tmax (closest) / bits(path) (shadow items)
  const int32_t* count;     // number of rays (device)
  int32_t* fetch;           // work cursor (device, zeroed before launch)
  // closest-hit outputs
  float4* hit;              // t, u, v, bits(prim)
  int32_t* hit_inst;
  // any-hit (shadow) outputs: unoccluded items add contrib to L[path]
  const float4* contrib;
  float4* L;
  unsigned long long* stats;
  int far_first;            // any-hit: descend into the farther child first
};

// Where a warp's rays come from and where their answers go: the renderer's queues, the rays
// taken from a shared cursor (a TraceQueue; xb_trace_rays_device has its own, in renderer.cu).
//   end()                   one past the last ray index this warp may take
//   grab(lane, leader, k)   the first of k consecutive ray indices for the warp's idle lanes
//                           (warp-uniform: every lane calls it with the same k)
//   load<kAny>(ray, o, d, tmin, tmax), finish_any(ray, occluded),
//   finish_closest(sc, ray, o, d, tmin, tmax, h), stats()
struct QueueIO {
  TraceQueue q;
  int n;
  __device__ __forceinline__ int end() const { return n; }
  __device__ __forceinline__ int grab(int lane, int leader, int k) const {
    int base = 0;
    if (lane == leader) base = atomicAdd(q.fetch, k);
    return __shfl_sync(0xffffffffu, base, leader);
  }
  template <bool kAny>
  __device__ __forceinline__ void load(int ray, V3& o, V3& d, float& tmin, float& tmax) const {
    const float4 a = q.ray_o[ray], b = q.ray_d[ray];
    o = v3(a.x, a.y, a.z);
    d = v3(b.x, b.y, b.z);
    if (kAny) { tmin = kShadowEps; tmax = a.w; }
    else { tmin = a.w; tmax = b.w; }
  }
  __device__ __forceinline__ void finish_any(int ray, bool occluded) const {
    if (occluded) return;
    const float4 c = q.contrib[ray];
    const int p = __float_as_int(q.ray_d[ray].w);
    float4 l = q.L[p];
    l.x = l.x + c.x; l.y = l.y + c.y; l.z = l.z + c.z;
    q.L[p] = l;
  }
  __device__ __forceinline__ void finish_closest(const DevScene&, int ray, V3, V3, float, float,
                                                 const HitState& h) const {
    q.hit[ray] = make_float4(h.t, h.u, h.v, __int_as_float(h.prim));
    q.hit_inst[ray] = h.inst;
  }
  __device__ __forceinline__ unsigned long long* stats() const { return q.stats; }
};

template <bool kAny, bool kCount, int kSh, class IO>
__device__ __forceinline__ void trace_persistent(const DevScene& sc, IO& io, int refill, bool far_first) {
  constexpr unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  uint32_t tstack[kStackSize];
  uint32_t bstack_local[kStackSize];
  extern __shared__ uint32_t s_stack[];
  const BStack<kSh> bstack{s_stack + threadIdx.x, bstack_local};
  TraversalCounters cnt{0, 0, 0, 0};
  bool overflow = false;

  int ray = -1;                   // queue index of this lane's ray, -1 = idle
  bool exhausted = false;         // the queue has no more rays for this warp
  V3 wo = v3s(0.f), wd = v3s(0.f), winv = v3s(0.f);
  float tmin = 0.f, tmax = kInf;
  int sign0 = 0, sign1 = 0, sign2 = 0;
  V3 lo = v3s(0.f), ld = v3s(0.f), linv = v3s(0.f);
  int tsp = 0, bsp = 0;
  uint32_t bcur = 0;              // BLAS node being expanded (a stack entry), valid if bactive
  bool bactive = false;
  int cur_inst = -1;              // instance being traversed (-1: at TLAS level)
  uint32_t tl_child = 0, tl_count = 0, tl_i = 0;   // instances of the current TLAS leaf
  HitState h{kInf, 0.f, 0.f, -1, -1};
  bool occluded = false;

  for (;;) {
    // ── refill idle lanes ──
    const unsigned idle = __ballot_sync(FULL, ray < 0);
    if (!exhausted && __popc(idle) >= refill) {
      const int leader = __ffs(idle) - 1;
      const int base = io.grab(lane, leader, __popc(idle));
      if (base >= io.end()) exhausted = true;
      if (ray < 0) {
        const int mine = base + __popc(idle & ((1u << lane) - 1u));
        if (mine < io.end()) {
          ray = mine;
          io.template load<kAny>(ray, wo, wd, tmin, tmax);
          winv = v3(1.f / wd.x, 1.f / wd.y, 1.f / wd.z);
          sign0 = wd.x < 0.f; sign1 = wd.y < 0.f; sign2 = wd.z < 0.f;
          tsp = 0; bsp = 0; bactive = false; cur_inst = -1; tl_count = 0; tl_i = 0;
          h = HitState{kInf, 0.f, 0.f, -1, -1};
          occluded = false;
          if (sc.num_tlas_nodes > 0) tstack[tsp++] = 0;
        }
      }
    }
    if (__ballot_sync(FULL, ray >= 0) == 0 && exhausted) break;

    // ── steps until enough lanes are idle to refill (or, the queue exhausted, all are) ──
    bool want = (ray >= 0);
    while (__any_sync(FULL, want)) {
      if (want) {
        if (bactive) {
          // BLAS node (blas.cpp:222-263): the near child continues in bcur, the far one is pushed
          uint32_t child, count;
          blas_unpack(sc, bcur, child, count);
          if (count > 0) {
            // the leaf's triangles (blas.cpp:224-233 / 281-287)
            float tbest = kAny ? tmax : h.t;
            for (uint32_t i = 0; i < count; ++i) {
              const float4* tp = sc.tris + 3 * (size_t)(child + i);
              const float4 a = ldg4(tp), b = ldg4(tp + 1), c = ldg4(tp + 2);
              if (kCount) cnt.tris++;
              float t, u, v;
              if (tri_hit(sc, lo, ld, linv, tmin, ld3(a), ld3(b), ld3(c), kAny ? tmax : tbest, t, u, v)) {
                if (kAny) {
                  occluded = true;
                  break;
                }
                tbest = t;
                h.t = t; h.u = u; h.v = v;
                h.prim = (int32_t)(child + i);
                h.inst = cur_inst;
              }
            }
            if (kAny && occluded) {
              bsp = 0; tsp = 0; tl_count = 0; bactive = false;
            } else if (bsp > 0) {
              bcur = bstack.get(--bsp);
            } else {
              bactive = false;
            }
          } else {
            if (kCount) cnt.nodes++;
            const float4* pp = sc.blas + 2 * (size_t)child;
            const float4 la = ldg4(pp), lb = ldg4(pp + 1), ra = ldg4(pp + 2), rb = ldg4(pp + 3);
            float tl, tr;
            const float tcull = kAny ? tmax : h.t;
            const bool hl = slab_sse(la, lb, linv, lo, tmin, tcull, tl);
            const bool hr = slab_sse(ra, rb, linv, lo, tmin, tcull, tr);
            const uint32_t el = blas_entry(__float_as_uint(lb.z), __float_as_uint(lb.w), child);
            const uint32_t er = blas_entry(__float_as_uint(rb.z), __float_as_uint(rb.w), child + 1);
            if (hl && hr) {
              if (bsp + 1 > kStackSize) {
                overflow = true;
                bactive = false; bsp = 0; tsp = 0; tl_count = 0;   // abandon (reported as overflow)
              } else if ((tl < tr) != (kAny && far_first)) {
                bstack.put(bsp++, er); bcur = el;
              } else {
                bstack.put(bsp++, el); bcur = er;
              }
            } else if (hl || hr) {
              bcur = hl ? el : er;
            } else if (bsp > 0) {
              bcur = bstack.get(--bsp);
            } else {
              bactive = false;
            }
          }
        } else if (tl_i < tl_count) {
          // enter the next instance of the current TLAS leaf (tlas.cpp:200-218)
          const int ii = (int)__ldg(sc.tlas_inst + tl_child + tl_i);
          ++tl_i;
          const DevInstance& in = sc.inst[ii];
          if (kCount) cnt.inst++;
          const Ray wr{wo, wd, tmin, tmax};
          const Ray lr = to_local(in, wr);
          if (in.kind == 0) {
            lo = lr.o; ld = lr.d;
            linv = v3(1.f / ld.x, 1.f / ld.y, 1.f / ld.z);
            cur_inst = ii;
            bcur = blas_root_entry(sc, in.root);
            bactive = true;
          } else {
            // analytic prims: a short scalar walk, done in place
            if (kAny) {
              if (pblas_any(sc, lr, bstack, overflow)) { occluded = true; bsp = 0; bactive = false; tsp = 0; tl_count = 0; }
            } else {
              pblas_closest(sc, lr, h, ii, bstack, overflow);
            }
          }
          if (kAny && occluded) want = false;
        } else if (tsp > 0) {
          // TLAS node (tlas.cpp:186-242)
          const uint32_t idx = tstack[--tsp];
          const float4 na = ldg4(sc.tlas + 2 * idx), nb = ldg4(sc.tlas + 2 * idx + 1);
          if (kCount) cnt.tlas++;
          const int sgn[3] = {sign0, sign1, sign2};
          if (aabb_fast(na, nb, winv, wo, sgn, tmin, kAny ? tmax : h.t)) {
            const uint32_t child = __float_as_uint(nb.z), count = __float_as_uint(nb.w);
            if (count > 0) {
              tl_child = child; tl_count = count; tl_i = 0;
            } else if (tsp + 2 > kStackSize) {
              overflow = true;
              tsp = 0;
            } else {
              const float ex = na.w - na.x, ey = nb.x - na.y, ez = nb.y - na.z;
              const int ax = (ex > ey && ex > ez) ? 0 : (ey > ez ? 1 : 2);
              const float4 la = ldg4(sc.tlas + 2 * child), lb = ldg4(sc.tlas + 2 * child + 1);
              const float4 ra = ldg4(sc.tlas + 2 * child + 2), rb = ldg4(sc.tlas + 2 * child + 3);
              float cl, cr;
              if (ax == 0) { cl = (la.x + la.w) * 0.5f; cr = (ra.x + ra.w) * 0.5f; }
              else if (ax == 1) { cl = (la.y + lb.x) * 0.5f; cr = (ra.y + rb.x) * 0.5f; }
              else { cl = (la.z + lb.y) * 0.5f; cr = (ra.z + rb.y) * 0.5f; }
              const float tl = (cl - comp(wo, ax)) * comp(winv, ax);
              const float tr = (cr - comp(wo, ax)) * comp(winv, ax);
              if (tl < tr) { tstack[tsp++] = child + 1; tstack[tsp++] = child; }
              else { tstack[tsp++] = child; tstack[tsp++] = child + 1; }
            }
          }
        } else {
          // ray finished
          want = false;
          if (kAny) io.finish_any(ray, occluded);
          else io.finish_closest(sc, ray, wo, wd, tmin, tmax, h);
          ray = -1;
        }
      }
      if (!exhausted && __popc(__ballot_sync(FULL, ray < 0)) >= refill) break;
    }
  }
  if (overflow) atomicAdd(io.stats() + 3, 1ull);
  if (kCount) {
    unsigned long long* dst = io.stats() + (kAny ? 12 : 8);
    atomicAdd(dst + 0, (unsigned long long)cnt.nodes);
    atomicAdd(dst + 1, (unsigned long long)cnt.tris);
    atomicAdd(dst + 2, (unsigned long long)cnt.tlas);
    atomicAdd(dst + 3, (unsigned long long)cnt.inst);
  }
}

}  // namespace xbd
