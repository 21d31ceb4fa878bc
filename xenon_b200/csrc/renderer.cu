// renderer.cu — the B200 wavefront path tracer behind the C ABI (xb_create ... xb_destroy).
//
// One renderer owns one device, one stream and the device copy of one scene. A call to
// xb_render adds samples in waves: a wave is `spp_per_wave` consecutive sample indices of
// every pixel (wave_paths paths). Each wave runs, on the renderer's stream, with no host sync:
//
//   raygen                  camera rays into ray queue 0                (cpu_tiled.cpp:20-32)
//   for depth in [0, max_bounces):
//     extend(depth)         closest hit of queue (depth&1)              (scene.h:124, tlas.cpp:172)
//     shade(depth)          miss→sky, emitter hit + MIS, area NEE and sun NEE shadow-ray
//                           generation, Russian roulette, BSDF sampling into queue
//                           ((depth+1)&1)                               (cpu_tiled.cpp:34-217)
//     shadow(depth, area)   any hit; unoccluded → radiance += contribution (cpu_tiled.cpp:133-135)
//     shadow(depth, sun)    same for the directional-light ray       (cpu_tiled.cpp:175-184)
//   accumulate              per pixel, the wave's samples in sample order (cpu_tiled.cpp:218)
//
// Queue sizes live in device counters; every stage kernel is a persistent grid that reads
// its item count on the device, so the host never waits inside a wave. Queue appends are
// warp-aggregated (one atomic per warp). Per-path radiance is added in the CPU order:
// emission / sky of bounce d, then area NEE of d, then sun NEE of d, then bounce d+1.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/xenon_b200.h"
#include "bvh_refit.h"
#include "refit_kernels.h"
#include "capi_common.h"
#include "output_dev.h"
#include "dev_bsdf.cuh"
#include "dev_math.cuh"
#include "dev_scene.cuh"
#include "scene_host.h"
#include "trace_persistent.cuh"
#include "guide.h"
#include "guide_dev.cuh"

using namespace xbd;

namespace {

inline float u32_bits_to_f(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }
inline float i32_bits_to_f(int32_t i) { float f; std::memcpy(&f, &i, 4); return f; }

constexpr int kMaxDepth = 64;
constexpr int kMaxLanes = 4;         // waves in flight at most
constexpr int kCntStride = 8;        // counters per depth
enum {
  CNT_RAYS = 0,                      // rays in queue for this depth
  CNT_SH_AREA = 1,                   // area-light shadow items produced at this depth
  CNT_SH_SUN = 2,                    // sun shadow items produced at this depth
  CNT_FETCH_EXT = 3,                 // work-fetch cursors
  CNT_FETCH_SH_AREA = 4,
  CNT_FETCH_SH_SUN = 5,
  CNT_GUIDE = 6,                     // guided vertices deferred to the network pass
};
enum { STAT_RAYS = 0, STAT_SHADOW = 1, STAT_PATHS = 2, STAT_OVERFLOW = 3,
       STAT_OVERFLOW_AT_START = 4,  // STAT_OVERFLOW when the current render call began
       STAT_NONFINITE = 7,
       STAT_REC_DROPPED = 5,  // guiding: training records beyond the per-wave capacity
       STAT_REC_TOTAL = 6,    // guiding: training records collected
       STAT_EXT_WORK = 8,    // 4 counters: blas nodes, tris, tlas nodes, instances (closest hit)
       STAT_SH_WORK = 12,    // same for shadow rays
       STAT_COUNT = 16 };

__device__ __forceinline__ void flush_counters(unsigned long long* dst, const TraversalCounters& c) {
  atomicAdd(dst + 0, (unsigned long long)c.nodes);
  atomicAdd(dst + 1, (unsigned long long)c.tris);
  atomicAdd(dst + 2, (unsigned long long)c.tlas);
  atomicAdd(dst + 3, (unsigned long long)c.inst);
}

#define CK(call)                                                                   \
  do {                                                                             \
    cudaError_t e_ = (call);                                                       \
    if (e_ != cudaSuccess)                                                         \
      return set_err(r, XB_E_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

struct WaveBuffers {
  int64_t capacity = 0;
  float4* ray_o[2] = {nullptr, nullptr};
  float4* ray_d[2] = {nullptr, nullptr};
  float4* tp[2] = {nullptr, nullptr};     // throughput xyz, w = prev pdf (< 0: previous delta)
  uint64_t* rng[2] = {nullptr, nullptr};
  int32_t* path[2] = {nullptr, nullptr};
  float4* hit = nullptr;                  // t, u, v, bits(prim)
  int32_t* hit_inst = nullptr;
  float4* sh_o[2] = {nullptr, nullptr};   // [0] area, [1] sun: origin xyz, w = tmax
  float4* sh_d[2] = {nullptr, nullptr};   // dir xyz, w = bits(path)
  float4* sh_c[2] = {nullptr, nullptr};   // contribution xyz
  float4* L = nullptr;                    // per path radiance
  int32_t* cnt = nullptr;                 // [kMaxDepth + 1][kCntStride]
  int32_t* rec[2] = {nullptr, nullptr};   // guiding: training record of the emitting vertex
  float* ratio[2] = {nullptr, nullptr};   // guiding: importance ratio of the path
  int8_t* maxd = nullptr;                 // views: bounce limit of each path
  // guiding, two-kernel form: vertices whose direction the network pass samples (see
  // guide_sample_kernel): position + material, shading normal + path, geometric normal + ratio,
  // outgoing direction, throughput; and the PCG state
  float4* gq[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  uint64_t* gq_rng = nullptr;
};

}  // namespace

struct xb_renderer {
  xb_config cfg{};
  int min_bounces = 3, max_bounces = 8;
  cudaStream_t stream = nullptr;
  cudaStream_t stream2 = nullptr;         // shadow rays, concurrent with the next bounce's hits
  cudaEvent_t ev_shade[kMaxDepth] = {};   // bounce d's shading done (its shadow queues are full)
  cudaEvent_t ev_shadow[kMaxDepth] = {};  // bounce d's shadow rays done (path radiance final)
  // wave lanes 1 .. kMaxLanes - 1 (several waves in flight; lane 0 is the fields above): each
  // with its own queues, streams and per-bounce events
  struct ExtraLane {
    WaveBuffers wb;
    cudaStream_t s = nullptr, s2 = nullptr;
    cudaEvent_t ev_shade[kMaxDepth] = {};
    cudaEvent_t ev_shadow[kMaxDepth] = {};
  } lane_x[kMaxLanes - 1];
  int lanes_alloc = 0;                              // lanes whose queues are allocated
  cudaEvent_t lane_done[kMaxLanes] = {};            // each lane's last wave finished
  cudaEvent_t lane_acc[kMaxLanes] = {};             // each lane's last accumulation finished
  cudaEvent_t ev_stagger[kMaxLanes] = {};           // the lane's wave has shaded lane_stagger bounces
  // captured bounce loops, by lane, plain or guided, depth range and bounce limits (bounce_key)
  std::map<uint32_t, cudaGraphExec_t> bounce_graphs;
  bool graph_broken = false;                       // a capture failed: direct launches from then on
  int num_sms = 0;
  std::string err;
  // scene
  std::vector<void*> scene_mem;
  DevScene scene{};
  bool has_scene = false;
  bool scene_opaque = false;   // no delta, transmissive or subsurface material: shade_kernel<*, true>
  // framebuffer
  float4* accum = nullptr;                // FP32 per-pixel sum
  double* sum64 = nullptr;                // FP64 sum (flag)
  double* m2_64 = nullptr;                // Welford M2 (flag)
  double* mean64 = nullptr;
  int spp = 0;                            // samples in the image
  int next_sample = 1;                    // index of the next sample xb_render renders
  float* resolve_buf = nullptr;
  unsigned long long* host_ov = nullptr;  // page-locked: overflow counter now / at call start
  // asynchronous resolve: two device images, read back on their own stream
  float* resolve_async_buf[2] = {nullptr, nullptr};
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t resolved[2] = {nullptr, nullptr};   // image k written on the render stream
  cudaEvent_t copied[2] = {nullptr, nullptr};     // image k read back
  int resolve_slot = 0;
  WaveBuffers wb;
  int spp_per_wave = 1;
  unsigned long long* stats = nullptr;    // device totals
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  float last_ms = 0.f;
  int grid_ext = 0, grid_shade = 0, grid_shadow = 0, block = 128;
  int grid_pext = 0, grid_pshadow = 0;
  bool thread_per_ray = false;   // XB_FLAG_THREAD_PER_RAY: one ray per thread traversal kernels
  int refill = 8;                // persistent traversal: refill a warp when this many lanes idle
  int ext_persistent_from = 0;   // bounces >= this trace closest hits with persistent warps
  bool shadow_persistent = true;
  int occ_ext = 1, occ_pext = 1, occ_shadow = 1, occ_pshadow = 1;  // limits
  int occ_api[2] = {1, 1};   // trace_api_persistent_kernel<closest / any>
  int stack_sh = 0;             // BLAS stack entries in shared memory (tuning shared_stack)
  xb_tuning tune{};
  // profiling
  int prof_flags = 0;
  std::vector<cudaEvent_t> ev_pool;          // event pairs, reused each call
  std::vector<int> ev_stage;                 // stage of each recorded pair
  size_t ev_used = 0;
  double stage_busy_ms[6] = {0, 0, 0, 0, 0, 0};
  double stage_ms[6] = {0, 0, 0, 0, 0, 0};      // raygen, extend, shade, shadow, accumulate, train
  int64_t stage_launches[6] = {0, 0, 0, 0, 0, 0};
  // learned path guiding
  xb_guiding gcfg{};
  bool guiding = false;
  xbg::Guide* guide = nullptr;
  float gbmin[3] = {0, 0, 0}, gbinv[3] = {1, 1, 1};   // network position box
  float scene_lo[3] = {0, 0, 0}, scene_hi[3] = {1, 1, 1};
  int occ_gshade = 1, grid_gshade = 0;
  int last_loss_index = -1;
  // generic scratch for trace/bsdf helpers
  void* scratch = nullptr;
  size_t scratch_bytes = 0;
  // BLAS refit (xb_refit_mesh): where each mesh's nodes and triangles sit in the uploaded arrays,
  // what the host TLAS rebuild needs (instance transforms, root boxes) and device scratch
  struct MeshLayout {
    int64_t node_base = 0, slot_base = 0;
    int32_t num_nodes = 0, num_tris = 0, num_verts = 0, tri_offset = 0, vtx_offset = 0;
    bool has_light = false, has_normals = false;
    xb_bvh_node root{};
  };
  std::vector<MeshLayout> mesh_layout;
  std::vector<int32_t> inst_geom;
  std::vector<xb::Affine> inst_l2w;
  xb_bvh_node prim_root{};
  bool has_prim_root = false;
  int64_t tlas_cap = 0;         // nodes the device TLAS array holds
  void* refit_mem = nullptr;
  size_t refit_bytes = 0;
};

namespace {

int set_err(xb_renderer* r, int code, const char* fmt, ...) __attribute__((format(printf, 3, 4)));
int set_err(xb_renderer* r, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (r) r->err = buf;
  xb::g_last_error = buf;
  return code;
}

// ── warp-aggregated queue append ──────────────────────────────────────────────
// All 32 lanes must call it (convergent); returns the slot for lanes with pred, or -1.
__device__ __forceinline__ int warp_append(int32_t* counter, bool pred, int capacity,
                                           unsigned long long* overflow) {
  const unsigned m = __ballot_sync(0xffffffffu, pred);
  if (m == 0) return -1;
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(m) - 1;
  int base = 0;
  if (lane == leader) base = atomicAdd(counter, __popc(m));
  base = __shfl_sync(0xffffffffu, base, leader);
  if (!pred) return -1;
  const int idx = base + __popc(m & ((1u << lane) - 1u));
  if (idx >= capacity) {
    atomicAdd(overflow, 1ull);
    return -1;
  }
  return idx;
}

// ── raygen (cpu_tiled.cpp:20-32) ────────────────────────────────────────────────
struct CamDev {
  V3 eye, ll, hor, ver;
};

// Pixel of queue slot j (of npix) when slots go to 8x4 pixel tiles: the 32 slots of a warp cover
// one tile, tiles in row-major order over the part of the image they fill; the pixels of the
// right and bottom remainders (width or height not a multiple of 8 or 4) follow in scanline
// order. A bijection on [0, npix).
__device__ __forceinline__ int64_t tile_pixel(int64_t j, int W, int H) {
  const int W8 = W & ~7, H4 = H & ~3;
  const int64_t nfull = (int64_t)W8 * H4;
  if (j < nfull) {
    const int64_t t = j >> 5;
    const int r = (int)(j & 31);
    const int tpr = W8 >> 3;
    const int64_t ty = t / tpr, tx = t - ty * tpr;
    return (ty * 4 + (r >> 3)) * W + tx * 8 + (r & 7);
  }
  int64_t q = j - nfull;
  const int rw = W - W8;
  if (q < (int64_t)rw * H4) return (q / rw) * W + W8 + q % rw;
  q -= (int64_t)rw * H4;
  return (H4 + q / W) * (int64_t)W + q % W;
}

// Queue slot p holds path p's camera ray (path p: sample p / npix of pixel p % npix), or with
// tiles, path (p / npix) * npix + tile_pixel(p % npix): the same paths, the same seeds, the same
// per-pixel sums (accumulation reads the radiance by path), but each warp's rays start in one 8x4
// tile, so its camera rays and their bounce-0 shadow rays traverse more of the same nodes.
__global__ void raygen_kernel(CamDev cam, int W, int H, int spp_first, int64_t paths,
                              float4* ray_o, float4* ray_d, float4* tp, uint64_t* rng,
                              int32_t* path, float4* L, int32_t* cnt, int tiles) {
  const int64_t npix = (int64_t)W * H;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < paths;
       p += (int64_t)gridDim.x * blockDim.x) {
    const int64_t pixel = tiles ? tile_pixel(p % npix, W, H) : p % npix;
    const int64_t pid = p - p % npix + pixel;
    const int64_t s = spp_first + p / npix;
    const int x = (int)(pixel % W), y = (int)(pixel / W);
    Pcg g{pcg_seed_state((uint64_t)pixel + (uint64_t)s * 0xdeadbeefULL)};
    const float u = (float)x + g.next_float();
    const float v = (float)y + g.next_float();
    const float su = u / (float)W, sv = v / (float)H;
    V3 d = normalize(cam.ll + su * cam.hor + sv * cam.ver - cam.eye);
    ray_o[p] = make_float4(cam.eye.x, cam.eye.y, cam.eye.z, kRayEps);
    ray_d[p] = make_float4(d.x, d.y, d.z, kInf);
    tp[p] = make_float4(1.f, 1.f, 1.f, -1.f);
    rng[p] = g.state;
    path[p] = (int32_t)pid;
    L[pid] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) cnt[CNT_RAYS] = (int32_t)paths;
}

// ── extend: closest hit of the bounce's ray queue ─────────────────────────────
template <bool kCount, int kSh>
__global__ void __launch_bounds__(128) extend_kernel(DevScene sc, const float4* __restrict__ ray_o,
                                                     const float4* __restrict__ ray_d,
                                                     float4* hit, int32_t* hit_inst, int32_t* cnt,
                                                     unsigned long long* stats) {
  __shared__ int s_base[4];
  const int n = cnt[CNT_RAYS];
  uint32_t tstack[kStackSize];
  uint32_t bstack_local[kStackSize];
  extern __shared__ uint32_t s_stack[];
  const BStack<kSh> bstack{s_stack + threadIdx.x, bstack_local};
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  bool overflow = false;
  TraversalCounters tc{0, 0, 0, 0};
  for (;;) {
    if (lane == 0) s_base[warp] = atomicAdd(cnt + CNT_FETCH_EXT, 32);
    __syncwarp();
    const int base = s_base[warp];
    __syncwarp();
    if (base >= n) break;
    const int i = base + lane;
    if (i < n) {
      const float4 o = ray_o[i], d = ray_d[i];
      Ray r{v3(o.x, o.y, o.z), v3(d.x, d.y, d.z), o.w, d.w};
      HitState h;
      scene_closest<kCount>(sc, r, h, tstack, bstack, tc, overflow);
      hit[i] = make_float4(h.t, h.u, h.v, __int_as_float(h.prim));
      hit_inst[i] = h.inst;
    }
  }
  if (overflow) atomicAdd(stats + STAT_OVERFLOW, 1ull);
  if (kCount) flush_counters(stats + STAT_EXT_WORK, tc);
}

// ── shadow: any hit; unoccluded items add their contribution ──────────────────
template <bool kCount, int kSh>
__global__ void __launch_bounds__(128) shadow_kernel(DevScene sc, const float4* __restrict__ so,
                                                     const float4* __restrict__ sd,
                                                     const float4* __restrict__ scn, float4* L,
                                                     const int32_t* count, int32_t* fetch,
                                                     unsigned long long* stats, int far_first) {
  __shared__ int s_base[4];
  const int n = *count;
  uint32_t tstack[kStackSize];
  uint32_t bstack_local[kStackSize];
  extern __shared__ uint32_t s_stack[];
  const BStack<kSh> bstack{s_stack + threadIdx.x, bstack_local};
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  bool overflow = false;
  TraversalCounters tc{0, 0, 0, 0};
  for (;;) {
    if (lane == 0) s_base[warp] = atomicAdd(fetch, 32);
    __syncwarp();
    const int base = s_base[warp];
    __syncwarp();
    if (base >= n) break;
    const int i = base + lane;
    if (i < n) {
      const float4 o = so[i], d = sd[i];
      Ray r{v3(o.x, o.y, o.z), v3(d.x, d.y, d.z), kShadowEps, o.w};
      if (!scene_any<kCount>(sc, r, tstack, bstack, tc, overflow, far_first != 0)) {
        const float4 c = scn[i];
        const int p = __float_as_int(d.w);
        float4 l = L[p];
        l.x = l.x + c.x; l.y = l.y + c.y; l.z = l.z + c.z;
        L[p] = l;
      }
    }
  }
  if (overflow) atomicAdd(stats + STAT_OVERFLOW, 1ull);
  if (kCount) flush_counters(stats + STAT_SH_WORK, tc);
}

// ── persistent-warp variants (trace_persistent.cuh) ────────────────────────────
template <bool kCount, int kSh>
__global__ void __launch_bounds__(128) extend_persistent_kernel(DevScene sc, TraceQueue q, int refill) {
  QueueIO io{q, *q.count};
  trace_persistent<false, kCount, kSh>(sc, io, refill, false);
}
template <bool kCount, int kSh>
__global__ void __launch_bounds__(128) shadow_persistent_kernel(DevScene sc, TraceQueue q, int refill) {
  QueueIO io{q, *q.count};
  trace_persistent<true, kCount, kSh>(sc, io, refill, q.far_first != 0);
}

// ── shade (cpu_tiled.cpp:34-217 for one bounce) ───────────────────────────────
struct ShadeArgs {
  DevScene sc;
  const float4* ray_o; const float4* ray_d; const float4* tp; const uint64_t* rng;
  const int32_t* path;
  float4* nray_o; float4* nray_d; float4* ntp; uint64_t* nrng; int32_t* npath;
  const float4* hit; const int32_t* hit_inst;
  float4* sh_o[2]; float4* sh_d[2]; float4* sh_c[2];
  float4* L;
  int32_t* cnt;         // this depth's counters
  int32_t* cnt_next;    // next depth's counters
  int depth, min_bounces, max_bounces;
  const int8_t* path_maxd;   // per path bounce limit (views of different depths), or nullptr
  int capacity;
  unsigned long long* stats;
};

__device__ __forceinline__ V3 sky_eval(const DevScene& sc, V3 d) {
  // Environment::evaluate (src/scene/environment.h:24-36)
  V3 hz = v3(sc.sky_horizon[0], sc.sky_horizon[1], sc.sky_horizon[2]);
  if (d.y < 0.f) {
    float t = smin(-d.y, 1.f);
    return sc.sky_intensity * lerp(hz, v3(sc.sky_ground[0], sc.sky_ground[1], sc.sky_ground[2]), t);
  }
  float t = powf(d.y, sc.sky_inv_sharpness);
  return sc.sky_intensity * lerp(hz, v3(sc.sky_zenith[0], sc.sky_zenith[1], sc.sky_zenith[2]), t);
}

__device__ __forceinline__ void add_L(float4* L, int p, V3 c) {
  float4 l = L[p];
  l.x = l.x + c.x; l.y = l.y + c.y; l.z = l.z + c.z;
  L[p] = l;
}

// kOcc: the blocks of 128 threads the kernel is compiled to fit on one SM (xb_tuning
// shade_occupancy): 4 keeps every value in registers (108), 8, 12 and 16 cap them at 64, 40 and
// 32 and spill the rest to L1; the bounce is latency-bound, so more resident warps usually win.
// kOpaque: the form for scenes without delta, transmissive or subsurface materials (smaller
// code: the bounce's largest stall is the instruction cache), the same results.
template <int kOcc, bool kOpaque>
__global__ void __launch_bounds__(128, kOcc) shade_kernel(ShadeArgs a) {
  const int n = a.cnt[CNT_RAYS];
  const DevScene& sc = a.sc;
  const bool last_all = (a.depth + 1 >= a.max_bounces);
  for (int base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    const int slot = base + threadIdx.x;
    bool emit_next = false, emit_area = false, emit_sun = false;
    float4 n_o, n_d, n_tp;
    uint64_t n_rng = 0;
    int32_t pid = 0;
    float4 a_o, a_d, a_c, s_o, s_d, s_c;
    if (slot < n) {
      const float4 ro = a.ray_o[slot], rd = a.ray_d[slot], tpv = a.tp[slot];
      pid = a.path[slot];
      const bool last = a.path_maxd ? (a.depth + 1 >= (int)a.path_maxd[pid]) : last_all;
      Pcg rng{a.rng[slot]};
      const Ray ray{v3(ro.x, ro.y, ro.z), v3(rd.x, rd.y, rd.z), ro.w, rd.w};
      V3 tp = v3(tpv.x, tpv.y, tpv.z);
      const float prev_pdf = tpv.w;             // < 0: previous bounce was delta
      const float4 hv = a.hit[slot];
      const int hinst = a.hit_inst[slot];
      do {
        if (hinst < 0) {
          if (sc.sky_intensity > 0.f) add_L(a.L, pid, tp * sky_eval(sc, ray.d));
          break;
        }
        HitState h{hv.x, hv.y, hv.z, __float_as_int(hv.w), hinst};
        FullHit fh;
        complete_hit(sc, ray, h, fh);
        const DevMaterial& mat = sc.mats[fh.mat_id];
        // ── emitter hit + MIS (cpu_tiled.cpp:62-86) ──
        bool hit_light = false;
        for (int li = 0; li < sc.num_lights; ++li) {
          const DevLight& lt = sc.lights[li];
          if (__float_as_int(lt.p2.w) == fh.prim_id && __float_as_int(lt.p1.w) == fh.instance_id) {
            float mis = 1.0f;
            const float cos_l = smax(0.0f, dot(fh.geo_normal, -ray.d));
            if (cos_l > 1e-6f) {
              if (a.depth > 0 && !(prev_pdf < 0.f)) {
                const float pdf_area = (1.0f / lt.p0.w) * (1.0f / (float)sc.num_lights);
                const float dsq = h.t * h.t;
                const float pdf_sa = (pdf_area * dsq) / cos_l;
                mis = mis_power2(prev_pdf, pdf_sa);
              }
              add_L(a.L, pid, tp * v3(lt.emission.x, lt.emission.y, lt.emission.z) * mis);
            }
            hit_light = true;
            break;
          }
        }
        if (hit_light) break;
        const bool is_delta = (mat.flags & kMatDelta) != 0;
        // ── area-light NEE (cpu_tiled.cpp:89-139) ──
        if (sc.num_lights > 0 && !is_delta) {
          const float upick = rng.next_float();
          int li = (int)(upick * (float)sc.num_lights);
          li = li < 0 ? 0 : (li > sc.num_lights - 1 ? sc.num_lights - 1 : li);
          const float pick_pdf = 1.f / (float)sc.num_lights;
          const DevLight& lt = sc.lights[li];
          const float u1 = rng.next_float();
          const float u2 = rng.next_float();
          const float su1 = sqrtf(u1);
          const float b0 = 1.0f - su1;
          const float b1 = u2 * su1;
          const float b2 = 1.0f - b0 - b1;
          const V3 lp = ld3(lt.p0) * b0 + ld3(lt.p1) * b1 + ld3(lt.p2) * b2;
          const V3 ln = ld3(lt.n);
          const V3 sdir = lp - fh.pos;
          const float dsq = length_sq(sdir);
          const float dist = sqrtf(dsq);
          if (dist > 1e-6f) {
            const V3 wi = sdir / dist;
            const float cos_l = smax(0.0f, dot(ln, -wi));
            const Onb onb(fh.geo_normal);
            const V3 wo_l = onb.to_local(-ray.d);
            const V3 wi_l = onb.to_local(wi);
            if (cos_l > 1e-6f && wi_l.z > 1e-6f) {
              const V3 f = bsdf_eval<kOpaque>(wo_l, wi_l, mat);
              const float bp = bsdf_pdf<kOpaque>(wo_l, wi_l, mat);
              const float lpdf = ((1.0f / lt.p0.w) * pick_pdf) * (dsq / cos_l);
              const float mis = mis_power2(lpdf, bp);
              const float cs = wi_l.z;
              if (mis > 0.0f && lpdf > 1e-12f) {
                const V3 org = offset_origin(fh.pos, fh.geo_normal, wi, kShadowEps);
                const V3 c = tp * f * cs * (v3(lt.emission.x, lt.emission.y, lt.emission.z) / lpdf) * mis;
                a_o = make_float4(org.x, org.y, org.z, dist - kShadowEps);
                a_d = make_float4(wi.x, wi.y, wi.z, __int_as_float(pid));
                a_c = make_float4(c.x, c.y, c.z, 0.f);
                emit_area = true;
              }
            }
          }
        }
        // ── directional-light NEE (cpu_tiled.cpp:148-187) ──
        if (sc.num_suns > 0 && !is_delta) {
          const float upick = rng.next_float();
          int di = (int)(upick * (float)sc.num_suns);
          di = di < 0 ? 0 : (di > sc.num_suns - 1 ? sc.num_suns - 1 : di);
          const float dpick = 1.f / (float)sc.num_suns;
          if (dpick > 0.f) {
            const DevSun& sun = sc.suns[di];
            const V3 sdir = v3(sun.dir[0], sun.dir[1], sun.dir[2]);
            const Onb onb(fh.geo_normal);
            const V3 wo_l = onb.to_local(-ray.d);
            const V3 wi_l = onb.to_local(sdir);
            if (wi_l.z > 1e-6f) {
              const V3 f = bsdf_eval<kOpaque>(wo_l, wi_l, mat);
              const float bp = bsdf_pdf<kOpaque>(wo_l, wi_l, mat);
              const float cs = wi_l.z;
              // cpu_tiled.cpp:166-183 divides by a 1e8 "pdf" (the sun then adds ~1e-8 of its
              // light); XB_FLAG_SUN_NEE weighs the delta light by its pick probability alone,
              // with MIS weight 1 (no BSDF sample can hit a direction)
              const float lpdf = sc.sun_nee ? dpick : 1e8f * dpick;
              const float mis = sc.sun_nee ? 1.f : mis_power2(lpdf, bp);
              const V3 org = offset_origin(fh.pos, fh.geo_normal, sdir, kShadowEps);
              const V3 em = v3(sun.emission[0], sun.emission[1], sun.emission[2]);
              const V3 c = tp * f * cs * (em / lpdf) * mis;
              s_o = make_float4(org.x, org.y, org.z, kInf);
              s_d = make_float4(sdir.x, sdir.y, sdir.z, __int_as_float(pid));
              s_c = make_float4(c.x, c.y, c.z, 0.f);
              emit_sun = true;
            }
          }
        }
        if (last) break;   // the reference samples once more, but nothing of it is ever used
        // ── Russian roulette (cpu_tiled.cpp:190-194) ──
        if (a.depth >= a.min_bounces) {
          const float p = smax(0.05f, max_component(tp));
          if (rng.next_float() > p) break;
          tp = tp / p;
        }
        // ── BSDF sampling and the next ray (cpu_tiled.cpp:197-216) ──
        const Onb onb(fh.normal);
        const V3 wo_l = onb.to_local(-ray.d);
        BsdfSample s;
        if (!bsdf_sample<kOpaque>(wo_l, mat, rng, s)) break;
        if (s.delta) {
          tp = tp * s.f;
        } else {
          const float ci = fabsf(s.wi.z);
          if (s.pdf < 1e-8f || ci < 1e-8f) break;
          tp = tp * (s.f * ci / s.pdf);
        }
        const V3 wiw = onb.to_world(s.wi);
        const V3 org = offset_origin(fh.pos, fh.geo_normal, wiw, kRayEps);
        n_o = make_float4(org.x, org.y, org.z, kRayEps);
        n_d = make_float4(wiw.x, wiw.y, wiw.z, kInf);
        n_tp = make_float4(tp.x, tp.y, tp.z, s.delta ? -1.f : s.pdf);
        n_rng = rng.state;
        emit_next = true;
      } while (false);
    }
    int idx = warp_append(a.cnt_next + CNT_RAYS, emit_next, a.capacity, a.stats + STAT_OVERFLOW);
    if (idx >= 0) {
      a.nray_o[idx] = n_o; a.nray_d[idx] = n_d; a.ntp[idx] = n_tp; a.nrng[idx] = n_rng;
      a.npath[idx] = pid;
    }
    idx = warp_append(a.cnt + CNT_SH_AREA, emit_area, a.capacity, a.stats + STAT_OVERFLOW);
    if (idx >= 0) { a.sh_o[0][idx] = a_o; a.sh_d[0][idx] = a_d; a.sh_c[0][idx] = a_c; }
    idx = warp_append(a.cnt + CNT_SH_SUN, emit_sun, a.capacity, a.stats + STAT_OVERFLOW);
    if (idx >= 0) { a.sh_o[1][idx] = s_o; a.sh_d[1][idx] = s_d; a.sh_c[1][idx] = s_c; }
  }
}

// ── guided shade: one bounce with the learned proposal (no reference counterpart) ──────
// Guiding here importance-samples the plain estimator: at a guided vertex the direction comes
// from the mixture p = a q_guide + (1 - a) p_bsdf (p_bsdf the true density of bsdf_sample, see
// bsdf_density) and the
// vertex keeps everything the plain sampler would have produced for that direction (the lobe,
// its f and pdf, hence the MIS weights and the Russian-roulette throughput), while the path
// carries the importance ratio prod p_bsdf / p as a separate scalar. The expectation therefore
// equals the plain tracer's exactly, whatever the scene, and the ratio never exceeds 1 / (1 - a).
// The network runs inside the kernel: each CTA encodes its 128 vertices into shared memory,
// runs the 4 layers on the tensor cores (tcgen05, TMEM accumulators) and keeps the lobes of its
// rows in shared memory for the rest of the bounce.
struct GuideShadeArgs {
  const __nv_bfloat16* wf;   // forward weights (bf16)
  const float* master;       // FP32 parameters (biases)
  float alpha;               // probability of sampling the network (< 0: learned per vertex)
  float bmin[3], binv[3];    // position -> [0,1]^3
  const float* ratio_in;     // importance ratio of each incoming path (nullptr: 1)
  float* ratio_out;
  float* recs;               // training records (nullptr: not training)
  int32_t* rec_count;
  int rec_cap, rec_stride;
  const int32_t* rec_in;     // record of the vertex that emitted each incoming ray (or nullptr)
  int32_t* rec_out;          // same for the outgoing queue
  int* err;
  float4* gq[5];             // two-kernel form: the deferred vertices (nullptr: fused form)
  uint64_t* gq_rng;
  float sky_alpha;           // network-free form with XB_FLAG_SKY_IS: probability of the sky proposal
  float ratio_cap;           // bound on the path's importance ratio (<= 0: none)
};

// The probability of sampling the proposal at a vertex whose path carries `ratio`: at most
// 1 - ratio / cap, so that the worst case of the vertex's factor p_bsdf / p = 1 / (1 - a) keeps
// the path's ratio within the cap. It depends on the path's prefix only, so the estimator stays
// unbiased; a path at or above the cap samples its BSDF alone.
__device__ __forceinline__ float capped_selection(float a, float ratio, float cap) {
  return cap > 0.f ? fminf(a, fmaxf(0.f, 1.f - ratio / cap)) : a;
}

constexpr float kNaN = __builtin_nanf("");
constexpr int kLobStride = xbg::kLobeFloats + 1;   // conflict-free per-thread rows
// The lobes of a tile's rows take the activation tile's place once its last layer has run.
constexpr size_t kLobBytes = (size_t)xbg::kTile * kLobStride * 4;
constexpr size_t kGuidedShadeSmem =
    xbg::kFwdWeightBytes + (kLobBytes > xbg::kTileBytes ? kLobBytes : xbg::kTileBytes) + 1024;

// 128 registers and 55 KB of shared memory: four CTAs (16 warps) per SM (kOcc applies to the
// network-free form only, as for shade_kernel). kNet = false is the
// same bounce past the bounces the network serves (xb_guiding.guided_bounces): every vertex
// samples its BSDF, the importance ratio of the path's earlier guided vertices is carried on, and
// there is no network, shared memory or barrier, so it launches like the plain bounce.
template <bool kNet, int kOcc>
__global__ void __launch_bounds__(128, kNet ? 4 : kOcc) guided_shade_kernel(ShadeArgs a, GuideShadeArgs g) {
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t* sW = smem;
  uint8_t* sA = smem + xbg::kFwdWeightBytes;
  float* sLob = reinterpret_cast<float*>(sA);
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmem_slot;
  __shared__ float sBias[xbg::kBiasFloats];
  const int n = a.cnt[CNT_RAYS];
  if ((int)blockIdx.x * 128 >= n) return;
  const DevScene& sc = a.sc;
  const bool last_all = (a.depth + 1 >= a.max_bounces);
  const bool training = g.recs != nullptr;
  if constexpr (kNet) {
    xbg::load_forward_weights(sW, sBias, g.wf, g.master);
    xbg::mma_setup(&tmem_slot, &mbar);
  }
  xbg::Mma m{tmem_slot, &mbar, 0u, g.err, true};
  float* lob = sLob + threadIdx.x * kLobStride;
  for (int base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    const int slot = base + threadIdx.x;
    bool emit_next = false, emit_area = false, emit_sun = false, emit_rec = false, emit_defer = false;
    float4 n_o, n_d, n_tp;
    uint64_t n_rng = 0;
    int32_t pid = 0;
    float n_ratio = 1.f;
    float4 a_o, a_d, a_c, s_o, s_d, s_c;
    float4 rec[6];
    float4 dq[5];
    // ── phase 1: emitter test and the network's input ──
    bool alive = false, guided = false;
    float feat[9] = {0.5f, 0.5f, 0.5f, 0.f, 0.f, 1.f, 0.f, 0.f, 1.f};
    float4 ro = make_float4(0, 0, 0, 0), rd = ro, tpv = ro;
    float ratio = 1.f;
    Pcg rng{0};
    FullHit fh;
    fh.mat_id = 0;
    if (slot < n) {
      ro = a.ray_o[slot]; rd = a.ray_d[slot]; tpv = a.tp[slot];
      pid = a.path[slot];
      rng.state = a.rng[slot];
      if (g.ratio_in) ratio = g.ratio_in[slot];
      if (g.rec_in) {
        const int ri = g.rec_in[slot];
        if (ri >= 0) {   // path radiance before the continuation of the record's vertex
          const float4 l = a.L[pid];
          float* R = g.recs + (size_t)ri * xbg::kRecFloats;
          R[17] = l.x; R[18] = l.y; R[19] = l.z;
        }
      }
      const Ray ray{v3(ro.x, ro.y, ro.z), v3(rd.x, rd.y, rd.z), ro.w, rd.w};
      const V3 tpr = v3(tpv.x, tpv.y, tpv.z) * ratio;   // the path's actual throughput
      const float4 hv = a.hit[slot];
      const int hinst = a.hit_inst[slot];
      if (hinst < 0) {
        if (sc.sky_intensity > 0.f) add_L(a.L, pid, tpr * sky_eval(sc, ray.d));
      } else {
        HitState h{hv.x, hv.y, hv.z, __float_as_int(hv.w), hinst};
        complete_hit(sc, ray, h, fh);
        bool hit_light = false;
        for (int li = 0; li < sc.num_lights; ++li) {
          const DevLight& lt = sc.lights[li];
          if (__float_as_int(lt.p2.w) == fh.prim_id && __float_as_int(lt.p1.w) == fh.instance_id) {
            float mis = 1.0f;
            const float cos_l = smax(0.0f, dot(fh.geo_normal, -ray.d));
            if (cos_l > 1e-6f) {
              if (a.depth > 0 && !(tpv.w < 0.f)) {
                const float pdf_area = (1.0f / lt.p0.w) * (1.0f / (float)sc.num_lights);
                const float pdf_sa = (pdf_area * (h.t * h.t)) / cos_l;
                mis = mis_power2(tpv.w, pdf_sa);
              }
              add_L(a.L, pid, tpr * v3(lt.emission.x, lt.emission.y, lt.emission.z) * mis);
            }
            hit_light = true;
            break;
          }
        }
        if (!hit_light) {
          alive = true;
          // The network proposes at non-delta, non-transmissive vertices seen from the front of
          // the shading normal, where the density of bsdf_sample is known (bsdf_density);
          // elsewhere the plain sampler runs. Rough dielectrics stay plain: the reference
          // evaluates their transmission with a half vector (wo + wi / ior) other than the one
          // its sampler refracts about (and its pdf can be NaN there), so neither its pdf nor a
          // corrected form of it is the density of what its sampler returns.
          // The sky proposal (network-free form with XB_FLAG_SKY_IS) serves broad lobes only:
          // a glossy conductor's lobe is rarely reached by a sky direction, so half of its
          // samples would be lost and the other half carry twice the weight.
          const DevMaterial& gm = sc.mats[fh.mat_id];
          const uint32_t mf = gm.flags;
          const bool proposal = kNet || g.gq[0] != nullptr ||
                                (g.sky_alpha > 0.f && (!(mf & kMatConductor) || gm.alpha >= 0.25f));
          guided = proposal && (mf & (kMatDelta | kMatTransmissive)) == 0 && dot(fh.normal, -ray.d) > 0.f;
          for (int k = 0; k < 3; ++k) {
            const float pk = (k == 0 ? fh.pos.x : k == 1 ? fh.pos.y : fh.pos.z);
            feat[k] = fminf(fmaxf((pk - g.bmin[k]) * g.binv[k], 0.f), 1.f);
          }
          feat[3] = fh.normal.x; feat[4] = fh.normal.y; feat[5] = fh.normal.z;
          feat[6] = -ray.d.x; feat[7] = -ray.d.y; feat[8] = -ray.d.z;
        }
      }
    }
    // ── the network on this CTA's 128 vertices ──
    float alpha = 0.f;
    if constexpr (kNet) {
      __syncthreads();   // the previous tile's lobes, in the same shared memory, are all read
      xbg::encode_row<true>(feat, sA, threadIdx.x);
      float raw[xbg::kOut];
      xbg::forward_tile(m, sA, sW, sBias, raw);
      if (!m.ok) break;   // uniform: every thread saw the same failed wait
      // every thread is past the last layer's completion: the activation tile is free
      xbg::raw_to_lobes<true>(raw, lob);
      alpha = g.alpha >= 0.f ? g.alpha : xbg::selection<true>(raw);
    }
    // ── phase 2: NEE, roulette, the next direction (cpu_tiled.cpp:89-216) ──
    if (alive) do {
      const Ray ray{v3(ro.x, ro.y, ro.z), v3(rd.x, rd.y, rd.z), ro.w, rd.w};
      V3 tp = v3(tpv.x, tpv.y, tpv.z);   // the plain estimator's throughput
      const DevMaterial& mat = sc.mats[fh.mat_id];
      const bool is_delta = (mat.flags & kMatDelta) != 0;
      if (sc.num_lights > 0 && !is_delta) {
        const float upick = rng.next_float();
        int li = (int)(upick * (float)sc.num_lights);
        li = li < 0 ? 0 : (li > sc.num_lights - 1 ? sc.num_lights - 1 : li);
        const float pick_pdf = 1.f / (float)sc.num_lights;
        const DevLight& lt = sc.lights[li];
        const float u1 = rng.next_float();
        const float u2 = rng.next_float();
        const float su1 = sqrtf(u1);
        const float b0 = 1.0f - su1;
        const float b1 = u2 * su1;
        const float b2 = 1.0f - b0 - b1;
        const V3 lp = ld3(lt.p0) * b0 + ld3(lt.p1) * b1 + ld3(lt.p2) * b2;
        const V3 sdir = lp - fh.pos;
        const float dsq = length_sq(sdir);
        const float dist = sqrtf(dsq);
        if (dist > 1e-6f) {
          const V3 wi = sdir / dist;
          const float cos_l = smax(0.0f, dot(ld3(lt.n), -wi));
          const Onb onb(fh.geo_normal);
          const V3 wo_l = onb.to_local(-ray.d);
          const V3 wi_l = onb.to_local(wi);
          if (cos_l > 1e-6f && wi_l.z > 1e-6f) {
            const V3 f = bsdf_eval(wo_l, wi_l, mat);
            const float bp = bsdf_pdf(wo_l, wi_l, mat);
            const float lpdf = ((1.0f / lt.p0.w) * pick_pdf) * (dsq / cos_l);
            const float mis = mis_power2(lpdf, bp);
            if (mis > 0.0f && lpdf > 1e-12f) {
              const V3 org = offset_origin(fh.pos, fh.geo_normal, wi, kShadowEps);
              const V3 c = (tp * ratio) * f * wi_l.z * (v3(lt.emission.x, lt.emission.y, lt.emission.z) / lpdf) * mis;
              a_o = make_float4(org.x, org.y, org.z, dist - kShadowEps);
              a_d = make_float4(wi.x, wi.y, wi.z, __int_as_float(pid));
              a_c = make_float4(c.x, c.y, c.z, 0.f);
              emit_area = true;
            }
          }
        }
      }
      if (sc.num_suns > 0 && !is_delta) {
        const float upick = rng.next_float();
        int di = (int)(upick * (float)sc.num_suns);
        di = di < 0 ? 0 : (di > sc.num_suns - 1 ? sc.num_suns - 1 : di);
        const float dpick = 1.f / (float)sc.num_suns;
        const DevSun& sun = sc.suns[di];
        const V3 sdir = v3(sun.dir[0], sun.dir[1], sun.dir[2]);
        const Onb onb(fh.geo_normal);
        const V3 wo_l = onb.to_local(-ray.d);
        const V3 wi_l = onb.to_local(sdir);
        if (wi_l.z > 1e-6f) {
          const V3 f = bsdf_eval(wo_l, wi_l, mat);
          const float bp = bsdf_pdf(wo_l, wi_l, mat);
          const float lpdf = sc.sun_nee ? dpick : 1e8f * dpick;   // as in shade_kernel
          const float mis = sc.sun_nee ? 1.f : mis_power2(lpdf, bp);
          const V3 org = offset_origin(fh.pos, fh.geo_normal, sdir, kShadowEps);
          const V3 em = v3(sun.emission[0], sun.emission[1], sun.emission[2]);
          const V3 c = (tp * ratio) * f * wi_l.z * (em / lpdf) * mis;
          s_o = make_float4(org.x, org.y, org.z, kInf);
          s_d = make_float4(sdir.x, sdir.y, sdir.z, __int_as_float(pid));
          s_c = make_float4(c.x, c.y, c.z, 0.f);
          emit_sun = true;
        }
      }
      if (a.path_maxd ? (a.depth + 1 >= (int)a.path_maxd[pid]) : last_all) break;
      if (a.depth >= a.min_bounces) {
        // cpu_tiled.cpp:190-194 on the plain throughput: p = max(0.05, max(tp)), survive with
        // min(1, p), divide by p. Its part above 1 is a deterministic rescale and stays as is;
        // the survival draw is made with the probability the actual throughput (tp * ratio)
        // asks for, and the ratio of the two survival probabilities joins the importance ratio.
        const float p = smax(0.05f, max_component(tp));
        const float surv = smin(1.f, p);
        const float surv_g = sclamp(max_component(tp * ratio) / smax(1.f, p), 0.05f, 1.f);
        if (rng.next_float() > surv_g) break;
        tp = tp / p;
        ratio = ratio * (surv / surv_g);
      }
      if (!kNet && guided && g.gq[0] != nullptr) {
        // two-kernel form: the network pass samples this vertex's direction
        dq[0] = make_float4(fh.pos.x, fh.pos.y, fh.pos.z, __int_as_float(fh.mat_id));
        dq[1] = make_float4(fh.normal.x, fh.normal.y, fh.normal.z, __int_as_float(pid));
        dq[2] = make_float4(fh.geo_normal.x, fh.geo_normal.y, fh.geo_normal.z, ratio);
        dq[3] = make_float4(-ray.d.x, -ray.d.y, -ray.d.z, 0.f);
        dq[4] = make_float4(tp.x, tp.y, tp.z, 0.f);
        n_rng = rng.state;
        emit_defer = true;
        break;
      }
      const Onb onb(fh.normal);
      const V3 wo_l = onb.to_local(-ray.d);
      BsdfSample s;
      V3 wiw;
      n_ratio = ratio;
      if (!guided) {
        if (!bsdf_sample(wo_l, mat, rng, s)) break;
        wiw = onb.to_world(s.wi);
      } else {
        // the proposal: the network's mixture (kNet) or the sky's luminance distribution
        float pb;
        const float ap = capped_selection(kNet ? alpha : g.sky_alpha, ratio, g.ratio_cap);
        if (rng.next_float() < ap) {
          if constexpr (kNet) {
            const float u0 = rng.next_float(), u1 = rng.next_float(), u2 = rng.next_float();
            float d[3];
            xbg::mix_sample(lob, u0, u1, u2, d);
            wiw = v3(d[0], d[1], d[2]);
          } else {
            const float u0 = rng.next_float(), u1 = rng.next_float();
            wiw = sky_sample(sc.sky_cdf, u0, u1);
          }
          s.wi = onb.to_local(wiw);
          s.delta = false;
          if (!bsdf_lobe_for_direction(wo_l, s.wi, mat, rng.next_float(), s.f, s.pdf, pb)) break;
        } else {
          if (!bsdf_sample(wo_l, mat, rng, s)) break;
          wiw = onb.to_world(s.wi);
          pb = bsdf_density(wo_l, s.wi, mat);
        }
        const float q = kNet ? xbg::mix_pdf(lob, wiw.x, wiw.y, wiw.z) : sky_pdf(sc.sky_cdf, wiw);
        const float pm = ap * q + (1.f - ap) * pb;
        if (!(pm > 0.f)) break;
        n_ratio = ratio * (pb / pm);
        if (training && (pid % g.rec_stride) == 0) {
          const V3 tb = tp * ratio;   // actual throughput before the vertex's scattering
          rec[0] = make_float4(feat[0], feat[1], feat[2], feat[3]);
          rec[1] = make_float4(feat[4], feat[5], feat[6], feat[7]);
          rec[2] = make_float4(feat[8], wiw.x, wiw.y, wiw.z);
          rec[3] = make_float4(0.f, __int_as_float(pid), tb.x, tb.y);
          rec[4] = make_float4(tb.z, kNaN, kNaN, kNaN);   // baseline: set by the next bounce
          rec[5] = make_float4(pb, 0.f, 0.f, 0.f);
          emit_rec = true;
        }
      }
      // cpu_tiled.cpp:197-216
      if (s.delta) {
        tp = tp * s.f;
      } else {
        const float ci = fabsf(s.wi.z);
        if (s.pdf < 1e-8f || ci < 1e-8f) { emit_rec = false; break; }
        tp = tp * (s.f * ci / s.pdf);
      }
      const V3 org = offset_origin(fh.pos, fh.geo_normal, wiw, kRayEps);
      n_o = make_float4(org.x, org.y, org.z, kRayEps);
      n_d = make_float4(wiw.x, wiw.y, wiw.z, kInf);
      n_tp = make_float4(tp.x, tp.y, tp.z, s.delta ? -1.f : s.pdf);
      n_rng = rng.state;
      emit_next = true;
    } while (false);
    if (!emit_next) emit_rec = false;
    if constexpr (!kNet) {
      const int gi = warp_append(a.cnt + CNT_GUIDE, emit_defer, a.capacity, a.stats + STAT_OVERFLOW);
      if (gi >= 0) {
        for (int k = 0; k < 5; ++k) g.gq[k][gi] = dq[k];
        g.gq_rng[gi] = n_rng;
      }
    }
    int ridx = -1;
    if (training) {
      ridx = warp_append(g.rec_count, emit_rec, g.rec_cap, a.stats + STAT_REC_DROPPED);
      if (ridx >= 0) {
        float4* R = reinterpret_cast<float4*>(g.recs + (size_t)ridx * xbg::kRecFloats);
        for (int i = 0; i < 6; ++i) R[i] = rec[i];
      }
    }
    int idx = warp_append(a.cnt_next + CNT_RAYS, emit_next, a.capacity, a.stats + STAT_OVERFLOW);
    if (idx >= 0) {
      a.nray_o[idx] = n_o; a.nray_d[idx] = n_d; a.ntp[idx] = n_tp; a.nrng[idx] = n_rng;
      a.npath[idx] = pid;
      g.ratio_out[idx] = n_ratio;
      if (g.rec_out) g.rec_out[idx] = ridx;
    }
    idx = warp_append(a.cnt + CNT_SH_AREA, emit_area, a.capacity, a.stats + STAT_OVERFLOW);
    if (idx >= 0) { a.sh_o[0][idx] = a_o; a.sh_d[0][idx] = a_d; a.sh_c[0][idx] = a_c; }
    idx = warp_append(a.cnt + CNT_SH_SUN, emit_sun, a.capacity, a.stats + STAT_OVERFLOW);
    if (idx >= 0) { a.sh_o[1][idx] = s_o; a.sh_d[1][idx] = s_d; a.sh_c[1][idx] = s_c; }
  }
  if constexpr (kNet) xbg::mma_teardown(m.tmem);
}

// ── guided directions, two-kernel form: the network pass over the deferred vertices ───────
// Given a guide queue, the bounce kernel (guided_shade_kernel<false, *>) does all of a bounce but
// the next direction of the guided vertices, which it queues with their state after next-event
// estimation and roulette. This persistent kernel runs the network on dense 128-vertex tiles of
// that queue and samples each direction as the fused kernel does: the same draws from the same
// PCG state, the same proposal, importance ratio and records — and a row's network output does
// not depend on the rest of its tile — so the two forms render the same image. The bounce
// kernel then launches like the plain bounce (no barriers or network state), beside the other
// wave lanes' kernels.
__global__ void __launch_bounds__(128, 4) guide_sample_kernel(ShadeArgs a, GuideShadeArgs g) {
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t* sW = smem;
  uint8_t* sA = smem + xbg::kFwdWeightBytes;
  float* sLob = reinterpret_cast<float*>(sA);
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmem_slot;
  __shared__ float sBias[xbg::kBiasFloats];
  const int n = a.cnt[CNT_GUIDE];
  if ((int)blockIdx.x * 128 >= n) return;
  const DevScene& sc = a.sc;
  const bool training = g.recs != nullptr;
  xbg::load_forward_weights(sW, sBias, g.wf, g.master);
  xbg::mma_setup(&tmem_slot, &mbar);
  xbg::Mma m{tmem_slot, &mbar, 0u, g.err, true};
  float* lob = sLob + threadIdx.x * kLobStride;
  for (int base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    const int slot = base + threadIdx.x;
    const bool valid = slot < n;
    float4 q[5];
    for (int k = 0; k < 5; ++k) q[k] = make_float4(0.f, 0.f, 0.f, 0.f);
    Pcg rng{0};
    float feat[9] = {0.5f, 0.5f, 0.5f, 0.f, 0.f, 1.f, 0.f, 0.f, 1.f};
    if (valid) {
      for (int k = 0; k < 5; ++k) q[k] = g.gq[k][slot];
      rng.state = g.gq_rng[slot];
      feat[0] = fminf(fmaxf((q[0].x - g.bmin[0]) * g.binv[0], 0.f), 1.f);
      feat[1] = fminf(fmaxf((q[0].y - g.bmin[1]) * g.binv[1], 0.f), 1.f);
      feat[2] = fminf(fmaxf((q[0].z - g.bmin[2]) * g.binv[2], 0.f), 1.f);
      feat[3] = q[1].x; feat[4] = q[1].y; feat[5] = q[1].z;
      feat[6] = q[3].x; feat[7] = q[3].y; feat[8] = q[3].z;
    }
    __syncthreads();   // the previous tile's lobes, in the same shared memory, are all read
    xbg::encode_row<true>(feat, sA, threadIdx.x);
    float alpha;
    {
      float raw[xbg::kOut];
      xbg::forward_tile(m, sA, sW, sBias, raw);
      if (!m.ok) break;   // uniform: every thread saw the same failed wait
      xbg::raw_to_lobes<true>(raw, lob);
      alpha = g.alpha >= 0.f ? g.alpha : xbg::selection<true>(raw);
    }
    bool emit_next = false, emit_rec = false;
    float4 n_o, n_d, n_tp;
    float4 rec[6];
    uint64_t n_rng = 0;
    float n_ratio = 1.f;
    const int32_t pid = __float_as_int(q[1].w);
    if (valid) do {
      const DevMaterial& mat = sc.mats[__float_as_int(q[0].w)];
      const V3 pos = v3(q[0].x, q[0].y, q[0].z), gn = v3(q[2].x, q[2].y, q[2].z);
      const float ratio = q[2].w;
      V3 tp = v3(q[4].x, q[4].y, q[4].z);
      const Onb onb(v3(q[1].x, q[1].y, q[1].z));
      const V3 wo_l = onb.to_local(v3(q[3].x, q[3].y, q[3].z));
      BsdfSample s;
      V3 wiw;
      float pb;
      const float ap = capped_selection(alpha, ratio, g.ratio_cap);
      if (rng.next_float() < ap) {
        const float u0 = rng.next_float(), u1 = rng.next_float(), u2 = rng.next_float();
        float d[3];
        xbg::mix_sample(lob, u0, u1, u2, d);
        wiw = v3(d[0], d[1], d[2]);
        s.wi = onb.to_local(wiw);
        s.delta = false;
        if (!bsdf_lobe_for_direction(wo_l, s.wi, mat, rng.next_float(), s.f, s.pdf, pb)) break;
      } else {
        if (!bsdf_sample(wo_l, mat, rng, s)) break;
        wiw = onb.to_world(s.wi);
        pb = bsdf_density(wo_l, s.wi, mat);
      }
      const float pm = ap * xbg::mix_pdf(lob, wiw.x, wiw.y, wiw.z) + (1.f - ap) * pb;
      if (!(pm > 0.f)) break;
      n_ratio = ratio * (pb / pm);
      if (training && (pid % g.rec_stride) == 0) {
        const V3 tb = tp * ratio;   // actual throughput before the vertex's scattering
        rec[0] = make_float4(feat[0], feat[1], feat[2], feat[3]);
        rec[1] = make_float4(feat[4], feat[5], feat[6], feat[7]);
        rec[2] = make_float4(feat[8], wiw.x, wiw.y, wiw.z);
        rec[3] = make_float4(0.f, __int_as_float(pid), tb.x, tb.y);
        rec[4] = make_float4(tb.z, kNaN, kNaN, kNaN);   // baseline: set by the next bounce
        rec[5] = make_float4(pb, 0.f, 0.f, 0.f);
        emit_rec = true;
      }
      // cpu_tiled.cpp:197-216 (the guided lobes are never delta)
      const float ci = fabsf(s.wi.z);
      if (s.pdf < 1e-8f || ci < 1e-8f) { emit_rec = false; break; }
      tp = tp * (s.f * ci / s.pdf);
      const V3 org = offset_origin(pos, gn, wiw, kRayEps);
      n_o = make_float4(org.x, org.y, org.z, kRayEps);
      n_d = make_float4(wiw.x, wiw.y, wiw.z, kInf);
      n_tp = make_float4(tp.x, tp.y, tp.z, s.pdf);
      n_rng = rng.state;
      emit_next = true;
    } while (false);
    if (!emit_next) emit_rec = false;
    int ridx = -1;
    if (training) {
      ridx = warp_append(g.rec_count, emit_rec, g.rec_cap, a.stats + STAT_REC_DROPPED);
      if (ridx >= 0) {
        float4* R = reinterpret_cast<float4*>(g.recs + (size_t)ridx * xbg::kRecFloats);
        for (int i = 0; i < 6; ++i) R[i] = rec[i];
      }
    }
    const int idx = warp_append(a.cnt_next + CNT_RAYS, emit_next, a.capacity, a.stats + STAT_OVERFLOW);
    if (idx >= 0) {
      a.nray_o[idx] = n_o; a.nray_d[idx] = n_d; a.ntp[idx] = n_tp; a.nrng[idx] = n_rng;
      a.npath[idx] = pid;
      g.ratio_out[idx] = n_ratio;
      if (g.rec_out) g.rec_out[idx] = ridx;
    }
  }
  xbg::mma_teardown(m.tmem);
}

// ── many views: raygen and accumulation over a table of pieces ────────────────────
constexpr int kMaxPieces = 64;
struct ViewPiece {
  CamDev cam;
  int W, H;
  int s_first, spp;        // 1-based first sample index, samples of every pixel in this wave
  int max_bounces;         // the view's bounce limit
  int64_t path_off;        // first path of the piece in the wave
  int64_t pix_off;         // first pixel of the piece in the wave's pixel list
  int64_t accum_off;       // first pixel of the view in the accumulation buffer
};
struct ViewPieces {
  int n;
  ViewPiece p[kMaxPieces];
};

__global__ void raygen_views_kernel(ViewPieces pk, int64_t paths, float4* ray_o, float4* ray_d, float4* tp,
                                    uint64_t* rng, int32_t* path, float4* L, int8_t* maxd, int32_t* cnt, int tiles) {
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < paths;
       p += (int64_t)gridDim.x * blockDim.x) {
    int i = 0;
    while (i + 1 < pk.n && p >= pk.p[i + 1].path_off) ++i;
    const ViewPiece& v = pk.p[i];
    const int64_t npix = (int64_t)v.W * v.H;
    const int64_t local = p - v.path_off;
    // a piece holds whole samples of its view: slots map to pixels as in raygen_kernel
    const int64_t pixel = tiles ? tile_pixel(local % npix, v.W, v.H) : local % npix;
    const int64_t pid = p - local % npix + pixel;
    const int64_t s = v.s_first + local / npix;
    const int x = (int)(pixel % v.W), y = (int)(pixel / v.W);
    // cpu_tiled.cpp:20-32, as raygen_kernel
    Pcg g{pcg_seed_state((uint64_t)pixel + (uint64_t)s * 0xdeadbeefULL)};
    const float u = (float)x + g.next_float();
    const float vv = (float)y + g.next_float();
    const float su = u / (float)v.W, sv = vv / (float)v.H;
    const V3 d = normalize(v.cam.ll + su * v.cam.hor + sv * v.cam.ver - v.cam.eye);
    ray_o[p] = make_float4(v.cam.eye.x, v.cam.eye.y, v.cam.eye.z, kRayEps);
    ray_d[p] = make_float4(d.x, d.y, d.z, kInf);
    tp[p] = make_float4(1.f, 1.f, 1.f, -1.f);
    rng[p] = g.state;
    path[p] = (int32_t)pid;
    L[pid] = make_float4(0.f, 0.f, 0.f, 0.f);
    maxd[pid] = (int8_t)v.max_bounces;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) cnt[CNT_RAYS] = (int32_t)paths;
}

// Adds every piece's samples, in sample order, to its view's FP32 sums (NaN guard as the
// single-view accumulation); counts the wave's rays.
__global__ void accumulate_views_kernel(const float4* L, ViewPieces pk, int64_t pix_total, float4* accum,
                                        const int32_t* cnt, int max_depth, int64_t paths,
                                        unsigned long long* stats) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < pix_total;
       q += (int64_t)gridDim.x * blockDim.x) {
    int i = 0;
    while (i + 1 < pk.n && q >= pk.p[i + 1].pix_off) ++i;
    const ViewPiece& v = pk.p[i];
    const int64_t npix = (int64_t)v.W * v.H;
    const int64_t pixel = q - v.pix_off;
    float4 acc = accum[v.accum_off + pixel];
    for (int k = 0; k < v.spp; ++k) {
      const float4 l = L[v.path_off + (int64_t)k * npix + pixel];
      if (!(isfinite(l.x) && isfinite(l.y) && isfinite(l.z))) {
        atomicAdd(stats + STAT_NONFINITE, 1ull);
        continue;
      }
      acc.x = acc.x + l.x; acc.y = acc.y + l.y; acc.z = acc.z + l.z;
    }
    accum[v.accum_off + pixel] = acc;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    unsigned long long rays = 0, sh = 0;
    for (int d = 0; d < max_depth; ++d) {
      rays += (unsigned long long)cnt[d * kCntStride + CNT_RAYS];
      sh += (unsigned long long)cnt[d * kCntStride + CNT_SH_AREA] +
            (unsigned long long)cnt[d * kCntStride + CNT_SH_SUN];
    }
    atomicAdd(stats + STAT_RAYS, rays);
    atomicAdd(stats + STAT_SHADOW, sh);
    atomicAdd(stats + STAT_PATHS, (unsigned long long)paths);
  }
}

// Mean of one view's sums, top-down rows (cpu_tiled.cpp:224-236).
__global__ void resolve_view_kernel(const float4* accum, int W, int H, float inv_spp, float* out) {
  const int64_t npix = (int64_t)W * H;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < npix;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(i % W), y = (int)(i / W);
    const float4 a = accum[i];
    const int64_t d = ((int64_t)(H - 1 - y) * W + x) * 3;
    out[d] = a.x * inv_spp;
    out[d + 1] = a.y * inv_spp;
    out[d + 2] = a.z * inv_spp;
  }
}

__global__ void snapshot_kernel(unsigned long long* stats) {
  if (threadIdx.x == 0) stats[STAT_OVERFLOW_AT_START] = stats[STAT_OVERFLOW];
}

// ── accumulate the wave into the framebuffer, in sample order ──────────────────
__global__ void accumulate_kernel(const float4* L, int64_t npix, int spw, int spp_before,
                                  float4* accum, double* sum64, double* m2_64, double* mean64,
                                  const int32_t* cnt, int max_depth, int64_t paths,
                                  unsigned long long* stats) {
  for (int64_t px = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; px < npix;
       px += (int64_t)gridDim.x * blockDim.x) {
    float4 acc = accum[px];
    double s0 = 0, s1 = 0, s2 = 0, m0 = 0, m1 = 0, m2 = 0, mu0 = 0, mu1 = 0, mu2 = 0;
    if (sum64) {
      s0 = sum64[3 * px]; s1 = sum64[3 * px + 1]; s2 = sum64[3 * px + 2];
      m0 = m2_64[3 * px]; m1 = m2_64[3 * px + 1]; m2 = m2_64[3 * px + 2];
      mu0 = mean64[3 * px]; mu1 = mean64[3 * px + 1]; mu2 = mean64[3 * px + 2];
    }
    for (int k = 0; k < spw; ++k) {
      const float4 l = L[(int64_t)k * npix + px];
      if (!(isfinite(l.x) && isfinite(l.y) && isfinite(l.z))) {
        atomicAdd(stats + STAT_NONFINITE, 1ull);
        continue;
      }
      acc.x = acc.x + l.x; acc.y = acc.y + l.y; acc.z = acc.z + l.z;
      if (sum64) {
        // Welford update over the sample sequence
        const double nn = (double)(spp_before + k + 1);
        double d;
        s0 += l.x; d = l.x - mu0; mu0 += d / nn; m0 += d * (l.x - mu0);
        s1 += l.y; d = l.y - mu1; mu1 += d / nn; m1 += d * (l.y - mu1);
        s2 += l.z; d = l.z - mu2; mu2 += d / nn; m2 += d * (l.z - mu2);
      }
    }
    accum[px] = acc;
    if (sum64) {
      sum64[3 * px] = s0; sum64[3 * px + 1] = s1; sum64[3 * px + 2] = s2;
      m2_64[3 * px] = m0; m2_64[3 * px + 1] = m1; m2_64[3 * px + 2] = m2;
      mean64[3 * px] = mu0; mean64[3 * px + 1] = mu1; mean64[3 * px + 2] = mu2;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    unsigned long long rays = 0, sh = 0;
    for (int d = 0; d < max_depth; ++d) {
      rays += (unsigned long long)cnt[d * kCntStride + CNT_RAYS];
      sh += (unsigned long long)cnt[d * kCntStride + CNT_SH_AREA] +
            (unsigned long long)cnt[d * kCntStride + CNT_SH_SUN];
    }
    atomicAdd(stats + STAT_RAYS, rays);
    atomicAdd(stats + STAT_SHADOW, sh);
    atomicAdd(stats + STAT_PATHS, (unsigned long long)paths);
  }
}

// ── resolve: mean, top-down rows (cpu_tiled.cpp:224-236) ───────────────────────
__global__ void resolve_kernel(const float4* accum, int W, int H, float inv_spp, float* out) {
  const int64_t npix = (int64_t)W * H;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < npix;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(i % W), y = (int)(i / W);
    const float4 a = accum[i];
    const int64_t d = ((int64_t)(H - 1 - y) * W + x) * 3;
    out[d] = a.x * inv_spp;
    out[d + 1] = a.y * inv_spp;
    out[d + 2] = a.z * inv_spp;
  }
}

// ── ray queries (xb_trace_rays) ─────────────────────────────────────────────────
__global__ void __launch_bounds__(128) trace_full_kernel(DevScene sc, const xb_ray* rays,
                                                         int64_t n, xb_hit* hits, int mode,
                                                         unsigned long long* stats) {
  uint32_t tstack[kStackSize];
  uint32_t bstack_local[kStackSize];
  const BStack<0> bstack{nullptr, bstack_local};
  bool overflow = false;
  TraversalCounters tc{0, 0, 0, 0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const xb_ray rr = rays[i];
    Ray r{v3(rr.org[0], rr.org[1], rr.org[2]), v3(rr.dir[0], rr.dir[1], rr.dir[2]), rr.tmin, rr.tmax};
    xb_hit out;
    memset(&out, 0, sizeof(out));
    out.t = kInf; out.prim_id = -1; out.instance_id = -1; out.mat_id = -1;
    if (mode == XB_TRACE_CLOSEST) {
      HitState h;
      if (scene_closest<true>(sc, r, h, tstack, bstack, tc, overflow)) {
        FullHit f;
        complete_hit(sc, r, h, f);
        out.t = h.t; out.u = f.u; out.v = f.v;
        out.prim_id = f.prim_id; out.instance_id = f.instance_id; out.mat_id = f.mat_id;
        out.front_face = f.front_face ? 1 : 0;
        out.pos[0] = f.pos.x; out.pos[1] = f.pos.y; out.pos[2] = f.pos.z;
        out.normal[0] = f.normal.x; out.normal[1] = f.normal.y; out.normal[2] = f.normal.z;
        out.geo_normal[0] = f.geo_normal.x; out.geo_normal[1] = f.geo_normal.y;
        out.geo_normal[2] = f.geo_normal.z;
      }
    } else {
      if (scene_any<true>(sc, r, tstack, bstack, tc, overflow)) out.t = 0.f;
    }
    hits[i] = out;
  }
  if (overflow) atomicAdd(stats + STAT_OVERFLOW, 1ull);
  flush_counters(stats + (mode == XB_TRACE_CLOSEST ? STAT_EXT_WORK : STAT_SH_WORK), tc);
}

// xb_trace_rays_device on persistent warps (trace_persistent.cuh): each warp owns a contiguous
// range of the caller's rays and refills its idle lanes from it, so a long ray no longer holds
// its warp's finished lanes, and no cursor is shared between calls (calls on different streams
// may overlap, as with trace_full_kernel). The hit records are trace_full_kernel's.
struct ApiIO {
  const xb_ray* rays;
  xb_hit* hits;
  unsigned long long* st;
  int next, stop;
  __device__ __forceinline__ int end() const { return stop; }
  __device__ __forceinline__ int grab(int, int, int k) {
    const int b = next;
    next += k;
    return b;
  }
  template <bool kAny>
  __device__ __forceinline__ void load(int ray, V3& o, V3& d, float& tmin, float& tmax) const {
    const xb_ray rr = rays[ray];
    o = v3(rr.org[0], rr.org[1], rr.org[2]);
    d = v3(rr.dir[0], rr.dir[1], rr.dir[2]);
    tmin = rr.tmin;
    tmax = rr.tmax;
  }
  __device__ __forceinline__ static xb_hit miss() {
    xb_hit out;
    memset(&out, 0, sizeof(out));
    out.t = kInf; out.prim_id = -1; out.instance_id = -1; out.mat_id = -1;
    return out;
  }
  __device__ __forceinline__ void finish_any(int ray, bool occluded) const {
    xb_hit out = miss();
    if (occluded) out.t = 0.f;
    hits[ray] = out;
  }
  __device__ __forceinline__ void finish_closest(const DevScene& sc, int ray, V3 o, V3 d, float tmin, float tmax,
                                                 const HitState& h) const {
    xb_hit out = miss();
    if (h.inst >= 0) {
      const Ray r{o, d, tmin, tmax};
      FullHit f;
      complete_hit(sc, r, h, f);
      out.t = h.t; out.u = f.u; out.v = f.v;
      out.prim_id = f.prim_id; out.instance_id = f.instance_id; out.mat_id = f.mat_id;
      out.front_face = f.front_face ? 1 : 0;
      out.pos[0] = f.pos.x; out.pos[1] = f.pos.y; out.pos[2] = f.pos.z;
      out.normal[0] = f.normal.x; out.normal[1] = f.normal.y; out.normal[2] = f.normal.z;
      out.geo_normal[0] = f.geo_normal.x; out.geo_normal[1] = f.geo_normal.y;
      out.geo_normal[2] = f.geo_normal.z;
    }
    hits[ray] = out;
  }
  __device__ __forceinline__ unsigned long long* stats() const { return st; }
};

template <bool kAny>
__global__ void __launch_bounds__(128) trace_api_persistent_kernel(DevScene sc, const xb_ray* rays, int n,
                                                                   xb_hit* hits, unsigned long long* stats,
                                                                   int refill) {
  const int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t chunk = (n + warps - 1) / warps;
  const int64_t b = w * chunk < n ? w * chunk : (int64_t)n;
  const int64_t e = b + chunk < n ? b + chunk : (int64_t)n;
  ApiIO io{rays, hits, stats, (int)b, (int)e};
  trace_persistent<kAny, true, 0>(sc, io, refill, false);
}

// ── BSDF queries (xb_bsdf_eval / xb_bsdf_sample) ───────────────────────────────
__global__ void bsdf_eval_kernel(DevMaterial m, int64_t n, const float* wo, const float* wi,
                                 float* f, float* pdf) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    V3 o = v3(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]);
    V3 w = v3(wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]);
    V3 fv = bsdf_eval(o, w, m);
    f[3 * i] = fv.x; f[3 * i + 1] = fv.y; f[3 * i + 2] = fv.z;
    pdf[i] = bsdf_pdf(o, w, m);
  }
}

__global__ void bsdf_density_kernel(DevMaterial m, int64_t n, const float* wo, const float* wi, float* dens) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const V3 o = v3(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]);
    const V3 w = v3(wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]);
    dens[i] = (o.z > 0.f && !(m.flags & (kMatDelta | kMatTransmissive))) ? bsdf_density(o, w, m) : 0.f;
  }
}

__global__ void bsdf_sample_kernel(DevMaterial m, int64_t n, const float* wo, uint64_t* st,
                                   float* wi, float* f, float* pdf, int32_t* flags) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    Pcg g{st[i]};
    V3 o = v3(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]);
    BsdfSample s;
    bool ok = bsdf_sample(o, m, g, s);
    st[i] = g.state;
    wi[3 * i] = s.wi.x; wi[3 * i + 1] = s.wi.y; wi[3 * i + 2] = s.wi.z;
    f[3 * i] = s.f.x; f[3 * i + 1] = s.f.y; f[3 * i + 2] = s.f.z;
    pdf[i] = s.pdf;
    flags[i] = (ok ? 1 : 0) | (s.delta ? 2 : 0);
  }
}

// ── trace without allocation (xb_trace_rays_noalloc) ─────────────────────────────
// Some callers cannot call cudaMalloc while they trace: a plugin whose host application owns
// every device allocation (its own allocator, or a fixed memory budget set at start-up).
// For them the work-stealing trace keeps its scratch (the ray cursor and the ray count) in this
// fixed file-scope array instead of renderer-allocated memory. It is 256 bytes; every GPU that
// loads the library holds one copy until the process exits.
//
// The cursor is 64-bit: every warp's last fetch moves it 32 past the end, so it can run up to
// n + 32 × (warps in the grid) — under 2^40 + 2^36 for any batch this entry point accepts and
// any grid it launches (fewer than 2^31 warps), far from wrapping.
constexpr int kNoAllocScratchWords = 32;                       // 64-bit words: 256 bytes
constexpr int64_t kNoAllocMaxRays = XB_NOALLOC_MAX_RAYS;
static __device__ __align__(256) unsigned long long g_noalloc_scratch[kNoAllocScratchWords];

__global__ void noalloc_begin_kernel(unsigned long long* scratch, int64_t n) {
  // every call starts from a cleared cursor: the array keeps the last call's values
  if (threadIdx.x < kNoAllocScratchWords) scratch[threadIdx.x] = threadIdx.x == 1 ? (unsigned long long)n : 0ull;
}

// Work-stealing variant of trace_full_kernel: warps take 32 rays at a time from the cursor in
// scratch[0] (ray count in scratch[1]). Threads that overflowed their traversal stack are counted
// in the renderer's statistics, as trace_full_kernel counts them.
__global__ void __launch_bounds__(128) trace_stealing_kernel(DevScene sc, const xb_ray* rays, xb_hit* hits,
                                                             int mode, unsigned long long* scratch,
                                                             unsigned long long* stats) {
  __shared__ unsigned long long s_base[4];
  const int64_t n = (int64_t)scratch[1];
  uint32_t tstack[kStackSize];
  uint32_t bstack_local[kStackSize];
  const BStack<0> bstack{nullptr, bstack_local};
  bool overflow = false;
  TraversalCounters tc{0, 0, 0, 0};
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (;;) {
    if (lane == 0) s_base[warp] = atomicAdd(scratch, 32ull);
    __syncwarp();
    const int64_t base = (int64_t)s_base[warp];
    __syncwarp();
    if (base >= n) break;
    const int64_t i = base + lane;
    if (i >= n) continue;
    const xb_ray rr = rays[i];
    Ray r{v3(rr.org[0], rr.org[1], rr.org[2]), v3(rr.dir[0], rr.dir[1], rr.dir[2]), rr.tmin, rr.tmax};
    xb_hit out;
    memset(&out, 0, sizeof(out));
    out.t = kInf; out.prim_id = -1; out.instance_id = -1; out.mat_id = -1;
    if (mode == XB_TRACE_CLOSEST) {
      HitState h;
      if (scene_closest<false>(sc, r, h, tstack, bstack, tc, overflow)) {
        FullHit f;
        complete_hit(sc, r, h, f);
        out.t = h.t; out.u = f.u; out.v = f.v;
        out.prim_id = f.prim_id; out.instance_id = f.instance_id; out.mat_id = f.mat_id;
        out.front_face = f.front_face ? 1 : 0;
        out.pos[0] = f.pos.x; out.pos[1] = f.pos.y; out.pos[2] = f.pos.z;
        out.normal[0] = f.normal.x; out.normal[1] = f.normal.y; out.normal[2] = f.normal.z;
        out.geo_normal[0] = f.geo_normal.x; out.geo_normal[1] = f.geo_normal.y;
        out.geo_normal[2] = f.geo_normal.z;
      }
    } else if (scene_any<false>(sc, r, tstack, bstack, tc, overflow)) {
      out.t = 0.f;
    }
    hits[i] = out;
  }
  if (overflow) atomicAdd(stats + STAT_OVERFLOW, 1ull);
}

// XB_FLAG_SKY_IS: the sky's luminance (Rec. 709 weights) at the centre of each of kSkyBins bins
// of y = cos(theta) in [-1, 1], by Environment::evaluate's formula (src/scene/environment.h:34-46),
// floored at 1e-3 of the largest so that every direction can be proposed, as normalised
// cumulative masses. False when the sky is black.
bool sky_table(const DevScene& sc, std::vector<float>& cdf) {
  std::vector<double> f(kSkyBins);
  double fmax = 0.0;
  for (int b = 0; b < kSkyBins; ++b) {
    const double y = -1.0 + (b + 0.5) * (2.0 / kSkyBins);
    double c[3];
    for (int k = 0; k < 3; ++k) {
      const double hz = sc.sky_horizon[k];
      c[k] = y < 0.0 ? hz + (sc.sky_ground[k] - hz) * std::min(-y, 1.0)
                     : hz + (sc.sky_zenith[k] - hz) * std::pow(y, (double)sc.sky_inv_sharpness);
      c[k] *= sc.sky_intensity;
    }
    f[b] = std::max(0.0, 0.2126 * c[0] + 0.7152 * c[1] + 0.0722 * c[2]);
    fmax = std::max(fmax, f[b]);
  }
  if (!(fmax > 0.0)) return false;
  cdf.assign(kSkyBins + 1, 0.f);
  std::vector<double> acc(kSkyBins + 1, 0.0);
  for (int b = 0; b < kSkyBins; ++b) acc[b + 1] = acc[b] + std::max(f[b], 1e-3 * fmax);
  for (int b = 0; b <= kSkyBins; ++b) cdf[b] = (float)(acc[b] / acc[kSkyBins]);
  cdf[kSkyBins] = 1.f;
  return true;
}

DevMaterial to_dev_material(const xb_material& m) {
  xb_material_derived d = xb::prepare_material(m);
  DevMaterial o{};
  for (int i = 0; i < 3; ++i) {
    o.base[i] = m.base_color[i];
    o.f0[i] = d.f0[i];
    o.ss_color[i] = m.subsurface_color[i];
  }
  o.metallic = m.metallic;
  o.ior = m.ior;
  o.alpha = d.alpha; o.alpha_x = d.alpha_x; o.alpha_y = d.alpha_y;
  o.subsurface = m.subsurface;
  o.flags = d.flags;
  xb::multiscatter_constants(d, &o.ms_k1, &o.ms_k2, o.ms_fms);
  return o;
}

void sync_lanes(xb_renderer* r) {
  for (cudaStream_t s : {r->stream, r->stream2}) if (s) cudaStreamSynchronize(s);
  for (auto& x : r->lane_x)
    for (cudaStream_t s : {x.s, x.s2}) if (s) cudaStreamSynchronize(s);
}

// Drops the captured bounce loops (after their launches have finished).
void drop_graphs(xb_renderer* r) {
  if (r->bounce_graphs.empty()) return;
  sync_lanes(r);
  for (auto& kv : r->bounce_graphs) cudaGraphExecDestroy(kv.second);
  r->bounce_graphs.clear();
}

void free_scene(xb_renderer* r) {
  drop_graphs(r);
  for (void* p : r->scene_mem) cudaFree(p);
  r->scene_mem.clear();
  r->has_scene = false;
  std::memset(&r->scene, 0, sizeof(r->scene));
}

void free_wave_buffers(WaveBuffers& w) {
  void* ptrs[] = {w.ray_o[0], w.ray_o[1], w.ray_d[0], w.ray_d[1], w.tp[0], w.tp[1], w.rng[0],
                  w.rng[1], w.path[0], w.path[1], w.hit, w.hit_inst, w.sh_o[0], w.sh_o[1],
                  w.sh_d[0], w.sh_d[1], w.sh_c[0], w.sh_c[1], w.L, w.cnt, w.rec[0], w.rec[1],
                  w.ratio[0], w.ratio[1], w.maxd, w.gq[0], w.gq[1], w.gq[2], w.gq[3], w.gq[4], w.gq_rng};
  for (void* p : ptrs) if (p) cudaFree(p);
  w = WaveBuffers();
}

void free_wave(xb_renderer* r) {
  drop_graphs(r);
  sync_lanes(r);
  free_wave_buffers(r->wb);
  for (auto& x : r->lane_x) free_wave_buffers(x.wb);
  r->lanes_alloc = 0;
}

template <class T>
int dev_upload(xb_renderer* r, const std::vector<T>& v, const T** out) {
  *out = nullptr;
  if (v.empty()) return XB_OK;
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, v.size() * sizeof(T));
  if (e != cudaSuccess) return set_err(r, XB_E_OOM, "cudaMalloc(%zu) failed: %s", v.size() * sizeof(T), cudaGetErrorString(e));
  r->scene_mem.push_back(p);
  e = cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return set_err(r, XB_E_CUDA, "cudaMemcpy failed: %s", cudaGetErrorString(e));
  *out = static_cast<const T*>(p);
  return XB_OK;
}

float4 node_lo(const xb_bvh_node& n) { return make_float4(n.mn[0], n.mn[1], n.mn[2], n.mx[0]); }
float4 node_hi(const xb_bvh_node& n, uint32_t child) {
  return make_float4(n.mx[1], n.mx[2], u32_bits_to_f(child), u32_bits_to_f(n.count));
}

bool alloc_wave_buffers(WaveBuffers& w, int64_t cap) {
  w.capacity = cap;
  auto A = [&](auto** p, size_t bytes) -> bool {
    return cudaMalloc((void**)p, bytes) == cudaSuccess;
  };
  bool ok = true;
  for (int q = 0; q < 2; ++q) {
    ok &= A(&w.ray_o[q], cap * sizeof(float4));
    ok &= A(&w.ray_d[q], cap * sizeof(float4));
    ok &= A(&w.tp[q], cap * sizeof(float4));
    ok &= A(&w.rng[q], cap * sizeof(uint64_t));
    ok &= A(&w.path[q], cap * sizeof(int32_t));
    ok &= A(&w.sh_o[q], cap * sizeof(float4));
    ok &= A(&w.sh_d[q], cap * sizeof(float4));
    ok &= A(&w.sh_c[q], cap * sizeof(float4));
    ok &= A(&w.rec[q], cap * sizeof(int32_t));
    ok &= A(&w.ratio[q], cap * sizeof(float));
  }
  ok &= A(&w.hit, cap * sizeof(float4));
  ok &= A(&w.maxd, cap * sizeof(int8_t));
  ok &= A(&w.hit_inst, cap * sizeof(int32_t));
  ok &= A(&w.L, cap * sizeof(float4));
  ok &= A(&w.cnt, (kMaxDepth + 1) * kCntStride * sizeof(int32_t));
  for (int k = 0; k < 5; ++k) ok &= A(&w.gq[k], cap * sizeof(float4));
  ok &= A(&w.gq_rng, cap * sizeof(uint64_t));
  return ok;
}

// Queues for `cap` paths per wave, in each of the `waves` lanes.
int alloc_wave(xb_renderer* r, int64_t cap) {
  free_wave(r);
  bool ok = alloc_wave_buffers(r->wb, cap);
  for (int k = 1; ok && k < r->tune.waves; ++k) ok = alloc_wave_buffers(r->lane_x[k - 1].wb, cap);
  if (!ok) {
    free_wave(r);
    return set_err(r, XB_E_OOM, "cannot allocate wave buffers for %lld paths", (long long)cap);
  }
  r->lanes_alloc = r->tune.waves;
  return XB_OK;
}

int check_ready(xb_renderer* r) {
  if (!r) return xb::fail(XB_E_INVALID, "null renderer");
  cudaError_t e = cudaSetDevice(r->cfg.device);
  if (e != cudaSuccess) return set_err(r, XB_E_CUDA, "cudaSetDevice: %s", cudaGetErrorString(e));
  return XB_OK;
}

// Applies a tuning (0 keeps a field, negative restores its default) and recomputes grids.
int apply_tuning(xb_renderer* r, const xb_tuning& t) {
  xb_tuning& c = r->tune;
  auto pick = [](int32_t v, int32_t cur, int32_t def) { return v == 0 ? cur : (v < 0 ? def : v); };
  c.extend_persistent_from_depth = pick(t.extend_persistent_from_depth, c.extend_persistent_from_depth, 1);
  c.shadow_persistent = pick(t.shadow_persistent, c.shadow_persistent, 1);
  c.refill = std::min(32, pick(t.refill, c.refill, 8));
  c.extend_blocks_per_sm = std::min(64, pick(t.extend_blocks_per_sm, c.extend_blocks_per_sm, 64));
  c.shadow_blocks_per_sm = std::min(64, pick(t.shadow_blocks_per_sm, c.shadow_blocks_per_sm, 64));
  c.shade_blocks_per_sm = std::min(64, pick(t.shade_blocks_per_sm, c.shade_blocks_per_sm, 64));
  c.wave_paths = pick(t.wave_paths, c.wave_paths, 1 << 21);
  c.shadow_order = pick(t.shadow_order, c.shadow_order, 1);
  c.overlap = pick(t.overlap, c.overlap, 1);
  c.waves = std::min(kMaxLanes, pick(t.waves, c.waves, 2));
  c.lane_stagger = std::min(kMaxDepth, pick(t.lane_stagger, c.lane_stagger, 1));
  c.graph = std::min(2, pick(t.graph, c.graph, 1));
  c.guided_form = std::min(2, pick(t.guided_form, c.guided_form, 1));
  c.shade_occupancy = pick(t.shade_occupancy, c.shade_occupancy, 8);
  if (c.shade_occupancy != 4 && c.shade_occupancy != 8 && c.shade_occupancy != 12 && c.shade_occupancy != 16)
    c.shade_occupancy = 8;
  c.pixel_order = std::min(2, pick(t.pixel_order, c.pixel_order, 2));
  c.shared_stack = pick(t.shared_stack, c.shared_stack, 1);
  if (c.shared_stack != 1 && c.shared_stack != kSharedStack) c.shared_stack = 1;
  r->stack_sh = c.shared_stack > 1 ? c.shared_stack : 0;
  drop_graphs(r);
  r->ext_persistent_from = c.extend_persistent_from_depth;
  r->shadow_persistent = c.shadow_persistent == 1;
  r->refill = c.refill;
  // Persistent kernels (their blocks loop until the queue is empty) launch at most the blocks
  // that fit at once; the others fetch warps of work from a counter or take tiles in a
  // grid-stride loop, so blocks beyond the resident ones queue and, as they start while others
  // retire, interleave with the other wave lane's kernels.
  r->grid_ext = r->num_sms * c.extend_blocks_per_sm;
  r->grid_pext = r->num_sms * std::min(r->occ_pext, c.extend_blocks_per_sm);
  r->grid_shadow = r->num_sms * c.shadow_blocks_per_sm;
  r->grid_pshadow = r->num_sms * std::min(r->occ_pshadow, c.shadow_blocks_per_sm);
  r->grid_shade = r->num_sms * c.shade_blocks_per_sm;
  r->grid_gshade = r->num_sms * std::min(r->occ_gshade, c.shade_blocks_per_sm);
  const int64_t npix = (int64_t)r->cfg.width * r->cfg.height;
  const int spw = (int)std::min<int64_t>(1024, std::max<int64_t>(1, c.wave_paths / npix));
  if (spw != r->spp_per_wave || r->wb.capacity == 0 || c.waves != r->lanes_alloc) {
    r->spp_per_wave = spw;
    return alloc_wave(r, npix * spw);
  }
  return XB_OK;
}

enum { STAGE_RAYGEN = 0, STAGE_EXTEND = 1, STAGE_SHADE = 2, STAGE_SHADOW = 3, STAGE_ACCUM = 4, STAGE_TRAIN = 5 };

// Stage timing: a pair of events around a launch, read back after the call's final sync.
struct StageTimer {
  xb_renderer* r;
  int stage;
  cudaEvent_t end = nullptr;
  cudaStream_t s = nullptr;
  StageTimer(xb_renderer* rr, int st, cudaStream_t ss = nullptr) : r(rr), stage(st), s(ss ? ss : rr->stream) {
    if (!(r->prof_flags & XB_PROFILE_STAGE_TIMES)) return;
    if (r->ev_used + 2 > r->ev_pool.size()) {
      for (int k = 0; k < 64; ++k) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        r->ev_pool.push_back(e);
      }
      r->ev_stage.resize(r->ev_pool.size() / 2);
    }
    cudaEventRecord(r->ev_pool[r->ev_used], s);
    end = r->ev_pool[r->ev_used + 1];
    r->ev_stage[r->ev_used / 2] = stage;
    r->ev_used += 2;
  }
  ~StageTimer() {
    if (end) cudaEventRecord(end, s);
  }
};

// Per stage: the summed launch durations, the launch count, and the busy time — the union of
// the launch intervals, placed on one clock by their start events' times after the call's first
// event (the first launch of the call; the lanes' waves start after it).
void collect_stage_times(xb_renderer* r) {
  std::vector<std::pair<double, double>> spans[6];
  for (size_t i = 0; i + 1 < r->ev_used; i += 2) {
    float ms = 0.f, start = 0.f;
    if (cudaEventElapsedTime(&ms, r->ev_pool[i], r->ev_pool[i + 1]) == cudaSuccess) {
      const int st = r->ev_stage[i / 2];
      r->stage_ms[st] += ms;
      r->stage_launches[st] += 1;
      if (cudaEventElapsedTime(&start, r->ev_pool[0], r->ev_pool[i]) == cudaSuccess)
        spans[st].emplace_back((double)start, (double)start + ms);
    }
  }
  for (int st = 0; st < 6; ++st) {
    std::vector<std::pair<double, double>>& v = spans[st];
    std::sort(v.begin(), v.end());
    double busy = 0.0, lo = 0.0, hi = 0.0;
    for (size_t k = 0; k < v.size(); ++k) {
      if (k == 0 || v[k].first > hi) {
        if (k) busy += hi - lo;
        lo = v[k].first;
        hi = v[k].second;
      } else {
        hi = std::max(hi, v[k].second);
      }
    }
    if (!v.empty()) busy += hi - lo;
    r->stage_busy_ms[st] += busy;
  }
  r->ev_used = 0;
}

// Position box of the network's input: the configured one, else the scene's bounds.
void guide_box(xb_renderer* r) {
  const xb_guiding& gc = r->gcfg;
  const bool boxed = gc.bounds_max[0] > gc.bounds_min[0] && gc.bounds_max[1] > gc.bounds_min[1] &&
                     gc.bounds_max[2] > gc.bounds_min[2];
  for (int k = 0; k < 3; ++k) {
    const float lo = boxed ? gc.bounds_min[k] : r->scene_lo[k];
    const float hi = boxed ? gc.bounds_max[k] : r->scene_hi[k];
    r->gbmin[k] = lo;
    r->gbinv[k] = hi > lo ? 1.f / (hi - lo) : 1.f;
  }
}

// A wave lane: the queues one wave uses and the streams and events of its bounce loop.
struct LaneRef {
  WaveBuffers* w;
  cudaStream_t s, s2;
  cudaEvent_t* ev_shade;
  cudaEvent_t* ev_shadow;
};

LaneRef lane_ref(xb_renderer* r, int k) {
  if (k == 0) return LaneRef{&r->wb, r->stream, r->stream2, r->ev_shade, r->ev_shadow};
  auto& x = r->lane_x[k - 1];
  return LaneRef{&x.wb, x.s, x.s2, x.ev_shade, x.ev_shadow};
}

// The traversal kernels come in two forms: the BLAS stack wholly in local memory (kSh = 0), or
// its first kSharedStack entries in shared memory (tuning shared_stack).

template <int kSh>
void launch_extend_k(xb_renderer* r, const LaneRef& L, int d, bool count) {
  WaveBuffers& w = *L.w;
  const int q = d & 1;
  int32_t* cd_ = w.cnt + d * kCntStride;
  const size_t smem = (size_t)kSh * kShStride * sizeof(uint32_t);
  if (r->thread_per_ray || d < r->ext_persistent_from) {
    auto kern = count ? extend_kernel<true, kSh> : extend_kernel<false, kSh>;
    kern<<<r->grid_ext, 128, smem, L.s>>>(r->scene, w.ray_o[q], w.ray_d[q], w.hit, w.hit_inst, cd_, r->stats);
  } else {
    TraceQueue tq{w.ray_o[q], w.ray_d[q], cd_ + CNT_RAYS, cd_ + CNT_FETCH_EXT, w.hit, w.hit_inst,
                  nullptr, nullptr, r->stats, 0};
    auto kern = count ? extend_persistent_kernel<true, kSh> : extend_persistent_kernel<false, kSh>;
    kern<<<r->grid_pext, 128, smem, L.s>>>(r->scene, tq, r->refill);
  }
}

void launch_extend(xb_renderer* r, const LaneRef& L, int d, bool count) {
  StageTimer t(r, STAGE_EXTEND, L.s);
  if (r->stack_sh) launch_extend_k<kSharedStack>(r, L, d, count);
  else launch_extend_k<0>(r, L, d, count);
}

template <int kSh>
void launch_shadow_k(xb_renderer* r, const LaneRef& L, int d, int k, bool count, cudaStream_t s) {
  WaveBuffers& w = *L.w;
  int32_t* cd_ = w.cnt + d * kCntStride;
  const size_t smem = (size_t)kSh * kShStride * sizeof(uint32_t);
  if (r->thread_per_ray || !r->shadow_persistent) {
    auto kern = count ? shadow_kernel<true, kSh> : shadow_kernel<false, kSh>;
    kern<<<r->grid_shadow, 128, smem, s>>>(r->scene, w.sh_o[k], w.sh_d[k], w.sh_c[k], w.L,
                                           cd_ + (k ? CNT_SH_SUN : CNT_SH_AREA),
                                           cd_ + (k ? CNT_FETCH_SH_SUN : CNT_FETCH_SH_AREA), r->stats,
                                           r->tune.shadow_order == 2);
  } else {
    TraceQueue tq{w.sh_o[k], w.sh_d[k], cd_ + (k ? CNT_SH_SUN : CNT_SH_AREA),
                  cd_ + (k ? CNT_FETCH_SH_SUN : CNT_FETCH_SH_AREA), nullptr, nullptr, w.sh_c[k], w.L,
                  r->stats, r->tune.shadow_order == 2};
    auto kern = count ? shadow_persistent_kernel<true, kSh> : shadow_persistent_kernel<false, kSh>;
    kern<<<r->grid_pshadow, 128, smem, s>>>(r->scene, tq, r->refill);
  }
}

void launch_shadows(xb_renderer* r, const LaneRef& L, int d, bool count, cudaStream_t s) {
  for (int k = 0; k < 2; ++k) {
    if (k == 0 && r->scene.num_lights == 0) continue;
    if (k == 1 && r->scene.num_suns == 0) continue;
    StageTimer t(r, STAGE_SHADOW, s);
    if (r->stack_sh) launch_shadow_k<kSharedStack>(r, L, d, k, count, s);
    else launch_shadow_k<0>(r, L, d, k, count, s);
  }
}

// The bounce loop of one wave whose camera rays are in queue 0: for every depth, closest hits,
// shading (plain or guided), then the area-light and sun shadow rays (cpu_tiled.cpp:34-217).
// With overlap, bounce d's shadow rays run on the second stream while bounce d+1's closest hits
// run on the first: the two only share the scene (shadow rays add to the path radiance, closest
// hits write the hit records), and shading d+1 waits for both. Each kernel's tail — a few warps
// finishing long rays after the queue has drained — then runs beside the other kernel's bulk.
// Bounces [d0, d1) of the loop (d1 < 0: to the last); a later range continues where an earlier
// one stopped (its closest hits of bounce d0 are already traced when overlap is on).
int trace_bounces(xb_renderer* r, const LaneRef& L, bool train, int rec_stride, int depth_limit = -1,
                  const int8_t* path_maxd = nullptr, int d0 = 0, int d1 = -1) {
  WaveBuffers& w = *L.w;
  const int depth_max = std::min(depth_limit >= 0 ? depth_limit : r->max_bounces, kMaxDepth);
  const bool count = (r->prof_flags & XB_PROFILE_COUNT_TRAVERSAL) != 0;
  const bool ov = r->tune.overlap == 1 && L.s2 != nullptr;
  xbg::Guide* gd = r->guiding ? r->guide : nullptr;
  const int d_end = d1 < 0 ? depth_max : std::min(d1, depth_max);
  for (int d = d0; d < d_end; ++d) {
    const int q = d & 1, nq = q ^ 1;
    int32_t* cd_ = w.cnt + d * kCntStride;
    if (d == 0 || !ov) launch_extend(r, L, d, count);
    ShadeArgs sa;
    sa.sc = r->scene;
    sa.ray_o = w.ray_o[q]; sa.ray_d = w.ray_d[q]; sa.tp = w.tp[q]; sa.rng = w.rng[q]; sa.path = w.path[q];
    sa.nray_o = w.ray_o[nq]; sa.nray_d = w.ray_d[nq]; sa.ntp = w.tp[nq]; sa.nrng = w.rng[nq];
    sa.npath = w.path[nq];
    sa.hit = w.hit; sa.hit_inst = w.hit_inst;
    for (int k = 0; k < 2; ++k) { sa.sh_o[k] = w.sh_o[k]; sa.sh_d[k] = w.sh_d[k]; sa.sh_c[k] = w.sh_c[k]; }
    sa.L = w.L;
    sa.cnt = cd_;
    sa.cnt_next = w.cnt + (d + 1) * kCntStride;
    sa.depth = d; sa.min_bounces = r->min_bounces; sa.max_bounces = depth_max;
    sa.path_maxd = path_maxd;
    sa.capacity = (int)w.capacity;
    sa.stats = r->stats;
    bool network_pass = false;
    GuideShadeArgs ga{};
    if (gd) {
      ga.wf = xbg::guide_weights_bf16(gd);
      ga.master = xbg::guide_master(gd);
      ga.alpha = r->gcfg.fixed_fraction ? r->gcfg.guide_fraction : -1.f;
      ga.ratio_cap = r->gcfg.ratio_cap;
      ga.ratio_in = d > 0 ? w.ratio[q] : nullptr;
      ga.ratio_out = w.ratio[nq];
      for (int k = 0; k < 3; ++k) { ga.bmin[k] = r->gbmin[k]; ga.binv[k] = r->gbinv[k]; }
      ga.recs = train ? xbg::guide_records(gd) : nullptr;
      ga.rec_count = xbg::guide_record_count(gd);
      ga.rec_cap = xbg::guide_record_capacity(gd);
      ga.rec_stride = rec_stride;
      ga.rec_in = (train && d > 0) ? w.rec[q] : nullptr;
      ga.rec_out = train ? w.rec[nq] : nullptr;
      ga.err = xbg::guide_error(gd);
      StageTimer t(r, STAGE_SHADE, L.s);
      const bool net = d < r->gcfg.guided_bounces;
      if (net && r->tune.guided_form == 2) {
        guided_shade_kernel<true, 4><<<r->grid_gshade, 128, kGuidedShadeSmem, L.s>>>(sa, ga);
      } else {
        if (net) {   // two-kernel form: the guided vertices' directions come from the network pass
          for (int k = 0; k < 5; ++k) ga.gq[k] = w.gq[k];
          ga.gq_rng = w.gq_rng;
          network_pass = true;
        }
        if (r->tune.shade_occupancy == 4)
          guided_shade_kernel<false, 4><<<r->grid_shade, 128, 0, L.s>>>(sa, ga);
        else
          guided_shade_kernel<false, 8><<<r->grid_shade, 128, 0, L.s>>>(sa, ga);
      }
    } else if (r->scene.sky_cdf) {
      // sky importance sampling: the network-free guided bounce with the sky as its proposal
      ga.ratio_in = d > 0 ? w.ratio[q] : nullptr;
      ga.ratio_out = w.ratio[nq];
      ga.rec_stride = 1;
      ga.sky_alpha = 0.5f;
      StageTimer t(r, STAGE_SHADE, L.s);
      if (r->tune.shade_occupancy == 4)
        guided_shade_kernel<false, 4><<<r->grid_shade, 128, 0, L.s>>>(sa, ga);
      else
        guided_shade_kernel<false, 8><<<r->grid_shade, 128, 0, L.s>>>(sa, ga);
    } else {
      StageTimer t(r, STAGE_SHADE, L.s);
      if (r->scene_opaque) {
        if (r->tune.shade_occupancy == 4) shade_kernel<4, true><<<r->grid_shade, 128, 0, L.s>>>(sa);
        else if (r->tune.shade_occupancy == 12) shade_kernel<12, true><<<r->grid_shade, 128, 0, L.s>>>(sa);
        else if (r->tune.shade_occupancy == 16) shade_kernel<16, true><<<r->grid_shade, 128, 0, L.s>>>(sa);
        else shade_kernel<8, true><<<r->grid_shade, 128, 0, L.s>>>(sa);
      } else {
        if (r->tune.shade_occupancy == 4) shade_kernel<4, false><<<r->grid_shade, 128, 0, L.s>>>(sa);
        else if (r->tune.shade_occupancy == 12) shade_kernel<12, false><<<r->grid_shade, 128, 0, L.s>>>(sa);
        else if (r->tune.shade_occupancy == 16) shade_kernel<16, false><<<r->grid_shade, 128, 0, L.s>>>(sa);
        else shade_kernel<8, false><<<r->grid_shade, 128, 0, L.s>>>(sa);
      }
    }
    CK(cudaEventRecord(L.ev_shade[d], L.s));
    if (network_pass) {   // beside the shadow rays of this bounce, before the next closest hits
      StageTimer t(r, STAGE_SHADE, L.s);
      guide_sample_kernel<<<r->grid_gshade, 128, kGuidedShadeSmem, L.s>>>(sa, ga);
    }
    if (!ov) {
      launch_shadows(r, L, d, count, L.s);
      continue;
    }
    CK(cudaStreamWaitEvent(L.s2, L.ev_shade[d], 0));
    launch_shadows(r, L, d, count, L.s2);
    CK(cudaEventRecord(L.ev_shadow[d], L.s2));
    if (d + 1 < depth_max) launch_extend(r, L, d + 1, count);
    CK(cudaStreamWaitEvent(L.s, L.ev_shadow[d], 0));
  }
  CK(cudaGetLastError());
  return XB_OK;
}

// Bounces [d0, d1) of lane k's wave, for a bounce loop of `depth` bounces (per-path limits in
// path_maxd, or none). With `graph` tuning 1, a non-training wave replays a CUDA graph captured
// from the same launches the first time (one per lane, plain or guided, depth range and bounce
// limits); the graphs hold the scene, queue and network pointers and launch settings by value,
// so every change of those drops them (drop_graphs). Raygen and accumulation, which carry the
// wave's samples and views, are not part of them. Replaying gives the same kernels in the same
// order, hence the same image.
int bounce_range(xb_renderer* r, const LaneRef& L, int k, bool train, int rec_stride, int depth,
                 const int8_t* path_maxd, int d0, int d1) {
  if (d0 >= d1) return XB_OK;
  const bool guided = r->guiding && r->guide;
  if (r->tune.graph != 1 || train || r->prof_flags != 0 || r->graph_broken)
    return trace_bounces(r, L, train, rec_stride, depth, path_maxd, d0, d1);
  const uint32_t key = (uint32_t)k | (guided ? 4u : 0u) | (path_maxd ? 8u : 0u) | ((uint32_t)depth << 4) |
                       ((uint32_t)d0 << 12);
  auto it = r->bounce_graphs.find(key);
  if (it == r->bounce_graphs.end()) {
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ge = nullptr;
    int rc = XB_OK;
    cudaError_t e = cudaStreamBeginCapture(L.s, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      rc = trace_bounces(r, L, false, 1, depth, path_maxd, d0, d1);
      e = cudaStreamEndCapture(L.s, &g);
    }
    if (e == cudaSuccess && rc == XB_OK && g) e = cudaGraphInstantiate(&ge, g, 0);
    if (g) cudaGraphDestroy(g);
    if (e != cudaSuccess || rc != XB_OK || !ge) {
      // the launches themselves work without capture: take them directly from now on
      cudaGetLastError();
      if (ge) cudaGraphExecDestroy(ge);
      r->graph_broken = true;
      return trace_bounces(r, L, train, rec_stride, depth, path_maxd, d0, d1);
    }
    it = r->bounce_graphs.emplace(key, ge).first;
  }
  CK(cudaGraphLaunch(it->second, L.s));
  return XB_OK;
}

// A wave's whole bounce loop: the bounces before the stagger point, lane 0's stagger event,
// the rest.
int run_bounces(xb_renderer* r, const LaneRef& L, int k, bool train, int rec_stride, int depth,
                const int8_t* path_maxd) {
  const int sp = std::min(r->tune.lane_stagger, depth);
  int rc = bounce_range(r, L, k, train, rec_stride, depth, path_maxd, 0, sp);
  if (rc) return rc;
  CK(cudaEventRecord(r->ev_stagger[k], L.s));
  return bounce_range(r, L, k, train, rec_stride, depth, path_maxd, sp, depth);
}

CamDev cam_dev(const xb_camera& c) {
  return CamDev{v3(c.eye[0], c.eye[1], c.eye[2]), v3(c.lower_left[0], c.lower_left[1], c.lower_left[2]),
                v3(c.horizontal[0], c.horizontal[1], c.horizontal[2]),
                v3(c.vertical[0], c.vertical[1], c.vertical[2])};
}

// Several waves in flight: wave i of a call runs on lane i % lanes (lane 0 is the renderer's
// stream), so one wave's latency-bound stretches and kernel tails run beside the others' bulk.
// The first wave of lane k > 0 starts once lane k - 1's first wave has shaded its first
// lane_stagger bounces (ev_stagger), so the waves' widest bounces do not coincide; through lane
// 0 it also follows the main stream's work before the call. Every accumulation waits for the
// previous wave's, so the image's sums keep sample order and equal a single lane's bit for bit.
// A serial wave (guide training: the network changes after it and the records buffer is
// shared) waits for every other lane, and every other lane's next wave waits for it. At the end
// the main stream waits for every lane.
struct LaneSched {
  xb_renderer* r;
  int lanes;
  int next = 0;
  int last_acc = -1;
  bool has[kMaxLanes] = {}, serial[kMaxLanes] = {};

  LaneSched(xb_renderer* rr) : r(rr), lanes(std::max(1, std::min(rr->tune.waves, rr->lanes_alloc))) {}
  int begin(bool is_serial) {
    const int k = next;
    next = (next + 1) % lanes;
    const LaneRef L = lane_ref(r, k);
    if (k > 0 && !has[k]) cudaStreamWaitEvent(L.s, r->ev_stagger[k - 1], 0);
    for (int o = 0; o < lanes; ++o)
      if (o != k && has[o] && (is_serial || serial[o])) cudaStreamWaitEvent(L.s, r->lane_done[o], 0);
    has[k] = true;
    serial[k] = is_serial;
    return k;
  }
  void before_accumulate(int k) {
    if (last_acc >= 0 && last_acc != k) cudaStreamWaitEvent(lane_ref(r, k).s, r->lane_acc[last_acc], 0);
  }
  void after_accumulate(int k) {
    cudaEventRecord(r->lane_acc[k], lane_ref(r, k).s);
    last_acc = k;
  }
  void end_wave(int k) { cudaEventRecord(r->lane_done[k], lane_ref(r, k).s); }
  ~LaneSched() {   // every return path: the main stream takes in the other lanes' work
    for (int k = 1; k < lanes; ++k)
      if (has[k]) cudaStreamWaitEvent(r->stream, r->lane_done[k], 0);
  }
};

// Renders samples [spp_first, spp_first + spp_count) and returns, in *kept_out, how many of
// them went into the image.
int run_waves(xb_renderer* r, const xb_camera* cam, int spp_first, int spp_count, int* kept_out) {
  int kept = 0;
  *kept_out = 0;
  const int W = r->cfg.width, H = r->cfg.height;
  const int64_t npix = (int64_t)W * H;
  const CamDev cd = cam_dev(*cam);
  const int depth_max = std::min(r->max_bounces, kMaxDepth);
  int done = 0;
  xbg::Guide* gd = r->guiding ? r->guide : nullptr;
  if (gd) guide_box(r);
  LaneSched ls(r);
  while (done < spp_count) {
    const int sample0 = spp_first + done;   // 1-based index of the wave's first sample
    const bool train = gd && sample0 <= r->gcfg.train_spp;
    int spw = std::min(r->spp_per_wave, spp_count - done);
    if (train) {
      // a training wave ends at train_spp and stays within one guide_train call's step budget
      spw = std::min(spw, r->gcfg.train_spp - sample0 + 1);
      spw = std::max(1, std::min(spw, xbg::kMaxTrainSteps / std::max(1, r->gcfg.steps_per_spp)));
      // and, when the second half is kept, at its first sample
      const int first_kept = (r->gcfg.train_spp + 1) / 2 + 1;
      if (r->gcfg.keep_training_samples == 2 && sample0 < first_kept) spw = std::min(spw, first_kept - sample0);
    }
    // samples rendered while the guide trains stay out of the image unless asked for (their
    // proposal is the still-untrained network); the accumulation still counts the wave's rays
    const bool keep = !train || r->gcfg.keep_training_samples == 1 ||
                      (r->gcfg.keep_training_samples == 2 && sample0 >= (r->gcfg.train_spp + 1) / 2 + 1);
    {
      const int k = ls.begin(train);
      const LaneRef L = lane_ref(r, k);
      WaveBuffers& w = *L.w;
      const int64_t paths = npix * spw;
      CK(cudaMemsetAsync(w.cnt, 0, (depth_max + 1) * kCntStride * sizeof(int32_t), L.s));
      int rec_stride = 1;
      if (train) {
        CK(cudaMemsetAsync(xbg::guide_record_count(gd), 0, sizeof(int32_t), L.s));
        const int64_t cap = xbg::guide_record_capacity(gd);
        rec_stride = r->gcfg.record_stride > 0 ? r->gcfg.record_stride
                                               : (int)std::max<int64_t>(1, (paths * 4 + cap - 1) / cap);
      }
      const int g_rg = (int)std::min<int64_t>((paths + 255) / 256, (int64_t)r->num_sms * 16);
      {
        StageTimer t(r, STAGE_RAYGEN, L.s);
        raygen_kernel<<<g_rg, 256, 0, L.s>>>(cd, W, H, sample0, paths, w.ray_o[0], w.ray_d[0], w.tp[0],
                                             w.rng[0], w.path[0], w.L, w.cnt, r->tune.pixel_order == 2);
      }
      int rc = run_bounces(r, L, k, train, rec_stride, depth_max, nullptr);
      if (rc) return rc;
      const int g_acc = (int)std::min<int64_t>((npix + 255) / 256, (int64_t)r->num_sms * 16);
      ls.before_accumulate(k);
      {
        StageTimer t(r, STAGE_ACCUM, L.s);
        accumulate_kernel<<<g_acc, 256, 0, L.s>>>(w.L, npix, keep ? spw : 0, r->spp + kept, r->accum, r->sum64,
                                                  r->m2_64, r->mean64, w.cnt, depth_max, paths, r->stats);
      }
      ls.after_accumulate(k);
      if (train) {
        StageTimer t(r, STAGE_TRAIN, L.s);
        xbg::guide_finalize_records(gd, L.s, w.L, r->num_sms * 8, r->stats + STAT_REC_TOTAL);
        const int steps = r->gcfg.steps_per_spp * spw;
        if (xbg::guide_train(gd, L.s, xbg::guide_records(gd), xbg::guide_record_count(gd),
                             xbg::guide_record_capacity(gd), steps, r->gcfg.batch, r->gcfg.learning_rate,
                             r->gcfg.seed, r->gcfg.fixed_fraction ? r->gcfg.guide_fraction : -1.f,
                             (int64_t)r->gcfg.train_spp * r->gcfg.steps_per_spp) != XB_OK)
          return set_err(r, XB_E_CUDA, "guide training launch failed");
        r->last_loss_index = steps - 1;
      }
      ls.end_wave(k);
    }
    if (keep) kept += spw;
    CK(cudaGetLastError());
    done += spw;
  }
  *kept_out = kept;
  return XB_OK;
}

// ── many views in shared waves ───────────────────────────────────────────────────
// A wave holds pieces: (view, a run of whole samples of every pixel of that view). Paths of a
// piece are laid out sample-major like a single-view wave, so each path is seeded exactly as a
// render of that view alone would seed it and the accumulation runs in sample order.
int run_view_waves(xb_renderer* r, const xb_view* views, int count, float4* accum, const int64_t* accum_off) {
  xbg::Guide* gd = r->guiding ? r->guide : nullptr;
  if (gd) guide_box(r);
  std::vector<int> left(count);
  for (int v = 0; v < count; ++v) left[v] = views[v].spp;
  int v0 = 0;
  LaneSched ls(r);
  while (v0 < count) {
    ViewPieces pk{};
    int64_t paths = 0;
    int64_t pix_total = 0;
    for (int v = v0; v < count && pk.n < kMaxPieces; ++v) {
      if (left[v] == 0) { if (v == v0) ++v0; continue; }
      const int64_t npix = (int64_t)views[v].width * views[v].height;
      const int64_t room = (r->wb.capacity - paths) / npix;   // both lanes hold this many paths
      if (room <= 0) break;
      const int n = (int)std::min<int64_t>(left[v], room);
      ViewPiece& p = pk.p[pk.n++];
      p.cam = cam_dev(views[v].camera);
      p.W = views[v].width;
      p.H = views[v].height;
      p.s_first = views[v].spp - left[v] + 1;
      p.spp = n;
      p.path_off = paths;
      p.pix_off = pix_total;
      p.accum_off = accum_off[v];
      p.max_bounces = std::min(views[v].max_bounces > 0 ? views[v].max_bounces : r->max_bounces, kMaxDepth);
      paths += npix * n;
      pix_total += npix;
      left[v] -= n;
      if (left[v] > 0) break;   // the next wave continues this view
    }
    while (v0 < count && left[v0] == 0) ++v0;
    if (pk.n == 0) break;
    const int k = ls.begin(false);
    const LaneRef L = lane_ref(r, k);
    WaveBuffers& w = *L.w;
    int wave_depth = 0;
    for (int i = 0; i < pk.n; ++i) wave_depth = std::max(wave_depth, pk.p[i].max_bounces);
    // the counters of every depth the wave's bounce loop reads start at zero
    CK(cudaMemsetAsync(w.cnt, 0, (wave_depth + 1) * kCntStride * sizeof(int32_t), L.s));
    const int g_rg = (int)std::min<int64_t>((paths + 255) / 256, (int64_t)r->num_sms * 16);
    {
      StageTimer t(r, STAGE_RAYGEN, L.s);
      raygen_views_kernel<<<g_rg, 256, 0, L.s>>>(pk, paths, w.ray_o[0], w.ray_d[0], w.tp[0], w.rng[0],
                                                 w.path[0], w.L, w.maxd, w.cnt, r->tune.pixel_order == 2);
    }
    int rc = run_bounces(r, L, k, false, 1, wave_depth, w.maxd);
    if (rc) return rc;
    const int g_acc = (int)std::min<int64_t>((pix_total + 255) / 256, (int64_t)r->num_sms * 16);
    {
      ls.before_accumulate(k);
      StageTimer t(r, STAGE_ACCUM, L.s);
      accumulate_views_kernel<<<g_acc, 256, 0, L.s>>>(w.L, pk, pix_total, accum, w.cnt, wave_depth, paths,
                                                      r->stats);
    }
    ls.after_accumulate(k);
    ls.end_wave(k);
    CK(cudaGetLastError());
  }
  return XB_OK;
}

// Rows of `rows` x `row` doubles copied with their order reversed (bottom-up accumulation order
// to the top-down order of the resolved image, cpu_tiled.cpp:224-236).
__global__ void flip_rows_f64_kernel(const double* __restrict__ src, double* __restrict__ dst, int row, int rows) {
  const int64_t n = (int64_t)row * rows;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t y = i / row, x = i - y * row;
    dst[(rows - 1 - y) * (int64_t)row + x] = src[i];
  }
}

// ── BLAS refit (xb_refit_mesh): one mesh's triangles and node boxes, topology kept ──────────
// The passes are refit_kernels.h's, which the host refit (xb_scene_refit_mesh) runs as loops.
__global__ void refit_tris_kernel(xb::RefitArgs a) {
  const int32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < a.num_tris) xb::refit_tris_at(a, s);
}
__global__ void refit_parents_kernel(xb::RefitArgs a) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < a.num_nodes) xb::refit_parents_at(a, i);
}
__global__ void refit_nodes_kernel(xb::RefitArgs a) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < a.num_nodes) xb::refit_nodes_at(a, i);
}

}  // namespace

extern "C" {

int xb_create(const xb_config* cfg, xb_renderer** out) {
  if (!cfg || !out) return xb::fail(XB_E_INVALID, "xb_create: null argument");
  *out = nullptr;
  if (cfg->width <= 0 || cfg->height <= 0 || cfg->max_bounces < 0 || cfg->min_bounces < 0)
    return xb::fail(XB_E_INVALID, "xb_create: bad size or bounces");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return xb::fail(XB_E_CUDA, "xb_create: no CUDA device");
  if (cfg->device < 0 || cfg->device >= ndev) return xb::fail(XB_E_INVALID, "xb_create: bad device %d", cfg->device);
  auto* r = new (std::nothrow) xb_renderer();
  if (!r) return xb::fail(XB_E_OOM, "xb_create: out of memory");
  r->cfg = *cfg;
  r->min_bounces = cfg->min_bounces;
  r->max_bounces = std::min(cfg->max_bounces, kMaxDepth);
  auto bail = [&](int code) { xb_destroy(r); return code; };
  if (cudaSetDevice(cfg->device) != cudaSuccess) return bail(xb::fail(XB_E_CUDA, "cudaSetDevice failed"));
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, cfg->device) != cudaSuccess) return bail(xb::fail(XB_E_CUDA, "cudaGetDeviceProperties failed"));
  r->num_sms = prop.multiProcessorCount;
  if (cudaStreamCreateWithFlags(&r->stream2, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&r->copy_stream, cudaStreamNonBlocking) != cudaSuccess)
    return bail(xb::fail(XB_E_CUDA, "stream creation failed"));
  for (int k = 0; k < 2; ++k)
    if (cudaEventCreateWithFlags(&r->resolved[k], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&r->copied[k], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventRecord(r->copied[k], r->copy_stream) != cudaSuccess)
      return bail(xb::fail(XB_E_CUDA, "event creation failed"));
  for (int d = 0; d < kMaxDepth; ++d)
    if (cudaEventCreateWithFlags(&r->ev_shade[d], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&r->ev_shadow[d], cudaEventDisableTiming) != cudaSuccess)
      return bail(xb::fail(XB_E_CUDA, "event creation failed"));
  for (auto& x : r->lane_x) {
    if (cudaStreamCreateWithFlags(&x.s, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&x.s2, cudaStreamNonBlocking) != cudaSuccess)
      return bail(xb::fail(XB_E_CUDA, "stream creation failed"));
    for (int d = 0; d < kMaxDepth; ++d)
      if (cudaEventCreateWithFlags(&x.ev_shade[d], cudaEventDisableTiming) != cudaSuccess ||
          cudaEventCreateWithFlags(&x.ev_shadow[d], cudaEventDisableTiming) != cudaSuccess)
        return bail(xb::fail(XB_E_CUDA, "event creation failed"));
  }
  for (int k = 0; k < kMaxLanes; ++k)
    if (cudaEventCreateWithFlags(&r->lane_done[k], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&r->lane_acc[k], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&r->ev_stagger[k], cudaEventDisableTiming) != cudaSuccess)
      return bail(xb::fail(XB_E_CUDA, "event creation failed"));
  if (cudaStreamCreateWithFlags(&r->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&r->ev0) != cudaSuccess || cudaEventCreate(&r->ev1) != cudaSuccess)
    return bail(xb::fail(XB_E_CUDA, "stream/event creation failed"));
  const int64_t npix = (int64_t)cfg->width * cfg->height;
  if (cudaMalloc(&r->accum, npix * sizeof(float4)) != cudaSuccess ||
      cudaMalloc(&r->resolve_buf, npix * 3 * sizeof(float)) != cudaSuccess ||
      cudaMallocHost(&r->host_ov, 2 * sizeof(unsigned long long)) != cudaSuccess ||
      cudaMalloc(&r->resolve_async_buf[0], npix * 3 * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&r->resolve_async_buf[1], npix * 3 * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&r->stats, STAT_COUNT * sizeof(unsigned long long)) != cudaSuccess)
    return bail(xb::fail(XB_E_OOM, "framebuffer allocation failed"));
  if (cfg->flags & XB_FLAG_FP64_ACCUM) {
    if (cudaMalloc(&r->sum64, npix * 3 * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&r->m2_64, npix * 3 * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&r->mean64, npix * 3 * sizeof(double)) != cudaSuccess)
      return bail(xb::fail(XB_E_OOM, "FP64 accumulation allocation failed"));
  }
  int rc = XB_OK;
  int occ = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, extend_kernel<false, 0>, 128, 0);
  r->occ_ext = std::max(occ, 1);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, shadow_kernel<false, 0>, 128, 0);
  r->occ_shadow = std::max(occ, 1);
  // guided shade: dynamic shared memory for the weights, one activation tile and the lobes; at
  // most 4 CTAs per SM so their TMEM (64 columns each) always fits the SM's 512 columns
  if (cudaFuncSetAttribute(guide_sample_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)kGuidedShadeSmem) != cudaSuccess)
    return bail(xb::fail(XB_E_CUDA, "guide sample kernel attribute failed"));
  if (cudaFuncSetAttribute(guided_shade_kernel<true, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)kGuidedShadeSmem) != cudaSuccess)
    return bail(xb::fail(XB_E_CUDA, "guided shade kernel attribute failed"));
  {
    // CTAs per SM from the kernel's own footprint (registers in 256-register warp units, shared
    // memory with the per-CTA reservation), capped at 4 for TMEM
    cudaFuncAttributes fa{};
    int regs_sm = 65536, smem_sm = 0, smem_rsv = 0;
    cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, cfg->device);
    cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, cfg->device);
    cudaDeviceGetAttribute(&smem_rsv, cudaDevAttrReservedSharedMemoryPerBlock, cfg->device);
    if (cudaFuncGetAttributes(&fa, guided_shade_kernel<true, 4>) != cudaSuccess)
      return bail(xb::fail(XB_E_CUDA, "guided shade kernel attributes failed"));
    const int warp_regs = ((fa.numRegs * 32 + 255) / 256) * 256;
    const int by_regs = regs_sm / std::max(1, warp_regs * 4);
    const int by_smem = smem_sm / std::max<int>(1, (int)(kGuidedShadeSmem + fa.sharedSizeBytes) + smem_rsv);
    r->occ_gshade = std::max(1, std::min(4, std::min(by_regs, by_smem)));
  }
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, extend_persistent_kernel<false, 0>, 128, 0);
  r->occ_pext = std::max(occ, 1);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, shadow_persistent_kernel<false, 0>, 128, 0);
  r->occ_pshadow = std::max(occ, 1);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, trace_api_persistent_kernel<false>, 128, 0);
  r->occ_api[0] = std::max(occ, 1);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, trace_api_persistent_kernel<true>, 128, 0);
  r->occ_api[1] = std::max(occ, 1);
  r->thread_per_ray = (cfg->flags & XB_FLAG_THREAD_PER_RAY) != 0;
  {
    // Paths per wave: whole samples of every pixel, about 2^21 paths in flight by default.
    xb_tuning def;
    std::memset(&def, 0xff, sizeof(def));   // every field negative: defaults
    if (cfg->wave_paths > 0) def.wave_paths = cfg->wave_paths;
    rc = apply_tuning(r, def);
    if (rc != XB_OK) return bail(rc);
  }
  rc = xb_reset(r);
  if (rc != XB_OK) return bail(rc);
  if (cudaMemset(r->stats, 0, STAT_COUNT * sizeof(unsigned long long)) != cudaSuccess)
    return bail(xb::fail(XB_E_CUDA, "cudaMemset failed"));
  *out = r;
  return XB_OK;
}

void xb_destroy(xb_renderer* r) {
  if (!r) return;
  cudaSetDevice(r->cfg.device);
  if (r->stream) cudaStreamSynchronize(r->stream);
  sync_lanes(r);
  free_scene(r);
  free_wave(r);
  xbg::guide_destroy(r->guide);
  if (r->copy_stream) cudaStreamSynchronize(r->copy_stream);
  for (int k = 0; k < 2; ++k) {
    if (r->resolved[k]) cudaEventDestroy(r->resolved[k]);
    if (r->copied[k]) cudaEventDestroy(r->copied[k]);
  }
  if (r->copy_stream) cudaStreamDestroy(r->copy_stream);
  if (r->host_ov) cudaFreeHost(r->host_ov);
  void* ptrs[] = {r->accum, r->sum64, r->m2_64, r->mean64, r->resolve_buf, r->stats, r->scratch,
                  r->resolve_async_buf[0], r->resolve_async_buf[1], r->refit_mem};
  for (void* p : ptrs) if (p) cudaFree(p);
  for (cudaEvent_t e : r->ev_pool) cudaEventDestroy(e);
  if (r->ev0) cudaEventDestroy(r->ev0);
  if (r->ev1) cudaEventDestroy(r->ev1);
  if (r->stream2) cudaStreamSynchronize(r->stream2);
  for (int d = 0; d < kMaxDepth; ++d)
    for (cudaEvent_t e : {r->ev_shade[d], r->ev_shadow[d]})
      if (e) cudaEventDestroy(e);
  drop_graphs(r);
  for (int k = 0; k < kMaxLanes; ++k)
    for (cudaEvent_t e : {r->lane_done[k], r->lane_acc[k], r->ev_stagger[k]})
      if (e) cudaEventDestroy(e);
  for (auto& x : r->lane_x) {
    for (int d = 0; d < kMaxDepth; ++d)
      for (cudaEvent_t e : {x.ev_shade[d], x.ev_shadow[d]})
        if (e) cudaEventDestroy(e);
    for (cudaStream_t st : {x.s, x.s2}) if (st) cudaStreamDestroy(st);
  }
  if (r->stream2) cudaStreamDestroy(r->stream2);
  if (r->stream) cudaStreamDestroy(r->stream);
  delete r;
}

int xb_last_error(const xb_renderer* r, char* buf, size_t len) {
  if (!buf || !len) return XB_E_INVALID;
  const std::string& s = (r && !r->err.empty()) ? r->err : xb::g_last_error;
  std::snprintf(buf, len, "%s", s.c_str());
  return XB_OK;
}

int xb_set_bounces(xb_renderer* r, int32_t min_b, int32_t max_b) {
  int rc = check_ready(r);
  if (rc) return rc;
  if (min_b < 0 || max_b < 0 || max_b > kMaxDepth) return set_err(r, XB_E_INVALID, "bad bounces %d..%d", min_b, max_b);
  drop_graphs(r);
  r->min_bounces = min_b;
  r->max_bounces = max_b;
  return XB_OK;
}

int xb_upload_scene(xb_renderer* r, const xb_scene_view* v) {
  int rc = check_ready(r);
  if (rc) return rc;
  if (!v) return set_err(r, XB_E_INVALID, "xb_upload_scene: null view");
  CK(cudaStreamSynchronize(r->stream));
  free_scene(r);
  // ── meshes: BLAS nodes (odd-aligned per mesh), slot-ordered triangles; the refit passes
  // (refit_kernels.h, which states this layout) and the host refit's packing read it too ──
  std::vector<float4> blas, tris;
  std::vector<int32_t> tri_index, tri_mat, root_of(v->num_meshes, -1);
  std::vector<float> nx, ny, nz;
  std::vector<DevMesh> meshes(v->num_meshes);
  r->mesh_layout.assign(v->num_meshes, xb_renderer::MeshLayout());
  int64_t slot_base = 0, tri_base = 0, vtx_base = 0;
  for (int m = 0; m < v->num_meshes; ++m) {
    const xb_mesh_view& mv = v->meshes[m];
    if (mv.num_triangles > 0 && (!mv.blas_nodes || mv.num_blas_nodes <= 0 || !mv.blas_prims))
      return set_err(r, XB_E_INVALID, "mesh %d has no BLAS", m);
    if ((blas.size() / 2) % 2 == 0) { blas.push_back(make_float4(0, 0, 0, 0)); blas.push_back(make_float4(0, 0, 0, 0)); }
    const int64_t node_base = (int64_t)blas.size() / 2;
    if (mv.num_blas_nodes > 0) root_of[m] = (int32_t)node_base;
    xb_renderer::MeshLayout& ml = r->mesh_layout[m];
    ml.node_base = node_base;
    ml.slot_base = slot_base;
    ml.num_nodes = mv.num_blas_nodes > 0 ? mv.num_blas_nodes : 0;
    ml.num_tris = mv.num_triangles;
    ml.num_verts = mv.num_vertices;
    ml.tri_offset = (int32_t)tri_base;
    ml.vtx_offset = (int32_t)vtx_base;
    ml.has_normals = mv.nx != nullptr;
    if (ml.num_nodes > 0) ml.root = mv.blas_nodes[0];
    for (int i = 0; i < mv.num_blas_nodes; ++i) {
      const xb_bvh_node& nd = mv.blas_nodes[i];
      uint32_t child;
      if (nd.count > 0) {
        if ((int64_t)nd.child + nd.count > mv.num_triangles) return set_err(r, XB_E_INVALID, "mesh %d BLAS leaf out of range", m);
        child = (uint32_t)(slot_base + nd.child);
      } else {
        if ((int64_t)nd.child + 1 >= mv.num_blas_nodes) return set_err(r, XB_E_INVALID, "mesh %d BLAS child out of range", m);
        child = (uint32_t)(node_base + nd.child);
      }
      blas.push_back(node_lo(nd));
      blas.push_back(node_hi(nd, child));
    }
    for (int s = 0; s < mv.num_triangles; ++s) {
      const uint32_t t = mv.blas_prims[s];
      if ((int)t >= mv.num_triangles) return set_err(r, XB_E_INVALID, "mesh %d prim index out of range", m);
      const int i0 = mv.indices[3 * t], i1 = mv.indices[3 * t + 1], i2 = mv.indices[3 * t + 2];
      tris.push_back(make_float4(mv.vx[i0], mv.vy[i0], mv.vz[i0], i32_bits_to_f((int)t)));
      tris.push_back(make_float4(mv.vx[i1], mv.vy[i1], mv.vz[i1], i32_bits_to_f((int)(tri_base + t))));
      tris.push_back(make_float4(mv.vx[i2], mv.vy[i2], mv.vz[i2], 0.f));
    }
    for (int t = 0; t < mv.num_triangles; ++t) {
      for (int k = 0; k < 3; ++k) {
        const int vi = mv.indices[3 * t + k];
        if (vi < 0 || vi >= mv.num_vertices) return set_err(r, XB_E_INVALID, "mesh %d vertex index out of range", m);
        tri_index.push_back((int32_t)(vtx_base + vi));
      }
      const int mid = mv.mat_ids ? mv.mat_ids[t] : 0;
      if (mid < 0 || mid >= v->num_materials) return set_err(r, XB_E_INVALID, "mesh %d triangle %d material %d out of range", m, t, mid);
      tri_mat.push_back(mid);
    }
    meshes[m].tri_offset = (int32_t)tri_base;
    meshes[m].vtx_offset = (int32_t)vtx_base;
    meshes[m].has_normals = mv.nx != nullptr;
    for (int i = 0; i < mv.num_vertices; ++i) {
      nx.push_back(mv.nx ? mv.nx[i] : 0.f);
      ny.push_back(mv.ny ? mv.ny[i] : 0.f);
      nz.push_back(mv.nz ? mv.nz[i] : 0.f);
    }
    slot_base += mv.num_triangles;
    tri_base += mv.num_triangles;
    vtx_base += mv.num_vertices;
  }
  if (blas.size() / 2 >= (1u << 28) || slot_base >= (1 << 28))
    return set_err(r, XB_E_UNSUPPORTED, "scene too large: more than 2^28 BLAS nodes or triangles");
  // ── analytic prims in PrimBLAS slot order ──
  std::vector<float4> pnodes, prims;
  for (int i = 0; i < v->num_prim_nodes; ++i) {
    const xb_bvh_node& nd = v->prim_nodes[i];
    pnodes.push_back(node_lo(nd));
    pnodes.push_back(node_hi(nd, nd.child));
  }
  for (int s = 0; s < v->num_prims; ++s) {
    const uint32_t pi = v->prim_indices ? v->prim_indices[s] : (uint32_t)s;
    if ((int)pi >= v->num_prims) return set_err(r, XB_E_INVALID, "prim index out of range");
    const xb_prim& q = v->prims[pi];
    if (q.mat_id < 0 || q.mat_id >= v->num_materials) return set_err(r, XB_E_INVALID, "prim %u material out of range", pi);
    prims.push_back(make_float4(i32_bits_to_f(q.type), i32_bits_to_f(q.mat_id), i32_bits_to_f((int)pi), 0.f));
    prims.push_back(make_float4(q.p[0], q.p[1], q.p[2], q.p[3]));
    prims.push_back(make_float4(q.p[4], q.p[5], q.p[6], q.p[7]));
    prims.push_back(make_float4(q.p[8], q.p[9], 0.f, 0.f));
  }
  // ── TLAS and instances ──
  std::vector<float4> tlas;
  for (int i = 0; i < v->num_tlas_nodes; ++i) {
    tlas.push_back(node_lo(v->tlas_nodes[i]));
    tlas.push_back(node_hi(v->tlas_nodes[i], v->tlas_nodes[i].child));
  }
  std::vector<uint32_t> tinst(v->tlas_inst_indices, v->tlas_inst_indices + v->num_instances);
  std::vector<DevInstance> insts(v->num_instances);
  r->inst_geom.assign(v->num_instances, 0);
  r->inst_l2w.assign(v->num_instances, xb::Affine());
  r->has_prim_root = v->num_prim_nodes > 0;
  if (r->has_prim_root) r->prim_root = v->prim_nodes[0];
  for (int i = 0; i < v->num_instances; ++i) {
    const xb_instance_view& iv = v->instances[i];
    r->inst_geom[i] = iv.geom;
    for (int c = 0; c < 4; ++c)
      r->inst_l2w[i].c[c] = xb::F3(iv.local_to_world[3 * c], iv.local_to_world[3 * c + 1], iv.local_to_world[3 * c + 2]);
    DevInstance& d = insts[i];
    std::memcpy(d.w2l, iv.world_to_local, sizeof(d.w2l));
    d.instance_id = iv.instance_id;
    if (iv.geom == XB_GEOM_PRIMS) {
      d.kind = 1; d.root = 0; d.mesh = -1;
      if (v->num_prim_nodes == 0) return set_err(r, XB_E_INVALID, "instance %d uses the empty prim group", i);
    } else {
      if (iv.geom < 0 || iv.geom >= v->num_meshes) return set_err(r, XB_E_INVALID, "instance %d: bad mesh %d", i, iv.geom);
      d.kind = 0; d.root = root_of[iv.geom]; d.mesh = iv.geom;
      if (d.root < 0) return set_err(r, XB_E_INVALID, "instance %d uses an empty mesh", i);
    }
  }
  // ── materials, emitters, sky ──
  std::vector<DevMaterial> mats;
  bool opaque = true;
  for (int i = 0; i < v->num_materials; ++i) {
    mats.push_back(to_dev_material(v->materials[i]));
    opaque = opaque && (mats.back().flags & (kMatDelta | kMatTransmissive | kMatSubsurface)) == 0;
  }
  std::vector<DevLight> lights;
  for (int i = 0; i < v->num_lights; ++i) {
    const xb_light& l = v->lights[i];
    if (l.mesh_id < (uint32_t)v->num_meshes) r->mesh_layout[l.mesh_id].has_light = true;
    xb::LightGeom g;
    if (!xb::light_geometry(*v, l, &g)) return set_err(r, XB_E_INVALID, "light %d refers to a missing triangle", i);
    DevLight d;
    d.p0 = make_float4(g.p0[0], g.p0[1], g.p0[2], l.area);
    d.p1 = make_float4(g.p1[0], g.p1[1], g.p1[2], i32_bits_to_f((int)l.mesh_id));
    d.p2 = make_float4(g.p2[0], g.p2[1], g.p2[2], i32_bits_to_f((int)l.tri_idx));
    d.n = make_float4(g.n[0], g.n[1], g.n[2], 0.f);
    d.emission = make_float4(l.emission[0], l.emission[1], l.emission[2], 0.f);
    lights.push_back(d);
  }
  std::vector<DevSun> suns;
  for (int i = 0; i < v->num_suns; ++i) {
    DevSun s;
    std::memcpy(s.dir, v->suns[i].direction, sizeof(s.dir));
    xb::sun_emission(v->suns[i], s.emission);
    suns.push_back(s);
  }
  DevScene& sc = r->scene;
  std::memset(&sc, 0, sizeof(sc));
  const float4* cp4;
  if ((rc = dev_upload(r, blas, &sc.blas))) return rc;
  if ((rc = dev_upload(r, tris, &sc.tris))) return rc;
  if ((rc = dev_upload(r, pnodes, &sc.pnodes))) return rc;
  if ((rc = dev_upload(r, prims, &sc.prims))) return rc;
  if ((rc = dev_upload(r, tlas, &cp4))) return rc;
  sc.tlas = cp4;
  if ((rc = dev_upload(r, tinst, &sc.tlas_inst))) return rc;
  if ((rc = dev_upload(r, insts, &sc.inst))) return rc;
  if ((rc = dev_upload(r, meshes, &sc.meshes))) return rc;
  if ((rc = dev_upload(r, tri_index, &sc.tri_index))) return rc;
  if ((rc = dev_upload(r, tri_mat, &sc.tri_mat))) return rc;
  if ((rc = dev_upload(r, nx, &sc.nx))) return rc;
  if ((rc = dev_upload(r, ny, &sc.ny))) return rc;
  if ((rc = dev_upload(r, nz, &sc.nz))) return rc;
  if ((rc = dev_upload(r, mats, &sc.mats))) return rc;
  if ((rc = dev_upload(r, lights, &sc.lights))) return rc;
  if ((rc = dev_upload(r, suns, &sc.suns))) return rc;
  if (v->num_tlas_nodes > 0) {
    for (int k = 0; k < 3; ++k) {
      r->scene_lo[k] = v->tlas_nodes[0].mn[k];
      r->scene_hi[k] = v->tlas_nodes[0].mx[k];
    }
  }
  sc.num_lights = v->num_lights;
  sc.num_suns = v->num_suns;
  sc.num_tlas_nodes = v->num_tlas_nodes;
  r->tlas_cap = v->num_tlas_nodes;
  sc.num_materials = v->num_materials;
  std::memcpy(sc.sky_zenith, v->sky.zenith, sizeof(sc.sky_zenith));
  std::memcpy(sc.sky_horizon, v->sky.horizon, sizeof(sc.sky_horizon));
  std::memcpy(sc.sky_ground, v->sky.ground, sizeof(sc.sky_ground));
  sc.sky_inv_sharpness = 1.0f / v->sky.sharpness;
  sc.sky_intensity = v->sky.intensity;
  sc.sun_nee = (r->cfg.flags & XB_FLAG_SUN_NEE) != 0;
  sc.watertight = (r->cfg.flags & XB_FLAG_WATERTIGHT) != 0;
  if ((r->cfg.flags & XB_FLAG_SKY_IS) && sc.sky_intensity > 0.f) {
    std::vector<float> cdf;
    if (sky_table(sc, cdf) && (rc = dev_upload(r, cdf, &sc.sky_cdf))) return rc;
  }
  r->scene_opaque = opaque;
  r->has_scene = true;
  return XB_OK;
}

int xb_refit_mesh(xb_renderer* r, int32_t mesh, const float* positions, const float* normals) {
  int rc = check_ready(r);
  if (rc) return rc;
  if (!r->has_scene) return set_err(r, XB_E_STATE, "xb_refit_mesh: no scene uploaded");
  if (mesh < 0 || mesh >= (int)r->mesh_layout.size() || !positions)
    return set_err(r, XB_E_INVALID, "xb_refit_mesh: bad mesh %d or null positions", mesh);
  xb_renderer::MeshLayout& ml = r->mesh_layout[mesh];
  if (ml.has_light)
    return set_err(r, XB_E_UNSUPPORTED, "xb_refit_mesh: mesh %d carries area lights (refit the host scene "
                   "with xb_scene_refit_mesh and upload it again)", mesh);
  if (normals && !ml.has_normals)
    return set_err(r, XB_E_INVALID, "xb_refit_mesh: mesh %d was uploaded without normals", mesh);
  const int64_t nv = ml.num_verts;
  for (int64_t i = 0; i < 3 * nv; ++i)
    if (!std::isfinite(positions[i]) || (normals && !std::isfinite(normals[i])))
      return set_err(r, XB_E_INVALID, "xb_refit_mesh: non-finite value at %lld", (long long)i);
  if (ml.num_nodes == 0 || ml.num_tris == 0) return XB_OK;
  sync_lanes(r);                          // no wave may read the scene while it changes
  CK(cudaStreamSynchronize(r->stream));
  // scratch: positions, normals, parents, arrival counts, status (256-byte aligned pieces)
  auto up = [](size_t b) { return (b + 255) & ~(size_t)255; };
  const size_t b_pos = up(12 * (size_t)nv), b_nodes = up(4 * (size_t)ml.num_nodes);
  const size_t need = b_pos * (normals ? 2 : 1) + 2 * b_nodes + 256;
  if (need > r->refit_bytes) {
    if (r->refit_mem) CK(cudaFree(r->refit_mem));
    r->refit_mem = nullptr;
    r->refit_bytes = 0;
    CK(cudaMalloc(&r->refit_mem, need));
    r->refit_bytes = need;
  }
  char* base = static_cast<char*>(r->refit_mem);
  xb::RefitArgs a;
  a.blas = reinterpret_cast<xb::Quad*>(const_cast<float4*>(r->scene.blas));
  a.tris = reinterpret_cast<xb::Quad*>(const_cast<float4*>(r->scene.tris));
  a.tri_index = r->scene.tri_index;
  float* pos_dev = reinterpret_cast<float*>(base);
  a.pos = pos_dev;
  float* nrm = normals ? reinterpret_cast<float*>(base + b_pos) : nullptr;
  char* rest = base + b_pos * (normals ? 2 : 1);
  a.parent = reinterpret_cast<int32_t*>(rest);
  a.arrivals = reinterpret_cast<uint32_t*>(rest + b_nodes);
  a.status = reinterpret_cast<int32_t*>(rest + 2 * b_nodes);
  a.node_base = ml.node_base;
  a.slot_base = ml.slot_base;
  a.num_nodes = ml.num_nodes;
  a.num_tris = ml.num_tris;
  a.num_verts = ml.num_verts;
  a.tri_offset = ml.tri_offset;
  a.vtx_offset = ml.vtx_offset;
  cudaStream_t s = r->stream;
  CK(cudaMemcpyAsync(pos_dev, positions, 12 * (size_t)nv, cudaMemcpyHostToDevice, s));
  if (normals) {
    // the device keeps normals as three arrays over all vertices: one copy per component
    CK(cudaMemcpyAsync(nrm, normals, 12 * (size_t)nv, cudaMemcpyHostToDevice, s));
    float* dst[3] = {const_cast<float*>(r->scene.nx), const_cast<float*>(r->scene.ny),
                     const_cast<float*>(r->scene.nz)};
    for (int k = 0; k < 3; ++k)
      CK(cudaMemcpy2DAsync(dst[k] + ml.vtx_offset, sizeof(float), nrm + k, 3 * sizeof(float), sizeof(float),
                           (size_t)nv, cudaMemcpyDeviceToDevice, s));
  }
  CK(cudaMemsetAsync(a.parent, 0xff, 4 * (size_t)ml.num_nodes, s));
  CK(cudaMemsetAsync(a.status, 0, sizeof(int32_t), s));
  refit_tris_kernel<<<(ml.num_tris + 255) / 256, 256, 0, s>>>(a);
  refit_parents_kernel<<<(ml.num_nodes + 255) / 256, 256, 0, s>>>(a);
  refit_nodes_kernel<<<(ml.num_nodes + 255) / 256, 256, 0, s>>>(a);
  CK(cudaGetLastError());
  int32_t status = 0;
  float4 root[2];
  CK(cudaMemcpyAsync(&status, a.status, sizeof(status), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(root, r->scene.blas + 2 * ml.node_base, sizeof(root), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  drop_graphs(r);
  if (status != 0) {
    // the triangles and some boxes are rewritten already: no render may trace this scene
    r->has_scene = false;
    return set_err(r, XB_E_INVALID, "xb_refit_mesh: mesh %d's BLAS is malformed (%s); upload the scene again",
                   mesh, status == 1 ? "an index out of range" : "a cycle");
  }
  ml.root.mn[0] = root[0].x; ml.root.mn[1] = root[0].y; ml.root.mn[2] = root[0].z;
  ml.root.mx[0] = root[0].w; ml.root.mx[1] = root[1].x; ml.root.mx[2] = root[1].y;
  // the TLAS over the instances' new world boxes, built on the host as xb_scene_build builds it
  std::vector<const xb_bvh_node*> roots(r->inst_geom.size(), nullptr);
  for (size_t i = 0; i < roots.size(); ++i) {
    const int32_t g = r->inst_geom[i];
    if (g >= 0 && g < (int32_t)r->mesh_layout.size() && r->mesh_layout[g].num_nodes > 0) roots[i] = &r->mesh_layout[g].root;
    else if (g == XB_GEOM_PRIMS && r->has_prim_root) roots[i] = &r->prim_root;
  }
  std::vector<xb_bvh_node> nodes;
  std::vector<uint32_t> order;
  try {
    xb::build_tlas(r->inst_l2w, roots, nodes, order);
  } catch (const std::bad_alloc&) {
    return set_err(r, XB_E_OOM, "xb_refit_mesh: out of host memory");
  }
  std::vector<float4> tlas;
  for (const xb_bvh_node& n : nodes) {
    tlas.push_back(node_lo(n));
    tlas.push_back(node_hi(n, n.child));
  }
  DevScene& sc = r->scene;
  if ((int64_t)nodes.size() > r->tlas_cap) {
    const float4* fresh;
    if ((rc = dev_upload(r, tlas, &fresh))) return rc;
    sc.tlas = fresh;
    r->tlas_cap = (int64_t)nodes.size();
  } else if (!tlas.empty()) {
    CK(cudaMemcpy(const_cast<float4*>(sc.tlas), tlas.data(), tlas.size() * sizeof(float4), cudaMemcpyHostToDevice));
  }
  if (!order.empty())
    CK(cudaMemcpy(const_cast<uint32_t*>(sc.tlas_inst), order.data(), order.size() * sizeof(uint32_t),
                  cudaMemcpyHostToDevice));
  sc.num_tlas_nodes = (int32_t)nodes.size();
  if (!nodes.empty()) {
    for (int k = 0; k < 3; ++k) {
      r->scene_lo[k] = nodes[0].mn[k];
      r->scene_hi[k] = nodes[0].mx[k];
    }
  }
  return XB_OK;
}

int xb_reset(xb_renderer* r) {
  int rc = check_ready(r);
  if (rc) return rc;
  const int64_t npix = (int64_t)r->cfg.width * r->cfg.height;
  CK(cudaMemsetAsync(r->accum, 0, npix * sizeof(float4), r->stream));
  if (r->sum64) {
    CK(cudaMemsetAsync(r->sum64, 0, npix * 3 * sizeof(double), r->stream));
    CK(cudaMemsetAsync(r->m2_64, 0, npix * 3 * sizeof(double), r->stream));
    CK(cudaMemsetAsync(r->mean64, 0, npix * 3 * sizeof(double), r->stream));
  }
  r->spp = 0;
  r->next_sample = 1;
  CK(cudaStreamSynchronize(r->stream));
  return XB_OK;
}

int xb_render_range(xb_renderer* r, const xb_camera* cam, int32_t spp_first, int32_t spp_count) {
  int rc = check_ready(r);
  if (rc) return rc;
  if (!cam) return set_err(r, XB_E_INVALID, "xb_render: null camera");
  if (!r->has_scene) return set_err(r, XB_E_STATE, "xb_render: no scene uploaded");
  if (spp_count < 0 || spp_first < 1) return set_err(r, XB_E_INVALID, "xb_render: bad sample range");
  if (spp_count == 0) return XB_OK;
  // the overflow counter is snapshotted on the device, so the call's only host read comes after
  // its work (a read at the start would queue behind a pending xb_resolve_async copy)
  snapshot_kernel<<<1, 32, 0, r->stream>>>(r->stats);
  CK(cudaEventRecord(r->ev0, r->stream));
  int kept = 0;
  rc = run_waves(r, cam, spp_first, spp_count, &kept);
  if (rc) return rc;
  CK(cudaEventRecord(r->ev1, r->stream));
  r->spp += kept;
  r->next_sample = std::max(r->next_sample, spp_first + spp_count);
  CK(cudaMemcpyAsync(r->host_ov, r->stats + STAT_OVERFLOW, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                     r->stream));
  CK(cudaStreamSynchronize(r->stream));
  CK(cudaEventElapsedTime(&r->last_ms, r->ev0, r->ev1));
  collect_stage_times(r);
  if (r->host_ov[0] != r->host_ov[1])
    return set_err(r, XB_E_OVERFLOW, "%llu queue/stack overflows during render (work dropped)",
                   r->host_ov[0] - r->host_ov[1]);
  return XB_OK;
}

int xb_render(xb_renderer* r, const xb_camera* cam, int32_t spp_to_add) {
  if (!r) return xb::fail(XB_E_INVALID, "null renderer");
  return xb_render_range(r, cam, r->next_sample, spp_to_add);
}

int xb_render_views(xb_renderer* r, const xb_view* views, int32_t count) {
  int rc = check_ready(r);
  if (rc) return rc;
  if (!views || count <= 0 || count > 65536) return set_err(r, XB_E_INVALID, "xb_render_views: bad view list");
  if (!r->has_scene) return set_err(r, XB_E_STATE, "xb_render_views: no scene uploaded");
  std::vector<int64_t> off(count);
  int64_t total = 0, max_npix = 0;
  for (int v = 0; v < count; ++v) {
    const xb_view& vw = views[v];
    if (vw.width <= 0 || vw.height <= 0 || vw.spp < 0 || !vw.out_rgb || vw.max_bounces < 0 ||
        vw.max_bounces > kMaxDepth || (int64_t)vw.width * vw.height > (1ll << 26))
      return set_err(r, XB_E_INVALID, "xb_render_views: view %d has a bad size, sample count or output", v);
    off[v] = total;
    const int64_t npix = (int64_t)vw.width * vw.height;
    total += npix;
    max_npix = std::max(max_npix, npix);
  }
  if (max_npix > r->wb.capacity) {
    rc = alloc_wave(r, max_npix);
    if (rc) return rc;
  }
  float4* accum = nullptr;
  float* out = nullptr;
  if (cudaMalloc(&accum, total * sizeof(float4)) != cudaSuccess ||
      cudaMalloc(&out, max_npix * 3 * sizeof(float)) != cudaSuccess) {
    cudaFree(accum);
    return set_err(r, XB_E_OOM, "xb_render_views: cannot allocate %lld view pixels", (long long)total);
  }
  auto fail = [&](int code) { cudaStreamSynchronize(r->stream); cudaFree(accum); cudaFree(out); return code; };
  unsigned long long ov_before = 0, ov_after = 0;
  if (cudaMemsetAsync(accum, 0, total * sizeof(float4), r->stream) != cudaSuccess ||
      cudaMemcpyAsync(&ov_before, r->stats + STAT_OVERFLOW, sizeof(ov_before), cudaMemcpyDeviceToHost,
                      r->stream) != cudaSuccess ||
      cudaEventRecord(r->ev0, r->stream) != cudaSuccess)
    return fail(set_err(r, XB_E_CUDA, "xb_render_views: setup failed"));
  rc = run_view_waves(r, views, count, accum, off.data());
  if (rc) return fail(rc);
  if (cudaEventRecord(r->ev1, r->stream) != cudaSuccess)
    return fail(set_err(r, XB_E_CUDA, "xb_render_views: event record failed"));
  for (int v = 0; v < count; ++v) {
    const xb_view& vw = views[v];
    const int64_t npix = (int64_t)vw.width * vw.height;
    const int g = (int)std::min<int64_t>((npix + 255) / 256, (int64_t)r->num_sms * 16);
    resolve_view_kernel<<<g, 256, 0, r->stream>>>(accum + off[v], vw.width, vw.height,
                                                  vw.spp > 0 ? 1.0f / (float)vw.spp : 0.f, out);
    if (cudaMemcpyAsync(vw.out_rgb, out, npix * 3 * sizeof(float), cudaMemcpyDeviceToHost, r->stream) !=
        cudaSuccess)
      return fail(set_err(r, XB_E_CUDA, "xb_render_views: copy of view %d failed", v));
  }
  if (cudaMemcpyAsync(&ov_after, r->stats + STAT_OVERFLOW, sizeof(ov_after), cudaMemcpyDeviceToHost,
                      r->stream) != cudaSuccess)
    return fail(set_err(r, XB_E_CUDA, "xb_render_views: stats copy failed"));
  cudaError_t e = cudaStreamSynchronize(r->stream);
  if (e != cudaSuccess) return fail(set_err(r, XB_E_CUDA, "xb_render_views: %s", cudaGetErrorString(e)));
  cudaEventElapsedTime(&r->last_ms, r->ev0, r->ev1);
  collect_stage_times(r);
  cudaFree(accum);
  cudaFree(out);
  if (ov_after != ov_before)
    return set_err(r, XB_E_OVERFLOW, "%llu queue/stack overflows during render (work dropped)", ov_after - ov_before);
  return XB_OK;
}

int xb_resolve_async(xb_renderer* r, float* out) {
  int rc = check_ready(r);
  if (rc) return rc;
  if (!out) return set_err(r, XB_E_INVALID, "xb_resolve_async: null output");
  const int W = r->cfg.width, H = r->cfg.height;
  const size_t bytes = (size_t)W * H * 3 * sizeof(float);
  const int k = r->resolve_slot;
  r->resolve_slot ^= 1;
  // the image of two calls ago must be read back before this call overwrites its buffer
  CK(cudaStreamWaitEvent(r->stream, r->copied[k], 0));
  const float inv = r->spp > 0 ? 1.0f / (float)r->spp : 0.f;
  resolve_kernel<<<r->num_sms * 8, 256, 0, r->stream>>>(r->accum, W, H, inv, r->resolve_async_buf[k]);
  CK(cudaGetLastError());
  CK(cudaEventRecord(r->resolved[k], r->stream));
  CK(cudaStreamWaitEvent(r->copy_stream, r->resolved[k], 0));
  CK(cudaMemcpyAsync(out, r->resolve_async_buf[k], bytes, cudaMemcpyDeviceToHost, r->copy_stream));
  CK(cudaEventRecord(r->copied[k], r->copy_stream));
  return XB_OK;
}

int xb_sync(xb_renderer* r) {
  int rc = check_ready(r);
  if (rc) return rc;
  CK(cudaStreamSynchronize(r->stream));
  if (r->copy_stream) CK(cudaStreamSynchronize(r->copy_stream));
  return XB_OK;
}

int xb_resolve(xb_renderer* r, float* out) {
  int rc = check_ready(r);
  if (rc) return rc;
  if (!out) return set_err(r, XB_E_INVALID, "xb_resolve: null output");
  const int W = r->cfg.width, H = r->cfg.height;
  const float inv = r->spp > 0 ? 1.0f / (float)r->spp : 0.f;
  resolve_kernel<<<r->num_sms * 8, 256, 0, r->stream>>>(r->accum, W, H, inv, r->resolve_buf);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out, r->resolve_buf, (size_t)W * H * 3 * sizeof(float), cudaMemcpyDeviceToHost, r->stream));
  CK(cudaStreamSynchronize(r->stream));
  return XB_OK;
}

int xb_output_stage(xb_renderer* r, uint8_t* rgb8, xb_noise_stats* stats) {
  int rc = check_ready(r);
  if (rc) return rc;
  const int W = r->cfg.width, H = r->cfg.height;
  const float inv = r->spp > 0 ? 1.0f / (float)r->spp : 0.f;
  resolve_kernel<<<r->num_sms * 8, 256, 0, r->stream>>>(r->accum, W, H, inv, r->resolve_buf);
  CK(cudaGetLastError());
  rc = xb::device_output_stage(r->resolve_buf, W, H, r->num_sms, r->stream, rgb8, stats);
  if (rc) return set_err(r, rc, "%s", xb::g_last_error.c_str());
  return XB_OK;
}

int xb_resolve_fp64(xb_renderer* r, double* sum, double* m2) {
  int rc = check_ready(r);
  if (rc) return rc;
  if (!r->sum64) return set_err(r, XB_E_STATE, "renderer was created without XB_FLAG_FP64_ACCUM");
  // rows are flipped to the top-down order of xb_resolve (cpu_tiled.cpp:224-236)
  const int W = r->cfg.width, H = r->cfg.height;
  const size_t row = (size_t)W * 3;
  std::vector<double> tmp((size_t)H * row);
  double* outs[2] = {sum, m2};
  const double* srcs[2] = {r->sum64, r->m2_64};
  for (int k = 0; k < 2; ++k) {
    if (!outs[k]) continue;
    CK(cudaMemcpyAsync(tmp.data(), srcs[k], tmp.size() * sizeof(double), cudaMemcpyDeviceToHost, r->stream));
    CK(cudaStreamSynchronize(r->stream));
    for (int y = 0; y < H; ++y) std::memcpy(outs[k] + (size_t)(H - 1 - y) * row, tmp.data() + (size_t)y * row, row * sizeof(double));
  }
  return XB_OK;
}

int xb_resolve_fp64_device(xb_renderer* r, double* sum, double* m2) {
  int rc = check_ready(r);
  if (rc) return rc;
  if (!r->sum64) return set_err(r, XB_E_STATE, "renderer was created without XB_FLAG_FP64_ACCUM");
  const int W = r->cfg.width, H = r->cfg.height;
  double* outs[2] = {sum, m2};
  const double* srcs[2] = {r->sum64, r->m2_64};
  for (int k = 0; k < 2; ++k) {
    if (!outs[k]) continue;
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, outs[k]) != cudaSuccess || at.type != cudaMemoryTypeDevice ||
        at.device != r->cfg.device)
      return set_err(r, XB_E_INVALID, "xb_resolve_fp64_device: output %d is not device memory of GPU %d", k,
                     r->cfg.device);
    flip_rows_f64_kernel<<<std::min<int64_t>((int64_t)H * W * 3 / 256 + 1, (int64_t)r->num_sms * 8), 256, 0,
                           r->stream>>>(srcs[k], outs[k], W * 3, H);
  }
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(r->stream));
  return XB_OK;
}

int xb_get_spp(const xb_renderer* r) { return r ? r->spp : XB_E_INVALID; }

int xb_get_render_stats(const xb_renderer* r_, xb_render_stats* out) {
  xb_renderer* r = const_cast<xb_renderer*>(r_);
  int rc = check_ready(r);
  if (rc) return rc;
  if (!out) return set_err(r, XB_E_INVALID, "null output");
  unsigned long long s[STAT_COUNT];
  CK(cudaMemcpyAsync(s, r->stats, sizeof(s), cudaMemcpyDeviceToHost, r->stream));
  CK(cudaStreamSynchronize(r->stream));
  out->rays_closest = (int64_t)s[STAT_RAYS];
  out->rays_shadow = (int64_t)s[STAT_SHADOW];
  out->paths = (int64_t)s[STAT_PATHS];
  out->overflow = (int64_t)s[STAT_OVERFLOW];
  out->last_ms = r->last_ms;
  out->nonfinite = (int64_t)s[STAT_NONFINITE];
  return XB_OK;
}

int xb_reset_render_stats(xb_renderer* r) {
  int rc = check_ready(r);
  if (rc) return rc;
  CK(cudaMemsetAsync(r->stats, 0, STAT_COUNT * sizeof(unsigned long long), r->stream));
  CK(cudaStreamSynchronize(r->stream));
  return XB_OK;
}

int xb_set_tuning(xb_renderer* r, const xb_tuning* t) {
  int rc = check_ready(r);
  if (rc) return rc;
  if (!t) return set_err(r, XB_E_INVALID, "xb_set_tuning: null tuning");
  if (t->refill > 32 || t->shadow_persistent > 2 || t->shadow_order > 2)
    return set_err(r, XB_E_INVALID, "xb_set_tuning: bad value");
  CK(cudaStreamSynchronize(r->stream));
  return apply_tuning(r, *t);
}

int xb_get_tuning(const xb_renderer* r, xb_tuning* out) {
  if (!r || !out) return xb::fail(XB_E_INVALID, "xb_get_tuning: null argument");
  *out = r->tune;
  return XB_OK;
}

// ── learned path guiding ─────────────────────────────────────────────────────────
int xb_set_guiding(xb_renderer* r, const xb_guiding* g) {
  int rc = check_ready(r);
  if (rc) return rc;
  if (!g) return set_err(r, XB_E_INVALID, "xb_set_guiding: null config");
  drop_graphs(r);
  xb_guiding c = *g;
  if (c.train_spp == 0) c.train_spp = 32;
  if (c.steps_per_spp == 0) c.steps_per_spp = 64;
  if (c.batch == 0) c.batch = 16384;
  if (c.learning_rate == 0.f) c.learning_rate = 5e-3f;
  if (c.guide_fraction == 0.f) c.guide_fraction = 0.7f;
  if (c.max_records == 0) c.max_records = 1 << 21;
  if (c.seed == 0) c.seed = 1;
  if (c.guided_bounces == 0) c.guided_bounces = kMaxDepth;
  if (c.ratio_cap == 0.f) c.ratio_cap = 2.5f;
  if (c.train_spp < -1 || c.steps_per_spp < 0 || c.steps_per_spp > xbg::kMaxTrainSteps || c.batch < 0 ||
      c.batch % 128 != 0 || c.batch > (1 << 20) || !(c.learning_rate > 0.f) || !(c.guide_fraction > 0.f) ||
      c.guide_fraction > 1.f || c.max_records < 128 || c.max_records > (1 << 24) || c.record_stride < 0 || c.guided_bounces < 0 ||
      (c.fixed_fraction != 0 && c.fixed_fraction != 1) || c.keep_training_samples < 0 || c.keep_training_samples > 2 ||
      !(c.ratio_cap < 0.f || c.ratio_cap >= 1.f))
    return set_err(r, XB_E_INVALID, "xb_set_guiding: bad configuration");
  if (!c.enabled) {
    r->guiding = false;
    r->gcfg = c;
    return XB_OK;
  }
  CK(cudaStreamSynchronize(r->stream));
  if (!r->guide || c.seed != r->gcfg.seed || c.max_records != r->gcfg.max_records) {
    xbg::guide_destroy(r->guide);
    r->guide = nullptr;
    rc = xbg::guide_create(&r->guide, c.seed, c.max_records);
    if (rc != XB_OK) return set_err(r, rc, "xb_set_guiding: cannot create the network (%d records)", c.max_records);
    r->last_loss_index = -1;
  }
  r->gcfg = c;
  r->guiding = true;
  return XB_OK;
}

int xb_get_guiding(const xb_renderer* r, xb_guiding* out) {
  if (!r || !out) return xb::fail(XB_E_INVALID, "xb_get_guiding: null argument");
  *out = r->gcfg;
  out->enabled = r->guiding ? 1 : 0;
  return XB_OK;
}

int xb_get_guiding_stats(const xb_renderer* r_, xb_guiding_stats* out) {
  xb_renderer* r = const_cast<xb_renderer*>(r_);
  int rc = check_ready(r);
  if (rc) return rc;
  if (!out) return set_err(r, XB_E_INVALID, "null output");
  std::memset(out, 0, sizeof(*out));
  unsigned long long s[STAT_COUNT];
  CK(cudaMemcpyAsync(s, r->stats, sizeof(s), cudaMemcpyDeviceToHost, r->stream));
  float loss = 0.f;
  if (r->guide && r->last_loss_index >= 0)
    CK(cudaMemcpyAsync(&loss, xbg::guide_losses(r->guide) + r->last_loss_index, sizeof(float),
                       cudaMemcpyDeviceToHost, r->stream));
  CK(cudaStreamSynchronize(r->stream));
  out->adam_steps = r->guide ? xbg::guide_steps_taken(r->guide) : 0;
  out->records = (int64_t)s[STAT_REC_TOTAL];
  out->records_dropped = (int64_t)s[STAT_REC_DROPPED];
  out->last_loss = loss;
  out->training = (r->guiding && r->next_sample <= r->gcfg.train_spp) ? 1 : 0;
  if (r->guide) {
    int herr = 0;
    CK(cudaMemcpy(&herr, xbg::guide_error(r->guide), sizeof(int), cudaMemcpyDeviceToHost));
    if (herr) return set_err(r, XB_E_TIMEOUT, "guiding: a tensor-core completion wait ran out");
  }
  return XB_OK;
}

int xb_guide_get_params(xb_renderer* r, float* params) {
  int rc = check_ready(r);
  if (rc) return rc;
  if (!params) return set_err(r, XB_E_INVALID, "null output");
  if (!r->guide) return set_err(r, XB_E_STATE, "guiding was never enabled");
  CK(cudaMemcpyAsync(params, xbg::guide_master(r->guide), xbg::kParams * sizeof(float), cudaMemcpyDeviceToHost,
                     r->stream));
  CK(cudaStreamSynchronize(r->stream));
  return XB_OK;
}

int xb_guide_set_params(xb_renderer* r, const float* params) {
  int rc = check_ready(r);
  if (rc) return rc;
  if (!params) return set_err(r, XB_E_INVALID, "null input");
  if (!r->guide) return set_err(r, XB_E_STATE, "guiding was never enabled");
  CK(cudaMemcpyAsync(xbg::guide_master(r->guide), params, xbg::kParams * sizeof(float), cudaMemcpyHostToDevice,
                     r->stream));
  xbg::guide_sync_bf16(r->guide, r->stream);
  xbg::guide_reset_optimizer(r->guide, r->stream);
  CK(cudaStreamSynchronize(r->stream));
  return XB_OK;
}

int xb_set_profiling(xb_renderer* r, int32_t flags) {
  int rc = check_ready(r);
  if (rc) return rc;
  if (flags & ~(XB_PROFILE_STAGE_TIMES | XB_PROFILE_COUNT_TRAVERSAL)) return set_err(r, XB_E_INVALID, "bad profiling flags");
  r->prof_flags = flags;
  return XB_OK;
}

int xb_get_profile(const xb_renderer* r_, xb_profile* out) {
  xb_renderer* r = const_cast<xb_renderer*>(r_);
  int rc = check_ready(r);
  if (rc) return rc;
  if (!out) return set_err(r, XB_E_INVALID, "null output");
  unsigned long long s[STAT_COUNT];
  CK(cudaMemcpyAsync(s, r->stats, sizeof(s), cudaMemcpyDeviceToHost, r->stream));
  CK(cudaStreamSynchronize(r->stream));
  std::memset(out, 0, sizeof(*out));
  out->raygen_ms = r->stage_ms[STAGE_RAYGEN]; out->extend_ms = r->stage_ms[STAGE_EXTEND];
  out->shade_ms = r->stage_ms[STAGE_SHADE]; out->shadow_ms = r->stage_ms[STAGE_SHADOW];
  out->accumulate_ms = r->stage_ms[STAGE_ACCUM];
  out->raygen_launches = r->stage_launches[STAGE_RAYGEN];
  out->extend_launches = r->stage_launches[STAGE_EXTEND];
  out->shade_launches = r->stage_launches[STAGE_SHADE];
  out->shadow_launches = r->stage_launches[STAGE_SHADOW];
  out->accumulate_launches = r->stage_launches[STAGE_ACCUM];
  out->ext_blas_nodes = (int64_t)s[STAT_EXT_WORK]; out->ext_tris = (int64_t)s[STAT_EXT_WORK + 1];
  out->ext_tlas_nodes = (int64_t)s[STAT_EXT_WORK + 2]; out->ext_instances = (int64_t)s[STAT_EXT_WORK + 3];
  out->sh_blas_nodes = (int64_t)s[STAT_SH_WORK]; out->sh_tris = (int64_t)s[STAT_SH_WORK + 1];
  out->sh_tlas_nodes = (int64_t)s[STAT_SH_WORK + 2]; out->sh_instances = (int64_t)s[STAT_SH_WORK + 3];
  out->train_ms = r->stage_ms[STAGE_TRAIN];
  out->train_launches = r->stage_launches[STAGE_TRAIN];
  out->extend_busy_ms = r->stage_busy_ms[STAGE_EXTEND];
  out->shade_busy_ms = r->stage_busy_ms[STAGE_SHADE];
  out->shadow_busy_ms = r->stage_busy_ms[STAGE_SHADOW];
  return XB_OK;
}

int xb_reset_profile(xb_renderer* r) {
  int rc = check_ready(r);
  if (rc) return rc;
  for (int i = 0; i < 6; ++i) { r->stage_ms[i] = 0; r->stage_launches[i] = 0; r->stage_busy_ms[i] = 0; }
  unsigned long long z[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  CK(cudaMemcpyAsync(r->stats + STAT_EXT_WORK, z, sizeof(z), cudaMemcpyHostToDevice, r->stream));
  CK(cudaStreamSynchronize(r->stream));
  return XB_OK;
}

int xb_trace_rays_device(xb_renderer* r, const xb_ray* rays, int64_t n, xb_hit* hits, int32_t mode,
                         void* stream) {
  int rc = check_ready(r);
  if (rc) return rc;
  if (!r->has_scene) return set_err(r, XB_E_STATE, "xb_trace_rays: no scene uploaded");
  if (n < 0 || (n > 0 && (!rays || !hits))) return set_err(r, XB_E_INVALID, "xb_trace_rays: bad arguments");
  if (mode != XB_TRACE_CLOSEST && mode != XB_TRACE_ANY) return set_err(r, XB_E_INVALID, "bad trace mode %d", mode);
  if (n == 0) return XB_OK;
  cudaStream_t s = stream ? (cudaStream_t)stream : r->stream;
  const int any = mode == XB_TRACE_ANY ? 1 : 0;
  // persistent warps, each over its own contiguous range of the batch, where the renderer's
  // tuning puts its own rays of that kind on persistent warps (bounce rays for closest hits)
  const bool persistent = any ? r->tune.shadow_persistent == 1 : r->tune.extend_persistent_from_depth <= 1;
  if (!r->thread_per_ray && persistent && n <= (int64_t)INT32_MAX / 2) {
    const int grid = (int)std::min<int64_t>((n + 127) / 128, (int64_t)r->num_sms * r->occ_api[any]);
    const int refill = std::max(1, r->tune.refill);
    if (any) trace_api_persistent_kernel<true><<<grid, 128, 0, s>>>(r->scene, rays, (int)n, hits, r->stats, refill);
    else trace_api_persistent_kernel<false><<<grid, 128, 0, s>>>(r->scene, rays, (int)n, hits, r->stats, refill);
  } else {
    const int grid = (int)std::min<int64_t>((n + 127) / 128, (int64_t)r->num_sms * 16);
    trace_full_kernel<<<grid, 128, 0, s>>>(r->scene, rays, n, hits, mode, r->stats);
  }
  CK(cudaGetLastError());
  return XB_OK;
}

// Device address of g_noalloc_scratch, looked up once per device (with that device current)
// by the first call made on it; cudaGetSymbolAddress allocates nothing.
static std::mutex g_noalloc_mu;
static unsigned long long* g_noalloc_ptr[128] = {};

int xb_trace_rays_noalloc(xb_renderer* r, const xb_ray* rays, int64_t n, xb_hit* hits, int32_t mode,
                          void* stream) {
  int rc = check_ready(r);
  if (rc) return rc;
  if (!r->has_scene) return set_err(r, XB_E_STATE, "xb_trace_rays_noalloc: no scene uploaded");
  if (n < 0 || (n > 0 && (!rays || !hits))) return set_err(r, XB_E_INVALID, "xb_trace_rays_noalloc: bad arguments");
  if (n > kNoAllocMaxRays)
    return set_err(r, XB_E_INVALID, "xb_trace_rays_noalloc: %lld rays exceed the maximum batch of %lld",
                   (long long)n, (long long)kNoAllocMaxRays);
  if (mode != XB_TRACE_CLOSEST && mode != XB_TRACE_ANY) return set_err(r, XB_E_INVALID, "bad trace mode %d", mode);
  if (n == 0) return XB_OK;
  const int dev = r->cfg.device;
  if (dev < 0 || dev >= 128) return set_err(r, XB_E_UNSUPPORTED, "xb_trace_rays_noalloc: device %d", dev);
  unsigned long long* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
      void* p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess || !p)
        return set_err(r, XB_E_CUDA, "cudaGetSymbolAddress(g_noalloc_scratch) failed: %s", cudaGetErrorString(e));
      g_noalloc_ptr[dev] = static_cast<unsigned long long*>(p);
    }
    scratch = g_noalloc_ptr[dev];
  }
  cudaStream_t s = stream ? (cudaStream_t)stream : r->stream;
  noalloc_begin_kernel<<<1, kNoAllocScratchWords, 0, s>>>(scratch, n);
  const int grid = (int)std::min<int64_t>((n + 127) / 128, (int64_t)r->num_sms * r->occ_ext);
  trace_stealing_kernel<<<grid, 128, 0, s>>>(r->scene, rays, hits, mode, scratch, r->stats);
  CK(cudaGetLastError());
  return XB_OK;
}

int xb_trace_rays(xb_renderer* r, const xb_ray* rays, int64_t n, xb_hit* hits, int32_t mode) {
  int rc = check_ready(r);
  if (rc) return rc;
  if (n < 0 || (n > 0 && (!rays || !hits))) return set_err(r, XB_E_INVALID, "xb_trace_rays: bad arguments");
  if (n == 0) return XB_OK;
  xb_ray* dr = nullptr;
  xb_hit* dh = nullptr;
  CK(cudaMalloc(&dr, n * sizeof(xb_ray)));
  if (cudaMalloc(&dh, n * sizeof(xb_hit)) != cudaSuccess) {
    cudaFree(dr);
    return set_err(r, XB_E_OOM, "xb_trace_rays: out of device memory");
  }
  unsigned long long ov0 = 0, ov1 = 0;
  cudaMemcpyAsync(&ov0, r->stats + STAT_OVERFLOW, sizeof(ov0), cudaMemcpyDeviceToHost, r->stream);
  cudaMemcpyAsync(dr, rays, n * sizeof(xb_ray), cudaMemcpyHostToDevice, r->stream);
  rc = xb_trace_rays_device(r, dr, n, dh, mode, r->stream);
  if (rc == XB_OK) {
    cudaMemcpyAsync(hits, dh, n * sizeof(xb_hit), cudaMemcpyDeviceToHost, r->stream);
    cudaMemcpyAsync(&ov1, r->stats + STAT_OVERFLOW, sizeof(ov1), cudaMemcpyDeviceToHost, r->stream);
    cudaError_t e = cudaStreamSynchronize(r->stream);
    if (e != cudaSuccess) rc = set_err(r, XB_E_CUDA, "xb_trace_rays: %s", cudaGetErrorString(e));
    else if (ov1 != ov0) rc = set_err(r, XB_E_OVERFLOW, "xb_trace_rays: traversal stack overflow");
  }
  cudaFree(dr);
  cudaFree(dh);
  return rc;
}

int xb_bsdf_eval(const xb_material* m, int64_t n, const float* wo, const float* wi, float* f, float* pdf) {
  if (!m || n < 0 || (n > 0 && (!wo || !wi || !f || !pdf))) return xb::fail(XB_E_INVALID, "xb_bsdf_eval: bad arguments");
  if (n == 0) return XB_OK;
  float *d = nullptr;
  const size_t bytes = (size_t)n * 10 * sizeof(float);
  if (cudaMalloc(&d, bytes) != cudaSuccess) return xb::fail(XB_E_OOM, "xb_bsdf_eval: out of device memory");
  float *dwo = d, *dwi = d + 3 * n, *df = d + 6 * n, *dp = d + 9 * n;
  cudaMemcpy(dwo, wo, n * 3 * sizeof(float), cudaMemcpyHostToDevice);
  cudaMemcpy(dwi, wi, n * 3 * sizeof(float), cudaMemcpyHostToDevice);
  bsdf_eval_kernel<<<(int)std::min<int64_t>((n + 255) / 256, 4096), 256>>>(to_dev_material(*m), n, dwo, dwi, df, dp);
  cudaMemcpy(f, df, n * 3 * sizeof(float), cudaMemcpyDeviceToHost);
  cudaError_t e = cudaMemcpy(pdf, dp, n * sizeof(float), cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return xb::fail(XB_E_CUDA, "xb_bsdf_eval: %s", cudaGetErrorString(e));
  return XB_OK;
}

int xb_bsdf_density(const xb_material* m, int64_t n, const float* wo, const float* wi, float* density) {
  if (!m || n < 0 || (n > 0 && (!wo || !wi || !density)))
    return xb::fail(XB_E_INVALID, "xb_bsdf_density: bad arguments");
  if (n == 0) return XB_OK;
  float* d = nullptr;
  if (cudaMalloc(&d, (size_t)n * 7 * sizeof(float)) != cudaSuccess)
    return xb::fail(XB_E_OOM, "xb_bsdf_density: out of device memory");
  float *dwo = d, *dwi = d + 3 * n, *dd = d + 6 * n;
  cudaMemcpy(dwo, wo, n * 3 * sizeof(float), cudaMemcpyHostToDevice);
  cudaMemcpy(dwi, wi, n * 3 * sizeof(float), cudaMemcpyHostToDevice);
  bsdf_density_kernel<<<(int)std::min<int64_t>((n + 255) / 256, 4096), 256>>>(to_dev_material(*m), n, dwo, dwi, dd);
  cudaError_t e = cudaMemcpy(density, dd, n * sizeof(float), cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return xb::fail(XB_E_CUDA, "xb_bsdf_density: %s", cudaGetErrorString(e));
  return XB_OK;
}

int xb_bsdf_sample(const xb_material* m, int64_t n, const float* wo, uint64_t* st, float* wi, float* f,
                   float* pdf, int32_t* flags) {
  if (!m || n < 0 || (n > 0 && (!wo || !st || !wi || !f || !pdf || !flags)))
    return xb::fail(XB_E_INVALID, "xb_bsdf_sample: bad arguments");
  if (n == 0) return XB_OK;
  char* d = nullptr;
  const size_t bytes = (size_t)n * (3 + 3 + 3 + 1 + 1) * sizeof(float) + (size_t)n * sizeof(uint64_t);
  if (cudaMalloc(&d, bytes) != cudaSuccess) return xb::fail(XB_E_OOM, "xb_bsdf_sample: out of device memory");
  uint64_t* dst = reinterpret_cast<uint64_t*>(d);
  float* dwo = reinterpret_cast<float*>(d + n * sizeof(uint64_t));
  float *dwi = dwo + 3 * n, *df = dwo + 6 * n, *dp = dwo + 9 * n;
  int32_t* dfl = reinterpret_cast<int32_t*>(dwo + 10 * n);
  cudaMemcpy(dst, st, n * sizeof(uint64_t), cudaMemcpyHostToDevice);
  cudaMemcpy(dwo, wo, n * 3 * sizeof(float), cudaMemcpyHostToDevice);
  bsdf_sample_kernel<<<(int)std::min<int64_t>((n + 255) / 256, 4096), 256>>>(to_dev_material(*m), n, dwo, dst, dwi, df, dp, dfl);
  cudaMemcpy(st, dst, n * sizeof(uint64_t), cudaMemcpyDeviceToHost);
  cudaMemcpy(wi, dwi, n * 3 * sizeof(float), cudaMemcpyDeviceToHost);
  cudaMemcpy(f, df, n * 3 * sizeof(float), cudaMemcpyDeviceToHost);
  cudaMemcpy(pdf, dp, n * sizeof(float), cudaMemcpyDeviceToHost);
  cudaError_t e = cudaMemcpy(flags, dfl, n * sizeof(int32_t), cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return xb::fail(XB_E_CUDA, "xb_bsdf_sample: %s", cudaGetErrorString(e));
  return XB_OK;
}

}  // extern "C"
