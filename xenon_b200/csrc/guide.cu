// guide.cu — the path-guiding network on the B200 tensor cores (tcgen05: BF16 operands in shared
// memory, FP32 accumulation in TMEM). No reference counterpart: the reference has no learned part.
//
// This translation unit may contract FMAs (it is not on the reference-exact path).
//
//   guide_infer_kernel      rows of surface features -> 64 encoded features -> 4 layers -> 8 vMF
//                           lobes (persistent CTAs, weights resident in shared memory, one 128-row
//                           MMA chain per tile; each layer's epilogue (bias, ReLU, bf16) feeds the
//                           next through shared memory)
//   guide_train_kernel      per 128-row tile of training records: forward keeping the activations,
//                           the mixture's weighted negative log-likelihood gradient at the outputs,
//                           backward through the layers on the tensor cores: per layer one commit
//                           of the weight gradient delta^T a (summed over the tile's rows) and the
//                           next error signal delta W
//   adam_kernel             FP32 master weights and Adam moments, and the BF16 copies of the new weights
//   finalize_records_kernel training weight of each record once its path has finished
//   tc_gemm_kernel          one tile of D = A * B^T: the MMA building block, checked on its own
//
// The mathematics (encoding, lobe mapping, pdf, loss and gradients) is the FP64 oracle's
// (oracle/guide_ref.py) in FP32.

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/xenon_b200.h"
#include "capi_common.h"
#include "guide.h"
#include "guide_dev.cuh"
#include "tc05.cuh"

using namespace xbd;

namespace xbg {

namespace {

// ── inference ─────────────────────────────────────────────────────────────────────
__global__ void __launch_bounds__(128) guide_infer_kernel(const float* __restrict__ feats, int feat_stride,
                                                          const int32_t* __restrict__ count, int max_rows,
                                                          const __nv_bfloat16* __restrict__ wf,
                                                          const float* __restrict__ master,
                                                          float* __restrict__ lobes, int* err) {
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t* sW = smem;
  uint8_t* sA = smem + kFwdWeightBytes;
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmem_slot;
  __shared__ float sBias[kBiasFloats];
  const int n = min(*count, max_rows);
  const int tiles = (n + kTile - 1) / kTile;
  if ((int)blockIdx.x >= tiles) return;
  load_forward_weights(sW, sBias, wf, master);
  mma_setup(&tmem_slot, &mbar);
  Mma m{tmem_slot, &mbar, 0u, err, true};
  for (int t = blockIdx.x; t < tiles && m.ok; t += gridDim.x) {
    const int row = t * kTile + threadIdx.x;
    float f[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (row < n)
      for (int i = 0; i < 9; ++i) f[i] = feats[(size_t)row * feat_stride + i];
    encode_row(f, sA, threadIdx.x);
    float raw[kOut];
    forward_tile(m, sA, sW, sBias, raw);
    if (!m.ok) break;
    float lob[kLobeFloats];
    raw_to_lobes(raw, lob);
    if (row < n) {
      float* o = lobes + (size_t)row * kOutRow;
      for (int i = 0; i < kLobeFloats; ++i) o[i] = lob[i];
      o[kLobeFloats] = selection(raw);
    }
  }
  mma_teardown(m.tmem);
}

// ── training ──────────────────────────────────────────────────────────────────────
__device__ __forceinline__ uint64_t mix64(uint64_t h) {
  h ^= h >> 31; h *= 0x94D049BB133111EBull; h ^= h >> 29; h *= 0xBF58476D1CE4E5B9ull; h ^= h >> 32;
  return h;
}

// First record of tile b of a training step. With no more records than the batch the tiles cover
// them in order; otherwise each tile is 128 consecutive records at a random start, so a batch
// mixes records from all over the set (they are stored in the order the bounces produced them).
__device__ __forceinline__ int tile_start(int n, int batch, uint64_t seed, uint64_t t, int b) {
  if (n <= batch) return b * kTile;
  const uint64_t h = mix64(seed * 0x9E3779B97F4A7C15ull + t * 0xD1B54A32D192ED03ull + (uint64_t)b);
  return (int)(h % (uint64_t)(n - kTile + 1));
}

// Sum of the weights c over the step's batch (one block per tile, added into *csum).
__global__ void weight_sum_kernel(const float* recs, const int32_t* rec_count, int cap, int batch, uint64_t seed,
                                  uint64_t t, float* csum) {
  __shared__ float part[4];
  const int n = min(*rec_count, cap);
  const int start = tile_start(n, batch, seed, t, blockIdx.x);
  const int i = start + threadIdx.x;
  float c = i < n ? recs[(size_t)i * kRecFloats + 12] : 0.f;
  for (int off = 16; off > 0; off >>= 1) c += __shfl_xor_sync(0xffffffffu, c, off);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) atomicAdd(csum, part[0] + part[1] + part[2] + part[3]);
}

struct TrainArgs {
  const float* recs;
  const int32_t* rec_count;
  int cap, batch;
  uint64_t seed, t;       // tile placement of this step
  float alpha_fixed;      // selection probability the renderer uses (< 0: the network's own)
  const float* csum;      // sum of the batch's weights
  const __nv_bfloat16* wf;
  const __nv_bfloat16* wb;
  const float* master;
  float* grad;
  float* loss;
  int* err;
};

// Gradient of c (-log p(omega)) / csum with respect to the 48 raw outputs, p = a q + (1 - a) pb
// the mixture the renderer samples (a: the learned selection probability; pb < 0: p = q alone)
// (oracle: loss_grad_raw).
__device__ __forceinline__ float output_gradient(const float* raw, const float* om, float cb, float pb,
                                                 float alpha_fixed, float* g) {
  float lob[kLobeFloats];
  raw_to_lobes(raw, lob);
  float v[kLobes], cosv[kLobes], q = 0.f;
#pragma unroll
  for (int k = 0; k < kLobes; ++k) {
    const float* L = lob + 5 * k;
    cosv[k] = L[0] * om[0] + L[1] * om[1] + L[2] * om[2];
    v[k] = vmf_norm(L[3]) * expf(L[3] * (cosv[k] - 1.f));
    q += L[4] * v[k];
  }
  q = fmaxf(q, 1e-30f);
  const bool mix = pb >= 0.f;
  const bool learned = mix && alpha_fixed < 0.f;
  const float a = mix ? (learned ? selection(raw) : alpha_fixed) : 1.f;
  const float pm = fmaxf(mix ? a * q + (1.f - a) * pb : q, 1e-30f);
  const float loss = cb > 0.f ? -cb * logf(pm) : 0.f;
  const float cq = cb * (a * q / pm);   // d(-log pm) = (a q / pm) d(-log q) for q's parameters
#pragma unroll
  for (int i = 40; i < kOut; ++i) g[i] = 0.f;
  if (learned) {
    const float sg = (a - kAMin) / (kAMax - kAMin);
    g[kSelect] = cb * (-(q - pb) / pm) * (kAMax - kAMin) * sg * (1.f - sg);
  }
#pragma unroll
  for (int k = 0; k < kLobes; ++k) {
    const float* L = lob + 5 * k;
    const float r = L[4] * v[k] / q;
    g[5 * k + 4] = cq * (L[4] - r);
    const float kp = L[3];
    const float dlogv = 1.f / kp - 2.f / expm1f(2.f * kp) + (cosv[k] - 1.f);
    const float kr = raw[5 * k + 3];
    g[5 * k + 3] = (kr > -4.f && kr < 6.f) ? -cq * r * dlogv * kp : 0.f;
    const float* m = raw + 5 * k;
    const float s = sqrtf(m[0] * m[0] + m[1] * m[1] + m[2] * m[2] + 1e-8f);
    float dmu[3], proj = 0.f;
#pragma unroll
    for (int a3 = 0; a3 < 3; ++a3) {
      dmu[a3] = -cq * r * kp * om[a3];
      proj += dmu[a3] * L[a3];
    }
#pragma unroll
    for (int a3 = 0; a3 < 3; ++a3) g[5 * k + a3] = (dmu[a3] - proj * L[a3]) / s;
  }
  return loss;
}

// This tile's weight gradient of a layer from TMEM columns [64, 128) (run_backward): thread o < O
// adds its row dW[o][0..64) into gW with 16-byte atomics; and db[o] += sum_r delta[r][o] from the
// FP32 error signal. Every thread takes part in the TMEM loads.
__device__ __forceinline__ void add_weight_grad(const Mma& m, const float* sDf, int O, float* gW, float* gB) {
  const int o = threadIdx.x;
#pragma unroll
  for (int c = 0; c < kK; c += 16) {
    float v[16];
    m.load16(64 + c, v);
    if (o < O) {
      float4* dst = reinterpret_cast<float4*>(gW + (size_t)o * kK + c);
#pragma unroll
      for (int q = 0; q < 4; ++q) atomicAdd(dst + q, make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]));
    }
  }
  if (o < O) {
    float s = 0.f;
    for (int r = 0; r < kTile; ++r) s += sDf[r * kHid + o];
    atomicAdd(gB + o, s);
  }
}

constexpr uint32_t kBwdWeightBytes = 3 * kWBytes + kW3bBytes;
constexpr size_t kInferSmem = kFwdWeightBytes + kTileBytes + 1024;
constexpr size_t kTrainSmem = kFwdWeightBytes + kBwdWeightBytes + 5 * kTileBytes + kTile * kHid * 4 + 1024;

__global__ void __launch_bounds__(128, 1) guide_train_kernel(TrainArgs A) {
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t* sWf = smem;
  uint8_t* sWb = sWf + kFwdWeightBytes;
  uint8_t* sAct = sWb + kBwdWeightBytes;                    // a0 .. a3, one tile each
  uint8_t* sD = sAct + 4 * kTileBytes;                      // delta as the bf16 A operand
  float* sDf = reinterpret_cast<float*>(sD + kTileBytes);   // delta in FP32, [128][64]
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmem_slot;
  __shared__ float sBias[kBiasFloats];
  __shared__ float sLoss[4];
  const int n = min(*A.rec_count, A.cap);
  const int start = tile_start(n, A.batch, A.seed, A.t, blockIdx.x);
  if (start >= n) return;
  const float csum = *A.csum;
  load_forward_weights(sWf, sBias, A.wf, A.master);
  for (int l = 0; l < 3; ++l) load_matrix(sWb + l * kWBytes, A.wb + l * kHid * kK, kHid, kK);
  load_matrix(sWb + 3 * kWBytes, A.wb + 3 * kHid * kK, kHid, kOut);
  mma_setup(&tmem_slot, &mbar, 128);
  Mma m{tmem_slot, &mbar, 0u, A.err, true};
  const bool valid = start + (int)threadIdx.x < n;
  float f[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, om[3] = {0, 0, 1}, c = 0.f, pb = -1.f;
  if (valid) {
    const float* R = A.recs + (size_t)(start + threadIdx.x) * kRecFloats;
    for (int i = 0; i < 9; ++i) f[i] = R[i];
    om[0] = R[9]; om[1] = R[10]; om[2] = R[11];
    c = R[12];
    pb = R[20];
  }
  encode_row(f, sAct, threadIdx.x);
  for (int l = 0; l < 3 && m.ok; ++l) {
    m.sync_before();
    m.run(smem_u32(sAct + l * kTileBytes), smem_u32(sWf + l * kWBytes), kK, kHid);
    if (m.ok) hidden_epilogue(m, sBias + l * kHid, sAct + (l + 1) * kTileBytes);
  }
  if (m.ok) {
    m.sync_before();
    m.run(smem_u32(sAct + 3 * kTileBytes), smem_u32(sWf + 3 * kWBytes), kK, kOut);
  }
  float loss_part = 0.f;
  if (m.ok) {
    float raw[kOut];
    for (int cc = 0; cc < kOut; cc += 16) m.load16(cc, raw + cc);
    for (int i = 0; i < kOut; ++i) raw[i] += sBias[3 * kHid + i];
    const float cb = (valid && csum > 0.f) ? c / csum : 0.f;
    float g[kOut];
    loss_part = output_gradient(raw, om, cb, pb, A.alpha_fixed, g);
    for (int i = 0; i < kOut; ++i) sDf[threadIdx.x * kHid + i] = g[i];
    for (int k0 = 0; k0 < kOut; k0 += 8) store8_bf16(sD, threadIdx.x, k0, kOut, g + k0);
  }
  for (int off = 16; off > 0; off >>= 1) loss_part += __shfl_xor_sync(0xffffffffu, loss_part, off);
  if ((threadIdx.x & 31) == 0) sLoss[threadIdx.x >> 5] = loss_part;
  __syncthreads();
  if (threadIdx.x == 0) atomicAdd(A.loss, sLoss[0] + sLoss[1] + sLoss[2] + sLoss[3]);
  // backward: dW_l = delta_l^T a_l and delta_{l-1} = (delta_l W_l) o [a_l > 0], both on the tensor
  // cores in one commit (run_backward)
  for (int l = 3; l >= 0 && m.ok; --l) {
    const int O = l == 3 ? kOut : kHid;
    m.sync_before();
    m.run_backward(smem_u32(sD), O, smem_u32(sAct + l * kTileBytes), l > 0 ? smem_u32(sWb + l * kWBytes) : 0u);
    if (!m.ok) break;
    add_weight_grad(m, sDf, O, A.grad + off_w(l), A.grad + off_b(l));
    if (l == 0) break;
    __syncthreads();   // every thread's column sums of sDf are done before it is overwritten
    for (int cc = 0; cc < kHid; cc += 16) {
      float dv[16];
      m.load16(cc, dv);
      for (int i = 0; i < 16; ++i) {
        const float a = load_bf16(sAct + l * kTileBytes, threadIdx.x, cc + i, kK);
        dv[i] = a > 0.f ? dv[i] : 0.f;
        sDf[threadIdx.x * kHid + cc + i] = dv[i];
      }
      store8_bf16(sD, threadIdx.x, cc, kK, dv);
      store8_bf16(sD, threadIdx.x, cc + 8, kK, dv + 8);
    }
  }
  mma_teardown(m.tmem, 128);
}

// One Adam step on the FP32 master parameters, their moments and the gradient (cleared for the
// next step), and the new weights' BF16 copies (forward W_l as [out][in], backward W_l^T as
// [in][out]) written in the same pass.
__global__ void adam_kernel(float* p, float* g, float* mo, float* ve, __nv_bfloat16* wf, __nv_bfloat16* wb, float lr,
                            float b1, float b2, float eps, float c1, float c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kParams; i += gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float m = b1 * mo[i] + (1.f - b1) * gi;
    const float v = b2 * ve[i] + (1.f - b2) * gi * gi;
    mo[i] = m;
    ve[i] = v;
    const float w = p[i] - lr * (m / c1) / (sqrtf(v / c2) + eps);
    p[i] = w;
    g[i] = 0.f;
    const int l = i / off_w(1), j = i - off_w(l);
    const int outs = l == 3 ? kOut : kHid;
    if (j < outs * kK) {
      const int o = j / kK, k = j % kK;
      wf[l * kHid * kK + o * kK + k] = __float2bfloat16_rn(w);
      wb[l * kHid * kK + k * outs + o] = __float2bfloat16_rn(w);
    }
  }
}

// BF16 copies of the weights: forward W_l as [out][in], backward W_l^T as [in][out].
__global__ void pack_bf16_kernel(const float* master, __nv_bfloat16* wf, __nv_bfloat16* wb) {
  for (int l = 0; l < 4; ++l) {
    const int outs = l == 3 ? kOut : kHid;
    const float* W = master + off_w(l);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < outs * kK; i += gridDim.x * blockDim.x) {
      const int o = i / kK, k = i % kK;
      wf[l * kHid * kK + o * kK + k] = __float2bfloat16_rn(W[i]);
      wb[l * kHid * kK + k * outs + o] = __float2bfloat16_rn(W[i]);
    }
  }
}

// c = F(omega) / p(omega) of each record: the radiance its continuation brought into the path,
// divided by the throughput before the vertex, averaged over the channels the path carries.
__global__ void finalize_records_kernel(float* recs, const int32_t* rec_count, int cap, const float4* L,
                                        unsigned long long* total) {
  const int n = min(*rec_count, cap);
  if (blockIdx.x == 0 && threadIdx.x == 0 && total) atomicAdd(total, (unsigned long long)n);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float* R = recs + (size_t)i * kRecFloats;
    const float4 le = L[__float_as_int(R[13])];
    const float lend[3] = {le.x, le.y, le.z};
    float c = 0.f;
    int k = 0;
    for (int ch = 0; ch < 3; ++ch) {
      const float T = R[14 + ch];
      if (T > 1e-20f) {
        c += (lend[ch] - R[17 + ch]) / T;
        ++k;
      }
    }
    c = k ? c / (float)k : 0.f;
    R[12] = (isfinite(c) && c > 0.f) ? c : 0.f;
  }
}

}  // namespace

struct Guide {
  float* master = nullptr;     // kParams FP32
  float* grad = nullptr;
  float* mom = nullptr;
  float* vel = nullptr;
  __nv_bfloat16* wf = nullptr; // 4 x 64 x 64 slots
  __nv_bfloat16* wb = nullptr;
  float* csum = nullptr;       // per step of one guide_train call: the batch's weight sum
  float* loss = nullptr;
  int* err = nullptr;
  float* recs = nullptr;       // training records
  int32_t* rec_count = nullptr;
  int rec_cap = 0;
  int max_steps = 0;
  int64_t t = 0;               // Adam steps taken
};

int guide_create(Guide** out, uint64_t seed, int rec_cap) {
  auto* g = new (std::nothrow) Guide();
  if (!g) return XB_E_OOM;
  g->max_steps = kMaxTrainSteps;
  g->rec_cap = std::max(0, rec_cap);
  bool ok = cudaMalloc(&g->master, kParams * 4) == cudaSuccess && cudaMalloc(&g->grad, kParams * 4) == cudaSuccess &&
            cudaMalloc(&g->mom, kParams * 4) == cudaSuccess && cudaMalloc(&g->vel, kParams * 4) == cudaSuccess &&
            cudaMalloc(&g->wf, 4 * kHid * kK * 2) == cudaSuccess && cudaMalloc(&g->wb, 4 * kHid * kK * 2) == cudaSuccess &&
            cudaMalloc(&g->csum, g->max_steps * 4) == cudaSuccess &&
            cudaMalloc(&g->loss, g->max_steps * 4) == cudaSuccess && cudaMalloc(&g->err, 4) == cudaSuccess &&
            cudaMalloc(&g->rec_count, 4) == cudaSuccess;
  if (ok && g->rec_cap > 0) ok = cudaMalloc(&g->recs, (size_t)g->rec_cap * kRecFloats * 4) == cudaSuccess;
  if (!ok) { guide_destroy(g); return XB_E_OOM; }
  // He-uniform hidden layers and a 0.1-scaled output layer (as the oracle's init_params), drawn
  // from a splitmix64 stream so the initial network depends only on the seed.
  std::vector<float> p(kParams, 0.f);
  uint64_t s = seed * 0x9E3779B97F4A7C15ull + 1;
  auto next = [&]() {
    s += 0x9E3779B97F4A7C15ull;
    uint64_t z = s;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
  };
  for (int l = 0; l < 4; ++l) {
    const int outs = l == 3 ? kOut : kHid;
    const double bound = std::sqrt(6.0 / kK) * (l == 3 ? 0.1 : 1.0);
    for (int i = 0; i < outs * kK; ++i) p[off_w(l) + i] = (float)((2.0 * next() - 1.0) * bound);
  }
  bool cok = cudaMemcpy(g->master, p.data(), kParams * 4, cudaMemcpyHostToDevice) == cudaSuccess;
  cok &= cudaMemset(g->grad, 0, kParams * 4) == cudaSuccess;
  cok &= cudaMemset(g->mom, 0, kParams * 4) == cudaSuccess;
  cok &= cudaMemset(g->vel, 0, kParams * 4) == cudaSuccess;
  cok &= cudaMemset(g->wf, 0, 4 * kHid * kK * 2) == cudaSuccess;
  cok &= cudaMemset(g->wb, 0, 4 * kHid * kK * 2) == cudaSuccess;
  cok &= cudaMemset(g->err, 0, 4) == cudaSuccess;
  cok &= cudaMemset(g->rec_count, 0, 4) == cudaSuccess;
  cok &= cudaFuncSetAttribute(guide_infer_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kInferSmem) == cudaSuccess;
  cok &= cudaFuncSetAttribute(guide_train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrainSmem) == cudaSuccess;
  guide_sync_bf16(g, 0);
  if (!cok || cudaDeviceSynchronize() != cudaSuccess) { guide_destroy(g); return XB_E_CUDA; }
  *out = g;
  return XB_OK;
}

void guide_destroy(Guide* g) {
  if (!g) return;
  void* ptrs[] = {g->master, g->grad, g->mom, g->vel, g->wf, g->wb, g->csum, g->loss, g->err,
                  g->recs, g->rec_count};
  for (void* q : ptrs) if (q) cudaFree(q);
  delete g;
}

float* guide_master(Guide* g) { return g->master; }
const __nv_bfloat16* guide_weights_bf16(Guide* g) { return g->wf; }
int* guide_error(Guide* g) { return g->err; }
float* guide_records(Guide* g) { return g->recs; }
int32_t* guide_record_count(Guide* g) { return g->rec_count; }
int guide_record_capacity(Guide* g) { return g->rec_cap; }
int64_t guide_steps_taken(Guide* g) { return g->t; }
const float* guide_losses(Guide* g) { return g->loss; }

void guide_sync_bf16(Guide* g, cudaStream_t s) {
  pack_bf16_kernel<<<16, 256, 0, s>>>(g->master, g->wf, g->wb);
}

void guide_reset_optimizer(Guide* g, cudaStream_t s) {
  cudaMemsetAsync(g->grad, 0, kParams * 4, s);
  cudaMemsetAsync(g->mom, 0, kParams * 4, s);
  cudaMemsetAsync(g->vel, 0, kParams * 4, s);
  g->t = 0;
}

void guide_infer(Guide* g, cudaStream_t s, const float* feats, int feat_stride, const int32_t* count, int max_rows,
                 float* lobes, int grid) {
  guide_infer_kernel<<<grid, kTile, kInferSmem, s>>>(feats, feat_stride, count, max_rows, g->wf, g->master, lobes,
                                                     g->err);
}

void guide_finalize_records(Guide* g, cudaStream_t s, const float4* L, int grid, unsigned long long* total) {
  finalize_records_kernel<<<grid, 256, 0, s>>>(g->recs, g->rec_count, g->rec_cap, L, total);
}

int guide_train(Guide* g, cudaStream_t s, const float* recs, const int32_t* rec_count, int cap, int steps,
                int batch, float lr, uint64_t seed, float alpha_fixed, int64_t total_steps) {
  steps = std::min(steps, g->max_steps);
  batch = std::max(kTile, (batch + kTile - 1) / kTile * kTile);
  const int tiles = batch / kTile;
  const float b1 = 0.9f, b2 = 0.99f;
  cudaMemsetAsync(g->csum, 0, (size_t)steps * 4, s);
  cudaMemsetAsync(g->loss, 0, (size_t)steps * 4, s);
  for (int k = 0; k < steps; ++k) {
    const uint64_t t = (uint64_t)g->t;
    weight_sum_kernel<<<tiles, kTile, 0, s>>>(recs, rec_count, cap, batch, seed, t, g->csum + k);
    TrainArgs a{recs, rec_count, cap, batch, seed, t, alpha_fixed, g->csum + k, g->wf, g->wb, g->master, g->grad,
                g->loss + k, g->err};
    guide_train_kernel<<<tiles, kTile, kTrainSmem, s>>>(a);
    g->t += 1;
    const float c1 = 1.f - (float)std::pow((double)b1, (double)g->t);
    const float c2 = 1.f - (float)std::pow((double)b2, (double)g->t);
    // cosine decay from lr to lr/10 over the planned steps (constant when none are planned)
    float lr_t = lr;
    if (total_steps > 0) {
      const double x = std::min(1.0, (double)(g->t - 1) / (double)total_steps);
      lr_t = (float)(lr * (0.1 + 0.45 * (1.0 + std::cos(3.14159265358979323846 * x))));
    }
    adam_kernel<<<64, 256, 0, s>>>(g->master, g->grad, g->mom, g->vel, g->wf, g->wb, lr_t, b1, b2, 1e-8f, c1, c2);
  }
  return cudaGetLastError() == cudaSuccess ? XB_OK : XB_E_CUDA;
}

int guide_gradient(Guide* g, cudaStream_t s, const float* recs, const int32_t* count, int n, float* grad_dev,
                   float* loss_dev) {
  const int batch = std::max(kTile, (n + kTile - 1) / kTile * kTile);
  cudaMemsetAsync(g->csum, 0, 4, s);
  weight_sum_kernel<<<batch / kTile, kTile, 0, s>>>(recs, count, n, batch, 0, 0, g->csum);
  cudaMemsetAsync(grad_dev, 0, kParams * 4, s);
  cudaMemsetAsync(loss_dev, 0, 4, s);
  TrainArgs a{recs, count, n, batch, 0, 0, -1.f, g->csum, g->wf, g->wb, g->master, grad_dev, loss_dev, g->err};
  guide_train_kernel<<<batch / kTile, kTile, kTrainSmem, s>>>(a);
  return cudaGetLastError() == cudaSuccess ? XB_OK : XB_E_CUDA;
}

}  // namespace xbg
// ── tcgen05 building-block check ───────────────────────────────────────────────────
namespace {

template <int N>
__global__ void __launch_bounds__(128) tc_gemm_kernel(const __nv_bfloat16* __restrict__ A,
                                                      const __nv_bfloat16* __restrict__ B,
                                                      float* __restrict__ D, int rows, int* err) {
  extern __shared__ __align__(1024) uint8_t dyn[];   // only pads the footprint: <= 6 CTAs per SM
  __shared__ __align__(1024) uint8_t sA[128 * 64 * 2];
  __shared__ __align__(1024) uint8_t sB[N * 64 * 2];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmem_base;
  (void)dyn;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int row0 = blockIdx.x * 128;
  for (int c = 0; c < 8; ++c) {
    uint4 v = make_uint4(0, 0, 0, 0);
    if (row0 + tid < rows) v = *reinterpret_cast<const uint4*>(A + (size_t)(row0 + tid) * 64 + c * 8);
    *reinterpret_cast<uint4*>(sA + kmajor_offset(tid, c * 8, 64)) = v;
  }
  for (int i = tid; i < N * 8; i += blockDim.x) {
    const int r = i / 8, c = i % 8;
    *reinterpret_cast<uint4*>(sB + kmajor_offset(r, c * 8, 64)) =
        *reinterpret_cast<const uint4*>(B + (size_t)r * 64 + c * 8);
  }
  if (warp == 0) {
    tmem_alloc(&tmem_base, 64);
    tmem_relinquish();
  }
  if (tid == 0) {
    mbar_init(&mbar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  fence_smem_to_async();
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tbase = tmem_base;
  if (tid == 0) {
    for (int j = 0; j < 4; ++j) {
      const uint64_t ad = smem_desc(smem_u32(sA) + j * 256, 128, 1024);
      const uint64_t bd = smem_desc(smem_u32(sB) + j * 256, 128, 1024);
      mma_bf16(tbase, ad, bd, idesc_bf16_f32(128, N), j > 0 ? 1u : 0u);
    }
    mma_commit(&mbar);
  }
  const bool done = mbar_wait(&mbar, 0);
  if (!done && lane == 0) atomicExch(err, 1);
  fence_after_sync();
  if (done) {
    for (int c = 0; c < N; c += 16) {
      float v[16];
      tmem_ld16(tbase + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
      tmem_wait_ld();
      const int r = row0 + warp * 32 + lane;
      if (r < rows)
        for (int i = 0; i < 16; ++i) D[(size_t)r * N + c + i] = v[i];
    }
  }
  fence_before_sync();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tbase, 64);
}

// The bounded completion wait of every tensor-core step, on an mbarrier that nothing completes
// (arrive = 0) or that one of its own threads completes (arrive = 1): the failed wait gives up
// after `limit` polls and reports through *err, and the kernel returns.
__global__ void wait_selftest_kernel(int arrive, uint32_t limit, int* err) {
  __shared__ __align__(8) uint64_t mbar;
  if (threadIdx.x == 0) mbar_init(&mbar, 1);
  __syncthreads();
  if (arrive && threadIdx.x == 0) mbar_arrive(&mbar);
  const bool done = mbar_wait(&mbar, 0, limit);
  if (!done && threadIdx.x == 0) atomicExch(err, 1);
}

}  // namespace

extern "C" {

int xb_selftest_wait(int32_t arrive) {
  int* derr = nullptr;
  if (cudaMalloc(&derr, sizeof(int)) != cudaSuccess) return xb::fail(XB_E_OOM, "xb_selftest_wait: out of device memory");
  int herr = 0;
  cudaError_t e = cudaMemset(derr, 0, sizeof(int));
  if (e == cudaSuccess) {
    wait_selftest_kernel<<<1, 32>>>(arrive ? 1 : 0, 1u << 14, derr);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaMemcpy(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost);
  cudaFree(derr);
  if (e != cudaSuccess) return xb::fail(XB_E_CUDA, "xb_selftest_wait: %s", cudaGetErrorString(e));
  if (herr) return xb::fail(XB_E_TIMEOUT, "xb_selftest_wait: the completion wait ran out (as asked)");
  return XB_OK;
}

int xb_tc_gemm_bf16(const uint16_t* A, const uint16_t* B, int64_t rows, int32_t n, float* D) {
  if (!A || !B || !D || rows <= 0 || rows > (1 << 24) || (n != 16 && n != 32 && n != 48 && n != 64))
    return xb::fail(XB_E_INVALID, "xb_tc_gemm_bf16: bad arguments");
  __nv_bfloat16 *dA = nullptr, *dB = nullptr;
  float* dD = nullptr;
  int* derr = nullptr;
  int rc = XB_OK;
  if (cudaMalloc(&dA, rows * 64 * 2) != cudaSuccess || cudaMalloc(&dB, (size_t)n * 64 * 2) != cudaSuccess ||
      cudaMalloc(&dD, rows * n * 4) != cudaSuccess || cudaMalloc(&derr, 4) != cudaSuccess) {
    rc = xb::fail(XB_E_OOM, "xb_tc_gemm_bf16: out of device memory");
  } else {
    cudaMemcpy(dA, A, rows * 64 * 2, cudaMemcpyHostToDevice);
    cudaMemcpy(dB, B, (size_t)n * 64 * 2, cudaMemcpyHostToDevice);
    cudaMemset(derr, 0, 4);
    const int grid = (int)((rows + 127) / 128);
    const size_t pad = 8 * 1024;
    switch (n) {
      case 16: tc_gemm_kernel<16><<<grid, 128, pad>>>(dA, dB, dD, (int)rows, derr); break;
      case 32: tc_gemm_kernel<32><<<grid, 128, pad>>>(dA, dB, dD, (int)rows, derr); break;
      case 48: tc_gemm_kernel<48><<<grid, 128, pad>>>(dA, dB, dD, (int)rows, derr); break;
      default: tc_gemm_kernel<64><<<grid, 128, pad>>>(dA, dB, dD, (int)rows, derr); break;
    }
    cudaError_t e = cudaDeviceSynchronize();
    int herr = 0;
    if (e == cudaSuccess) e = cudaMemcpy(&herr, derr, 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(D, dD, rows * n * 4, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) rc = xb::fail(XB_E_CUDA, "xb_tc_gemm_bf16: %s", cudaGetErrorString(e));
    else if (herr) rc = xb::fail(XB_E_TIMEOUT, "xb_tc_gemm_bf16: MMA completion wait timed out");
  }
  cudaFree(dA); cudaFree(dB); cudaFree(dD); cudaFree(derr);
  return rc;
}

}  // extern "C"

// ── standalone network entry points (parity tests and diagnostics) ─────────────────
namespace {

__global__ void mixture_pdf_kernel(const float* lobes, int64_t rows, const float* dirs, float* pdf) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < rows; i += (int64_t)gridDim.x * blockDim.x) {
    const float* P = lobes + i * xbg::kLobeFloats;
    pdf[i] = xbg::mix_pdf(P, dirs[3 * i], dirs[3 * i + 1], dirs[3 * i + 2]);
  }
}

__global__ void mixture_sample_kernel(const float* lobes, int64_t rows, const float* u, float* dirs, float* pdf) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < rows; i += (int64_t)gridDim.x * blockDim.x) {
    const float* L = lobes + i * xbg::kLobeFloats;
    float d[3];
    xbg::mix_sample(L, u[3 * i], u[3 * i + 1], u[3 * i + 2], d);
    dirs[3 * i] = d[0]; dirs[3 * i + 1] = d[1]; dirs[3 * i + 2] = d[2];
    pdf[i] = xbg::mix_pdf(L, d[0], d[1], d[2]);
  }
}

// Device buffers of one call, freed on every return path.
struct Scratch {
  std::vector<void*> ptrs;
  ~Scratch() { for (void* p : ptrs) cudaFree(p); }
  template <class T>
  T* alloc(size_t count) {
    void* p = nullptr;
    if (cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)) != cudaSuccess) return nullptr;
    ptrs.push_back(p);
    return static_cast<T*>(p);
  }
  template <class T>
  T* upload(const T* src, size_t count) {
    T* d = alloc<T>(count);
    if (d && cudaMemcpy(d, src, count * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess) return nullptr;
    return d;
  }
};

struct GuideHandle {
  xbg::Guide* g = nullptr;
  ~GuideHandle() { xbg::guide_destroy(g); }
};

// A network holding `params` (kParams floats), or an error status.
int make_guide(GuideHandle& h, const float* params) {
  int rc = xbg::guide_create(&h.g, 0, 0);
  if (rc != XB_OK) return xb::fail(rc, "guide: cannot create the network");
  if (cudaMemcpy(xbg::guide_master(h.g), params, xbg::kParams * 4, cudaMemcpyHostToDevice) != cudaSuccess)
    return xb::fail(XB_E_CUDA, "guide: parameter upload failed");
  xbg::guide_sync_bf16(h.g, 0);
  return XB_OK;
}

int finish(xbg::Guide* g, const char* what) {
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return xb::fail(XB_E_CUDA, "%s: %s", what, cudaGetErrorString(e));
  int herr = 0;
  if (g && cudaMemcpy(&herr, xbg::guide_error(g), 4, cudaMemcpyDeviceToHost) != cudaSuccess)
    return xb::fail(XB_E_CUDA, "%s: error word read failed", what);
  if (herr) return xb::fail(XB_E_TIMEOUT, "%s: a tensor-core completion wait ran out", what);
  return XB_OK;
}

int sm_count() {
  int dev = 0, n = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  return std::max(1, n);
}

}  // namespace

extern "C" {

int xb_guide_init_params(uint64_t seed, float* params) {
  if (!params) return xb::fail(XB_E_INVALID, "xb_guide_init_params: null output");
  GuideHandle h;
  int rc = xbg::guide_create(&h.g, seed, 0);
  if (rc != XB_OK) return xb::fail(rc, "xb_guide_init_params: cannot create the network");
  if (cudaMemcpy(params, xbg::guide_master(h.g), xbg::kParams * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
    return xb::fail(XB_E_CUDA, "xb_guide_init_params: copy failed");
  return XB_OK;
}

int xb_guide_forward(const float* params, const float* feats, int64_t rows, float* lobes) {
  if (!params || !feats || !lobes || rows <= 0 || rows > (1 << 26))
    return xb::fail(XB_E_INVALID, "xb_guide_forward: bad arguments");
  GuideHandle h;
  int rc = make_guide(h, params);
  if (rc != XB_OK) return rc;
  Scratch s;
  const int32_t n = (int32_t)rows;
  float* dF = s.upload(feats, (size_t)rows * 9);
  int32_t* dN = s.upload(&n, 1);
  float* dL = s.alloc<float>((size_t)rows * xbg::kOutRow);
  if (!dF || !dN || !dL) return xb::fail(XB_E_OOM, "xb_guide_forward: out of device memory");
  const int tiles = (int)((rows + 127) / 128);
  xbg::guide_infer(h.g, 0, dF, 9, dN, n, dL, std::min(tiles, sm_count() * 4));
  if ((rc = finish(h.g, "xb_guide_forward")) != XB_OK) return rc;
  if (cudaMemcpy(lobes, dL, (size_t)rows * xbg::kOutRow * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
    return xb::fail(XB_E_CUDA, "xb_guide_forward: copy failed");
  return XB_OK;
}

int xb_guide_loss_grad(const float* params, const float* recs, int64_t n, float* grad, float* loss) {
  if (!params || !recs || !grad || !loss || n <= 0 || n > (1 << 24))
    return xb::fail(XB_E_INVALID, "xb_guide_loss_grad: bad arguments");
  GuideHandle h;
  int rc = make_guide(h, params);
  if (rc != XB_OK) return rc;
  Scratch s;
  const int32_t cnt = (int32_t)n;
  float* dR = s.upload(recs, (size_t)n * xbg::kRecFloats);
  int32_t* dN = s.upload(&cnt, 1);
  float* dG = s.alloc<float>(xbg::kParams);
  float* dLoss = s.alloc<float>(1);
  if (!dR || !dN || !dG || !dLoss) return xb::fail(XB_E_OOM, "xb_guide_loss_grad: out of device memory");
  if (xbg::guide_gradient(h.g, 0, dR, dN, cnt, dG, dLoss) != XB_OK)
    return xb::fail(XB_E_CUDA, "xb_guide_loss_grad: launch failed");
  if ((rc = finish(h.g, "xb_guide_loss_grad")) != XB_OK) return rc;
  if (cudaMemcpy(grad, dG, xbg::kParams * 4, cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(loss, dLoss, 4, cudaMemcpyDeviceToHost) != cudaSuccess)
    return xb::fail(XB_E_CUDA, "xb_guide_loss_grad: copy failed");
  return XB_OK;
}

int xb_guide_train(const float* params, const float* recs, int64_t n, int32_t steps, int32_t batch, float lr,
                   uint64_t seed, float* params_out, float* losses) {
  if (!params || !recs || !params_out || n <= 0 || n > (1 << 24) || steps <= 0 || steps > xbg::kMaxTrainSteps ||
      batch <= 0 || batch > (1 << 24) || !(lr > 0.f))
    return xb::fail(XB_E_INVALID, "xb_guide_train: bad arguments");
  GuideHandle h;
  int rc = make_guide(h, params);
  if (rc != XB_OK) return rc;
  Scratch s;
  const int32_t cnt = (int32_t)n;
  float* dR = s.upload(recs, (size_t)n * xbg::kRecFloats);
  int32_t* dN = s.upload(&cnt, 1);
  if (!dR || !dN) return xb::fail(XB_E_OOM, "xb_guide_train: out of device memory");
  if (xbg::guide_train(h.g, 0, dR, dN, cnt, steps, batch, lr, seed, -1.f, 0) != XB_OK)
    return xb::fail(XB_E_CUDA, "xb_guide_train: launch failed");
  if ((rc = finish(h.g, "xb_guide_train")) != XB_OK) return rc;
  if (cudaMemcpy(params_out, xbg::guide_master(h.g), xbg::kParams * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
    return xb::fail(XB_E_CUDA, "xb_guide_train: copy failed");
  if (losses && cudaMemcpy(losses, xbg::guide_losses(h.g), (size_t)steps * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
    return xb::fail(XB_E_CUDA, "xb_guide_train: copy failed");
  return XB_OK;
}

int xb_guide_mixture_pdf(const float* lobes, int64_t rows, const float* dirs, float* pdf) {
  if (!lobes || !dirs || !pdf || rows <= 0 || rows > (1 << 26))
    return xb::fail(XB_E_INVALID, "xb_guide_mixture_pdf: bad arguments");
  Scratch s;
  float* dL = s.upload(lobes, (size_t)rows * xbg::kLobeFloats);
  float* dD = s.upload(dirs, (size_t)rows * 3);
  float* dP = s.alloc<float>((size_t)rows);
  if (!dL || !dD || !dP) return xb::fail(XB_E_OOM, "xb_guide_mixture_pdf: out of device memory");
  mixture_pdf_kernel<<<sm_count() * 8, 256>>>(dL, rows, dD, dP);
  int rc = finish(nullptr, "xb_guide_mixture_pdf");
  if (rc != XB_OK) return rc;
  if (cudaMemcpy(pdf, dP, (size_t)rows * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
    return xb::fail(XB_E_CUDA, "xb_guide_mixture_pdf: copy failed");
  return XB_OK;
}

int xb_guide_mixture_sample(const float* lobes, int64_t rows, const float* u, float* dirs, float* pdf) {
  if (!lobes || !u || !dirs || !pdf || rows <= 0 || rows > (1 << 26))
    return xb::fail(XB_E_INVALID, "xb_guide_mixture_sample: bad arguments");
  Scratch s;
  float* dL = s.upload(lobes, (size_t)rows * xbg::kLobeFloats);
  float* dU = s.upload(u, (size_t)rows * 3);
  float* dD = s.alloc<float>((size_t)rows * 3);
  float* dP = s.alloc<float>((size_t)rows);
  if (!dL || !dU || !dD || !dP) return xb::fail(XB_E_OOM, "xb_guide_mixture_sample: out of device memory");
  mixture_sample_kernel<<<sm_count() * 8, 256>>>(dL, rows, dU, dD, dP);
  int rc = finish(nullptr, "xb_guide_mixture_sample");
  if (rc != XB_OK) return rc;
  if (cudaMemcpy(dirs, dD, (size_t)rows * 12, cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(pdf, dP, (size_t)rows * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
    return xb::fail(XB_E_CUDA, "xb_guide_mixture_sample: copy failed");
  return XB_OK;
}

}  // extern "C"
