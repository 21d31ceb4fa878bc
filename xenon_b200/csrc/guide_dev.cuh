// guide_dev.cuh — device pieces of the path-guiding network shared by the standalone network
// kernels (guide.cu) and the fused guided shade kernel (renderer.cu): input encoding, the
// 128-row tcgen05 layer chain with its epilogues, the lobe mapping, and the von Mises-Fisher
// mixture's pdf and sampling. No reference counterpart (the reference has no learned part);
// the FP64 restatement of every formula here is oracle/guide_ref.py.
#pragma once

#include <cuda_bf16.h>

#include <cstdint>

#include "guide.h"
#include "tc05.cuh"

namespace xbg {

constexpr int kK = 64;                                // K of every forward layer
constexpr int kTile = 128;                            // rows per MMA chain (one per thread)
constexpr float kGuidePi = 3.14159265358979323846f;
constexpr uint32_t kTileBytes = kTile * kK * 2;       // 128 x 64 bf16 activations
constexpr uint32_t kWBytes = kHid * kK * 2;           // 64 x 64 bf16 weights
constexpr uint32_t kW3fBytes = kOut * kK * 2;         // 48 x 64 bf16 (output layer, forward)
constexpr uint32_t kW3bBytes = kHid * kOut * 2;       // 64 x 48 bf16 (output layer, transposed)
constexpr uint32_t kFwdWeightBytes = 3 * kWBytes + kW3fBytes;
constexpr int kBiasFloats = 3 * kHid + kOut;

__device__ __forceinline__ void store8_bf16(uint8_t* tile, int r, int k0, int K, const float* v) {
  __nv_bfloat162 h[4];
  for (int i = 0; i < 4; ++i) h[i] = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
  *reinterpret_cast<uint4*>(tile + xbd::kmajor_offset(r, k0, K)) = *reinterpret_cast<const uint4*>(h);
}

// (lo, hi) -> bf16x2 (lo in the low half), each max(x, 0) rounded to nearest: one
// cvt.rn.relu.bf16x2.f32, the same bits as rounding fmaxf(x, 0.f).
__device__ __forceinline__ uint32_t relu_bf16x2(float lo, float hi) {
  uint32_t r;
  asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
  return r;
}

__device__ __forceinline__ float load_bf16(const uint8_t* tile, int r, int k, int K) {
  return __bfloat162float(*reinterpret_cast<const __nv_bfloat16*>(tile + xbd::kmajor_offset(r, k, K)));
}

// Row-major bf16 [rows][K] in global memory -> core-matrix tile in shared memory (block-wide).
__device__ __forceinline__ void load_matrix(uint8_t* dst, const __nv_bfloat16* src, int rows, int K) {
  const int chunks = K / 8;
  for (int i = threadIdx.x; i < rows * chunks; i += blockDim.x) {
    const int r = i / chunks, c = i % chunks;
    *reinterpret_cast<uint4*>(dst + xbd::kmajor_offset(r, c * 8, K)) =
        *reinterpret_cast<const uint4*>(src + (size_t)r * K + c * 8);
  }
}

// Forward weights (wf: 4 x [out][64] bf16) and biases (from the FP32 master vector) into shared
// memory: W0 W1 W2 at kWBytes each, then W3; biases b0 b1 b2 b3 contiguous.
__device__ __forceinline__ void load_forward_weights(uint8_t* sW, float* sBias, const __nv_bfloat16* wf,
                                                     const float* master) {
  for (int l = 0; l < 3; ++l) load_matrix(sW + l * kWBytes, wf + l * kHid * kK, kHid, kK);
  load_matrix(sW + 3 * kWBytes, wf + 3 * kHid * kK, kOut, kK);
  for (int i = threadIdx.x; i < kBiasFloats; i += blockDim.x) {
    const int l = i < 3 * kHid ? i / kHid : 3;
    const int j = i < 3 * kHid ? i % kHid : i - 3 * kHid;
    sBias[i] = master[off_b(l) + j];
  }
}

// The 64 input features of one row into the A tile: sin/cos(2^k pi x) of the position in
// [0,1]^3 (k < 6), the normal (k < 2) and the outgoing direction (k < 2), then p xyz and 1.
// f: p01 xyz, n xyz, wo xyz. One sincospif per coordinate; the higher octaves follow from the
// double-angle identities sin 2a = 2 sin a cos a, cos 2a = 1 - 2 sin^2 a (error doubling per
// octave stays far below the bf16 rounding of the result). kFast: __sincosf(pi x) instead
// (|pi x| <= pi here: absolute error below 1e-6 before the doublings, 3e-5 after the fifth,
// against the bf16 step of 4e-3 at 1).
template <bool kFast = false>
__device__ __forceinline__ void encode_row(const float* f, uint8_t* tile, int r) {
  float x[kIn];
#pragma unroll
  for (int c = 0; c < 9; ++c) {
    const int nf = c < 3 ? 6 : 2;
    const int o = c < 3 ? 12 * c : 36 + 4 * (c - 3);
    float s, co;
    if (kFast) __sincosf(kGuidePi * f[c], &s, &co);
    else sincospif(f[c], &s, &co);
#pragma unroll
    for (int k = 0; k < nf; ++k) {
      x[o + 2 * k] = s;
      x[o + 2 * k + 1] = co;
      const float s2 = 2.f * s * co;
      co = 1.f - 2.f * s * s;
      s = s2;
    }
  }
  x[60] = f[0]; x[61] = f[1]; x[62] = f[2]; x[63] = 1.f;
#pragma unroll
  for (int k0 = 0; k0 < kIn; k0 += 8) store8_bf16(tile, r, k0, kK, x + k0);
}

// One CTA of 128 threads driving 128-row MMA chains: TMEM (64 columns) and an mbarrier.
// Every wait is bounded; a wait that runs out marks the whole CTA failed (ok = false, the
// device error word set) and every later step is skipped uniformly.
struct Mma {
  uint32_t tmem;
  uint64_t* mbar;
  uint32_t phase;
  int* err;
  bool ok;

  // Shared-memory writes of this CTA become visible to the tensor core; TMEM reads of the
  // previous step are ordered before the next MMA.
  __device__ __forceinline__ void sync_before() {
    xbd::fence_smem_to_async();
    xbd::fence_before_sync();
    __syncthreads();
    xbd::fence_after_sync();
  }
  // D[128 x N] = A[128 x K] * B[N x K]^T into TMEM columns [0, N).
  __device__ __forceinline__ void run(uint32_t a_addr, uint32_t b_addr, int K, int N) {
    if (threadIdx.x == 0) {
      const uint32_t sbo = (uint32_t)(K / 8) * 128;
      for (int j = 0; j < K / 16; ++j)
        xbd::mma_bf16(tmem, xbd::smem_desc(a_addr + j * 256, 128, sbo), xbd::smem_desc(b_addr + j * 256, 128, sbo),
                      xbd::idesc_bf16_f32(kTile, N), j > 0 ? 1u : 0u);
      xbd::mma_commit(mbar);
    }
    const bool done = xbd::mbar_wait(mbar, phase);
    phase ^= 1u;
    xbd::fence_after_sync();
    if (__syncthreads_or(done ? 0 : 1)) {
      ok = false;
      if (threadIdx.x == 0) atomicExch(err, 1);
    }
  }
  // Training's backward step of one layer, as one commit: the weight gradient
  // D[128 x 64] = delta^T a over the tile's 128 rows into TMEM columns [64, 128) (row o < O of D
  // is dW[o][0..64); rows O..127 read other bytes of the tile and are not used), and with
  // next_addr != 0 the next layer's error signal delta W_l (next_addr: W_l^T [64][O]) into
  // columns [0, 64). delta: [row][o] bf16 K-major over O columns at d_addr, which the weight
  // gradient reads as an MN-major operand (o contiguous), as it reads the activations a:
  // [row][i] over 64 columns at a_addr. MN-major descriptors: SBO = byte stride between 8-element
  // blocks along M (or N), LBO = byte stride between 8-row blocks along K.
  __device__ __forceinline__ void run_backward(uint32_t d_addr, int O, uint32_t a_addr, uint32_t next_addr) {
    if (threadIdx.x == 0) {
      const uint32_t d_rows = (uint32_t)(O / 8) * 128, a_rows = (uint32_t)(kK / 8) * 128;
      const uint32_t idesc_w = xbd::idesc_bf16_f32(kTile, kK) | (1u << 15) | (1u << 16);
      for (int j = 0; j < kTile / 16; ++j)
        xbd::mma_bf16(tmem + 64, xbd::smem_desc(d_addr + j * 2 * d_rows, d_rows, 128),
                      xbd::smem_desc(a_addr + j * 2 * a_rows, a_rows, 128), idesc_w, j > 0 ? 1u : 0u);
      if (next_addr) {
        const uint32_t sbo = (uint32_t)(O / 8) * 128;
        for (int j = 0; j < O / 16; ++j)
          xbd::mma_bf16(tmem, xbd::smem_desc(d_addr + j * 256, 128, sbo), xbd::smem_desc(next_addr + j * 256, 128, sbo),
                        xbd::idesc_bf16_f32(kTile, kHid), j > 0 ? 1u : 0u);
      }
      xbd::mma_commit(mbar);
    }
    const bool done = xbd::mbar_wait(mbar, phase);
    phase ^= 1u;
    xbd::fence_after_sync();
    if (__syncthreads_or(done ? 0 : 1)) {
      ok = false;
      if (threadIdx.x == 0) atomicExch(err, 1);
    }
  }
  // This thread's row (TMEM lane = threadIdx.x), columns [c, c + 16).
  __device__ __forceinline__ void load16(int c, float* v) const {
    const uint32_t warp = threadIdx.x >> 5;
    xbd::tmem_ld16(tmem + ((warp * 32) << 16) + (uint32_t)c, v);
    xbd::tmem_wait_ld();
  }
};

// ncols: TMEM columns of the CTA (64; training 128: its weight gradients use columns 64..127).
__device__ __forceinline__ void mma_setup(uint32_t* tmem_slot, uint64_t* mbar, uint32_t ncols = 64) {
  if ((threadIdx.x >> 5) == 0) {
    xbd::tmem_alloc(tmem_slot, ncols);
    xbd::tmem_relinquish();
  }
  if (threadIdx.x == 0) {
    xbd::mbar_init(mbar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  xbd::fence_before_sync();
  __syncthreads();
  xbd::fence_after_sync();
}

__device__ __forceinline__ void mma_teardown(uint32_t tmem, uint32_t ncols = 64) {
  xbd::fence_before_sync();
  __syncthreads();
  if ((threadIdx.x >> 5) == 0) xbd::tmem_dealloc(tmem, ncols);
}

// Hidden-layer epilogue: this thread's row of TMEM + bias, ReLU, to bf16 in `dst`.
__device__ __forceinline__ void hidden_epilogue(const Mma& m, const float* bias, uint8_t* dst) {
  const int r = threadIdx.x;
#pragma unroll
  for (int c = 0; c < kHid; c += 16) {
    float v[16];
    m.load16(c, v);
    uint32_t h[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) h[i] = relu_bf16x2(v[2 * i] + bias[c + 2 * i], v[2 * i + 1] + bias[c + 2 * i + 1]);
    *reinterpret_cast<uint4*>(dst + xbd::kmajor_offset(r, c, kK)) = make_uint4(h[0], h[1], h[2], h[3]);
    *reinterpret_cast<uint4*>(dst + xbd::kmajor_offset(r, c + 8, kK)) = make_uint4(h[4], h[5], h[6], h[7]);
  }
}

// Runs the 4 layers on the encoded tile `sA` (overwritten by the hidden activations) and leaves
// this thread's 48 raw outputs (bias added) in `raw`. Uniform across the CTA.
__device__ __forceinline__ void forward_tile(Mma& m, uint8_t* sA, const uint8_t* sW, const float* sBias,
                                             float* raw) {
  const uint32_t aA = xbd::smem_u32(sA);
#pragma unroll 1
  for (int l = 0; l < 3; ++l) {
    m.sync_before();
    m.run(aA, xbd::smem_u32(sW + l * kWBytes), kK, kHid);
    if (!m.ok) return;
    hidden_epilogue(m, sBias + l * kHid, sA);
  }
  m.sync_before();
  m.run(aA, xbd::smem_u32(sW + 3 * kWBytes), kK, kOut);
  if (!m.ok) return;
#pragma unroll
  for (int c = 0; c < kOut; c += 16) m.load16(c, raw + c);
#pragma unroll
  for (int i = 0; i < kOut; ++i) raw[i] += sBias[3 * kHid + i];
}

// Lobe k from raw[5k .. 5k+4]: mu = m / sqrt(|m|^2 + 1e-8), kappa = exp(clamp(raw, -4, 6)),
// weights = softmax. Writes mu xyz, kappa, w per lobe (stride 5) to `out`. kFast: exponentials
// and the reciprocal through the hardware approximations (__expf, __fdividef: a few ulp), as the
// renderer's guided bounce evaluates them; training keeps the correctly rounded forms.
template <bool kFast = false>
__device__ __forceinline__ void raw_to_lobes(const float* raw, float* out) {
  float mx = -3.0e38f;
#pragma unroll
  for (int k = 0; k < kLobes; ++k) mx = fmaxf(mx, raw[5 * k + 4]);
  float sum = 0.f;
  float e[kLobes];
#pragma unroll
  for (int k = 0; k < kLobes; ++k) {
    e[k] = kFast ? __expf(raw[5 * k + 4] - mx) : expf(raw[5 * k + 4] - mx);
    sum += e[k];
  }
  const float inv = kFast ? __fdividef(1.f, sum) : 1.f / sum;
#pragma unroll
  for (int k = 0; k < kLobes; ++k) {
    const float* m = raw + 5 * k;
    const float rs = rsqrtf(m[0] * m[0] + m[1] * m[1] + m[2] * m[2] + 1e-8f);
    out[5 * k] = m[0] * rs;
    out[5 * k + 1] = m[1] * rs;
    out[5 * k + 2] = m[2] * rs;
    const float lk = fminf(fmaxf(m[3], -4.f), 6.f);
    out[5 * k + 3] = kFast ? __expf(lk) : expf(lk);
    out[5 * k + 4] = e[k] * inv;
  }
}

// Probability of sampling the network at the vertex: kAMin + (kAMax - kAMin) sigmoid(raw[kSelect]).
template <bool kFast = false>
__device__ __forceinline__ float selection(const float* raw) {
  return kFast ? kAMin + __fdividef(kAMax - kAMin, 1.f + __expf(-raw[kSelect]))
               : kAMin + (kAMax - kAMin) / (1.f + expf(-raw[kSelect]));
}

// kappa / (2 pi (1 - exp(-2 kappa))): the vMF density's normalisation on the unit sphere.
__device__ __forceinline__ float vmf_norm(float kappa) {
  return kappa / (2.f * kGuidePi * (-expm1f(-2.f * kappa)));
}
// The same through __expf / __fdividef. kappa >= e^-4 here, so 1 - e^{-2 kappa} >= 0.036 and
// its absolute error of a few 1e-7 stays below 1e-5 relative.
__device__ __forceinline__ float vmf_norm_fast(float kappa) {
  return __fdividef(kappa, 2.f * kGuidePi * (1.f - __expf(-2.f * kappa)));
}

// Mixture pdf (per steradian) of the unit direction (x, y, z), from the lobes as raw_to_lobes
// writes them (mu xyz, kappa, w per lobe):
//   q = sum_k w_k kappa_k / (2 pi (1 - e^{-2 kappa_k})) e^{kappa_k (mu_k . w - 1)}
// The renderer samples with mix_sample and weighs with this pdf; both read the same stored
// lobes, so the pdf is the sampler's density up to the rounding of the approximations.
__device__ __forceinline__ float mix_pdf(const float* L5, float x, float y, float z) {
  float q = 0.f;
#pragma unroll
  for (int k = 0; k < kLobes; ++k) {
    const float* L = L5 + 5 * k;
    const float c = L[0] * x + L[1] * y + L[2] * z;
    q += L[4] * vmf_norm_fast(L[3]) * __expf(L[3] * (c - 1.f));
  }
  return q;
}

// A direction from the mixture: u0 picks the lobe by its weight, u1 the angle to the mean
// (inverse CDF of the vMF: cos = 1 + log(u1 + (1 - u1) e^{-2 kappa}) / kappa), u2 the azimuth.
__device__ __forceinline__ void mix_sample(const float* L5, float u0, float u1, float u2, float* d) {
  int k = 0;
  float cdf = L5[4];
  while (k < kLobes - 1 && u0 > cdf) {
    ++k;
    cdf += L5[5 * k + 4];
  }
  const float* L = L5 + 5 * k;
  const float kp = L[3];
  float c = 1.f + __fdividef(__logf(u1 + (1.f - u1) * __expf(-2.f * kp)), kp);
  c = fminf(fmaxf(c, -1.f), 1.f);
  const float s = sqrtf(fmaxf(0.f, 1.f - c * c));
  float sp, cp;
  sincospif(2.f * u2, &sp, &cp);
  const float mx = L[0], my = L[1], mz = L[2];
  // t = normalize(m x a), a = (0,1,0) when |m.x| > 0.9 else (1,0,0); b = m x t
  float tx, ty, tz;
  if (fabsf(mx) > 0.9f) { tx = -mz; ty = 0.f; tz = mx; }
  else { tx = 0.f; ty = mz; tz = -my; }
  const float ti = rsqrtf(tx * tx + ty * ty + tz * tz);
  tx *= ti; ty *= ti; tz *= ti;
  const float bx = my * tz - mz * ty, by = mz * tx - mx * tz, bz = mx * ty - my * tx;
  d[0] = c * mx + s * (cp * tx + sp * bx);
  d[1] = c * my + s * (cp * ty + sp * by);
  d[2] = c * mz + s * (cp * tz + sp * bz);
}

}  // namespace xbg
