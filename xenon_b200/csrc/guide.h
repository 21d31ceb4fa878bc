// guide.h — the path-guiding network's device state and launches (implemented in guide.cu).
//
// Network: 64 encoded features -> 3 x 64 ReLU -> 48 outputs (8 von Mises-Fisher lobes: mean
// direction, concentration, mixture weight). BF16 weights and activations on the tensor cores
// (tcgen05) with FP32 accumulation in TMEM; FP32 master weights and Adam moments.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace xbg {

constexpr int kIn = 64, kHid = 64, kOut = 48, kLobes = 8;
constexpr int kLobeFloats = 40;  // 8 x (mu xyz, kappa, weight)
constexpr int kSelect = 40;      // raw output holding the selection logit
constexpr int kOutRow = 41;      // forward output per row: the lobes, then the selection probability
// Range of the learned selection probability. A vertex's importance ratio p_bsdf / p stays below
// 1 / (1 - kAMax): 2.5 here. Wider ranges (up to 0.95, ratio 20) gave the same bulk improvement
// on config 4 but let a rare caustic path's weight compound over several guided vertices into a
// single-sample firefly (three sample blocks: pooled relMSE ratio 0.32 at 0.95, 1.08 at 0.6).
#ifndef XB_GUIDE_AMAX
#define XB_GUIDE_AMAX 0.6f
#endif
constexpr float kAMin = 0.05f, kAMax = XB_GUIDE_AMAX;
// Training record (floats): 0-8 features (position in [0,1]^3, normal, outgoing direction),
// 9-11 sampled direction omega, 12 weight c (set once the path has finished), 13 path index
// (int bits), 14-16 throughput before the vertex, 17-19 path radiance before the continuation,
// 20 density of the BSDF sampler at omega (< 0: the loss uses q alone), 21-23 unused.
constexpr int kRecFloats = 24;
// Parameter vector: W0 b0 W1 b1 W2 b2 W3 b3, each W row-major [out][in].
__host__ __device__ constexpr int off_w(int l) { return 4160 * l; }
__host__ __device__ constexpr int off_b(int l) { return 4160 * l + (l == 3 ? 3072 : 4096); }
constexpr int kParams = 15600;
constexpr int kMaxTrainSteps = 4096;   // Adam steps per guide_train call

struct Guide;

// `rec_cap` training records are allocated with the network (0: none).
int guide_create(Guide** out, uint64_t seed, int rec_cap);
void guide_destroy(Guide* g);
// Lobes and selection probability (kOutRow per row) for rows [0, min(*count, max_rows)) of feats
// (9 floats used per row, `feat_stride` apart). Device-side count: no host synchronisation.
void guide_infer(Guide* g, cudaStream_t s, const float* feats, int feat_stride, const int32_t* count, int max_rows,
                 float* lobes, int grid);
// `steps` Adam steps on records [0, min(*rec_count, cap)): each step takes batch / 128 tiles of 128
// consecutive records at random starts (the whole set, in order, when there are no more records
// than the batch).
// alpha_fixed: the selection probability the renderer samples with (< 0: the network's own output,
// which is then trained too). total_steps > 0: the learning rate follows a cosine from lr down
// to lr / 10 over that many Adam steps (counted from the network's first step); 0: constant lr.
int guide_train(Guide* g, cudaStream_t s, const float* recs, const int32_t* rec_count, int cap, int steps,
                int batch, float lr, uint64_t seed, float alpha_fixed, int64_t total_steps);
// Loss and gradient (no update) over records [0, min(*count, n)) into grad_dev[kParams], loss_dev[1].
int guide_gradient(Guide* g, cudaStream_t s, const float* recs, const int32_t* count, int n, float* grad_dev,
                   float* loss_dev);
// Sets each record's weight c from the path radiance L (float4 per path) after its wave and adds
// the record count to *total.
void guide_finalize_records(Guide* g, cudaStream_t s, const float4* L, int grid, unsigned long long* total);
void guide_reset_optimizer(Guide* g, cudaStream_t s);
void guide_sync_bf16(Guide* g, cudaStream_t s);   // after writing master: rebuild the BF16 copies

float* guide_master(Guide* g);                     // device FP32 parameters
const __nv_bfloat16* guide_weights_bf16(Guide* g); // device forward weights, 4 x [64][64]
int* guide_error(Guide* g);                        // device error word (a bounded wait ran out)
float* guide_records(Guide* g);
int32_t* guide_record_count(Guide* g);
int guide_record_capacity(Guide* g);
int64_t guide_steps_taken(Guide* g);
const float* guide_losses(Guide* g);               // device, per step of the last guide_train call

}  // namespace xbg
