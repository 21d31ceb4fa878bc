// guide.cu — the path-guiding network on the B200 tensor cores (tcgen05, BF16 in, FP32 in TMEM).
//
// This translation unit is compiled with FMA contraction allowed (it is not part of the
// reference-exact path). Kernels:
//   tc_gemm_kernel   one 128-row tile of D = A * B^T (K = 64): the building block of every layer,
//                    exposed as xb_tc_gemm_bf16 so tests can check the MMA path on its own.

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>

#include "../../include/xenon_b200.h"
#include "capi_common.h"
#include "tc05.cuh"

using namespace xbd;

namespace {

constexpr int kK = 64;             // inner dimension of every layer
constexpr int kTileRows = 128;     // MMA M

// D[rows x N] = A[rows x 64] * B[N x 64]^T; one CTA per 128-row tile, 4 warps.
template <int N>
__global__ void __launch_bounds__(128) tc_gemm_kernel(const __nv_bfloat16* __restrict__ A,
                                                      const __nv_bfloat16* __restrict__ B,
                                                      float* __restrict__ D, int rows, int* err) {
  extern __shared__ __align__(1024) uint8_t dyn[];   // only pads the footprint: <= 7 CTAs per SM
  __shared__ __align__(1024) uint8_t sA[kTileRows * kK * 2];
  __shared__ __align__(1024) uint8_t sB[N * kK * 2];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmem_base;
  (void)dyn;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int row0 = blockIdx.x * kTileRows;
  // A tile: thread t owns row t (8 chunks of 8 bf16 = 16 B)
  for (int c = 0; c < kK / 8; ++c) {
    uint4 v = make_uint4(0, 0, 0, 0);
    if (row0 + tid < rows) v = *reinterpret_cast<const uint4*>(A + (size_t)(row0 + tid) * kK + c * 8);
    *reinterpret_cast<uint4*>(sA + kmajor_offset(tid, c * 8, kK)) = v;
  }
  for (int i = tid; i < N * (kK / 8); i += blockDim.x) {
    const int r = i / (kK / 8), c = i % (kK / 8);
    *reinterpret_cast<uint4*>(sB + kmajor_offset(r, c * 8, kK)) =
        *reinterpret_cast<const uint4*>(B + (size_t)r * kK + c * 8);
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
    const uint32_t sbo = (kK / 8) * 128;
    for (int j = 0; j < kK / 16; ++j) {
      const uint64_t ad = smem_desc(smem_u32(sA) + j * 256, 128, sbo);
      const uint64_t bd = smem_desc(smem_u32(sB) + j * 256, 128, sbo);
      mma_bf16(tbase, ad, bd, idesc_bf16_f32(kTileRows, N), j > 0 ? 1u : 0u);
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

}  // namespace

extern "C" {

// Diagnostic entry point: D = A * B^T with A [rows x 64] and B [n x 64] bf16 (row-major, host
// memory), D [rows x n] f32; n in {16, 32, 48, 64}. Runs one tcgen05 tile per 128 rows.
int xb_tc_gemm_bf16(const uint16_t* A, const uint16_t* B, int64_t rows, int32_t n, float* D) {
  if (!A || !B || !D || rows <= 0 || rows > (1 << 24) || (n != 16 && n != 32 && n != 48 && n != 64))
    return xb::fail(XB_E_INVALID, "xb_tc_gemm_bf16: bad arguments");
  __nv_bfloat16 *dA = nullptr, *dB = nullptr;
  float* dD = nullptr;
  int* derr = nullptr;
  int rc = XB_OK;
  if (cudaMalloc(&dA, rows * kK * 2) != cudaSuccess || cudaMalloc(&dB, (size_t)n * kK * 2) != cudaSuccess ||
      cudaMalloc(&dD, rows * n * 4) != cudaSuccess || cudaMalloc(&derr, 4) != cudaSuccess) {
    rc = xb::fail(XB_E_OOM, "xb_tc_gemm_bf16: out of device memory");
  } else {
    cudaMemcpy(dA, A, rows * kK * 2, cudaMemcpyHostToDevice);
    cudaMemcpy(dB, B, (size_t)n * kK * 2, cudaMemcpyHostToDevice);
    cudaMemset(derr, 0, 4);
    const int grid = (int)((rows + kTileRows - 1) / kTileRows);
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
