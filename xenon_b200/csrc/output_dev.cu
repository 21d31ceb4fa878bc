// output_dev.cu — the output stage on the device, right after accumulation: the 8-bit pixels the
// reference writes to its PNG (src/main.cpp:24-32: clamp, gamma 1/2.2, times 255.99, truncated,
// rows flipped on write) and its blur-residual noise statistics (ImageNoiseEstimator,
// src/math/image.h:35-118), over the mean image as xb_resolve lays it out, without copying the
// image to the host. The host form (image_out.cpp) states the same steps; both follow the
// reference's float operations in its order (this translation unit is compiled without FMA
// contraction and with IEEE division and square root), so the per-pixel values are the host's.
// Sums are FP64 as in the reference, reduced per block and then over blocks in index order; the
// order statistics (median, 95th percentile at floor(p (n - 1))) are exact: a radix select on
// the bit patterns of the non-negative residuals (two 16-bit digits, histograms on the device,
// the digit choice on the host).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/xenon_b200.h"
#include "capi_common.h"
#include "output_dev.h"

namespace xb {
namespace {

constexpr int kThreads = 256;
constexpr uint32_t kInvalid = 0xffffffffu;   // a residual left out (edge, or image border)

__global__ void rgb8_kernel(const float* __restrict__ img, int W, int H, uint8_t* __restrict__ out) {
  const int64_t row = (int64_t)W * 3, n = row * H;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = i / row, c = i - r * row;
    const float v = img[(H - 1 - r) * row + c];
    const float g = powf(fminf(fmaxf(v, 0.f), 1.f), 1.f / 2.2f);
    out[i] = (uint8_t)(255.99f * g);
  }
}

// Block sums of FP64 values, one per block (thread 0 writes), summed in a fixed tree order.
__device__ __forceinline__ double block_sum(double v, double* sh) {
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int s = kThreads / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
    __syncthreads();
  }
  const double r = sh[0];
  __syncthreads();
  return r;
}

__global__ void __launch_bounds__(kThreads) lum_kernel(const float* __restrict__ img, int64_t n,
                                                       float* __restrict__ lum, double* __restrict__ part) {
  __shared__ double sh[kThreads];
  double acc = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float l = 0.2126f * img[3 * i] + 0.7152f * img[3 * i + 1] + 0.0722f * img[3 * i + 2];
    lum[i] = l;
    acc += (double)l;
  }
  const double s = block_sum(acc, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// Interior pixel (x, y) away from strong edges: |lum - blur| / sqrt(blur^2 + eps) into rel (as
// bits), else kInvalid; per block the FP64 sums of (lum - blur)^2 / den and of the residuals, the
// count and the largest residual.
__global__ void __launch_bounds__(kThreads) residual_kernel(const float* __restrict__ lum, int W, int H, float thr,
                                                            float eps, uint32_t* __restrict__ rel,
                                                            double* __restrict__ part, int* __restrict__ cnt,
                                                            unsigned int* __restrict__ amax) {
  __shared__ double sh[kThreads];
  const int64_t n = (int64_t)W * H;
  double sq = 0.0, ab = 0.0;
  int c = 0;
  float mx = 0.f;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(i % W), y = (int)(i / W);
    uint32_t out = kInvalid;
    if (x >= 1 && x < W - 1 && y >= 1 && y < H - 1) {
      const float gx = 0.5f * (lum[i + 1] - lum[i - 1]);
      const float gy = 0.5f * (lum[i + W] - lum[i - W]);
      if (!(sqrtf(gx * gx + gy * gy) >= thr)) {
        // 3x3 binomial blur, terms added row by row (all neighbours in the image: interior pixel)
        float s = 0.f;
        s += 1.f * lum[i - W - 1]; s += 2.f * lum[i - W]; s += 1.f * lum[i - W + 1];
        s += 2.f * lum[i - 1];     s += 4.f * lum[i];     s += 2.f * lum[i + 1];
        s += 1.f * lum[i + W - 1]; s += 2.f * lum[i + W]; s += 1.f * lum[i + W + 1];
        const float blur = s / 16.f;
        const float d = lum[i] - blur;
        const float den = blur * blur + eps;
        const float a = fabsf(d) / sqrtf(den);
        sq += (double)((d * d) / den);
        ab += (double)a;
        ++c;
        mx = fmaxf(mx, a);
        out = __float_as_uint(a);
      }
    }
    rel[i] = out;
  }
  const double s1 = block_sum(sq, sh);
  const double s2 = block_sum(ab, sh);
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = s1;
    part[2 * blockIdx.x + 1] = s2;
  }
  for (int off = 16; off > 0; off >>= 1) {
    c += __shfl_xor_sync(0xffffffffu, c, off);
    mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, off));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(cnt, c);
    atomicMax(amax, __float_as_uint(mx));   // non-negative floats order as their bits
  }
}

// Histogram of one 16-bit digit of the valid residuals' bits: the high digit (prefix < 0), or
// the low digit of those whose high digit is `prefix`.
__global__ void digit_hist_kernel(const uint32_t* __restrict__ rel, int64_t n, int prefix, unsigned int* __restrict__ hist) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t b = rel[i];
    if (b == kInvalid) continue;
    if (prefix < 0) atomicAdd(hist + (b >> 16), 1u);
    else if ((int)(b >> 16) == prefix) atomicAdd(hist + (b & 0xffffu), 1u);
  }
}

struct Scratch {
  void* p = nullptr;
  ~Scratch() { if (p) cudaFree(p); }
};

}  // namespace

int device_output_stage(const float* d_img, int W, int H, int num_sms, cudaStream_t s, uint8_t* rgb8,
                        xb_noise_stats* out) {
  const int64_t n = (int64_t)W * H;
  const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((n + kThreads - 1) / kThreads, (int64_t)num_sms * 8));
  auto ck = [](cudaError_t e) { return e == cudaSuccess; };
  if (rgb8) {
    Scratch d8;
    if (!ck(cudaMalloc(&d8.p, (size_t)n * 3))) return fail(XB_E_OOM, "output stage: out of device memory");
    rgb8_kernel<<<blocks, kThreads, 0, s>>>(d_img, W, H, static_cast<uint8_t*>(d8.p));
    if (!ck(cudaMemcpyAsync(rgb8, d8.p, (size_t)n * 3, cudaMemcpyDeviceToHost, s)) || !ck(cudaStreamSynchronize(s)))
      return fail(XB_E_CUDA, "output stage: %s", cudaGetErrorString(cudaGetLastError()));
  }
  if (!out) return XB_OK;
  std::memset(out, 0, sizeof(*out));
  if (W <= 2 || H <= 2) return XB_OK;   // no interior pixel
  out->total_interior_pixel_count = (W - 2) * (H - 2);
  // scratch: luminance and residual bits (n each), block sums, count and maximum, one histogram
  const size_t b_lum = (size_t)n * 4, b_part = (size_t)blocks * 2 * 8, b_hist = 65536 * 4;
  Scratch sc;
  if (!ck(cudaMalloc(&sc.p, 2 * b_lum + b_part + 256 + b_hist))) return fail(XB_E_OOM, "output stage: out of device memory");
  char* base = static_cast<char*>(sc.p);
  float* lum = reinterpret_cast<float*>(base);
  uint32_t* rel = reinterpret_cast<uint32_t*>(base + b_lum);
  double* part = reinterpret_cast<double*>(base + 2 * b_lum);
  int* cnt = reinterpret_cast<int*>(base + 2 * b_lum + b_part);
  unsigned int* amax = reinterpret_cast<unsigned int*>(cnt + 1);
  unsigned int* hist = reinterpret_cast<unsigned int*>(base + 2 * b_lum + b_part + 256);
  std::vector<double> hp((size_t)blocks * 2);
  lum_kernel<<<blocks, kThreads, 0, s>>>(d_img, n, lum, part);
  if (!ck(cudaMemcpyAsync(hp.data(), part, (size_t)blocks * 8, cudaMemcpyDeviceToHost, s)) || !ck(cudaStreamSynchronize(s)))
    return fail(XB_E_CUDA, "output stage: %s", cudaGetErrorString(cudaGetLastError()));
  double sum = 0.0;
  for (int b = 0; b < blocks; ++b) sum += hp[b];
  out->avg_luminance = (float)(sum / (double)n);
  out->edge_threshold = std::max(1e-6f, out->avg_luminance * 0.1f);
  out->epsilon = std::max(1e-8f, out->avg_luminance * out->avg_luminance * 1e-4f);
  if (!ck(cudaMemsetAsync(cnt, 0, 8, s))) return fail(XB_E_CUDA, "output stage: memset");
  residual_kernel<<<blocks, kThreads, 0, s>>>(lum, W, H, out->edge_threshold, out->epsilon, rel, part, cnt, amax);
  int ca[2] = {0, 0};
  if (!ck(cudaMemcpyAsync(hp.data(), part, b_part, cudaMemcpyDeviceToHost, s)) ||
      !ck(cudaMemcpyAsync(ca, cnt, 8, cudaMemcpyDeviceToHost, s)) || !ck(cudaStreamSynchronize(s)))
    return fail(XB_E_CUDA, "output stage: %s", cudaGetErrorString(cudaGetLastError()));
  double sum_sq = 0.0, sum_abs = 0.0;
  for (int b = 0; b < blocks; ++b) {
    sum_sq += hp[2 * b];
    sum_abs += hp[2 * b + 1];
  }
  const int count = ca[0];
  uint32_t mxb = (uint32_t)ca[1];
  std::memcpy(&out->max_absolute, &mxb, 4);
  out->valid_pixel_count = count;
  out->valid_pixel_ratio = (float)count / (float)out->total_interior_pixel_count;
  if (count == 0) return XB_OK;
  out->mean_squared_score = (float)(sum_sq / (double)count);
  out->rms_score = std::sqrt(out->mean_squared_score);
  out->mean_absolute = (float)(sum_abs / (double)count);
  // order statistics at floor(p (n - 1)), p in float: the k-th smallest residual by its bits
  std::vector<unsigned int> h(65536);
  auto histogram = [&](int prefix) {
    if (!ck(cudaMemsetAsync(hist, 0, b_hist, s))) return false;
    digit_hist_kernel<<<blocks, kThreads, 0, s>>>(rel, n, prefix, hist);
    return ck(cudaMemcpyAsync(h.data(), hist, b_hist, cudaMemcpyDeviceToHost, s)) && ck(cudaStreamSynchronize(s));
  };
  auto pick = [&](uint64_t& k) {   // the digit holding the k-th element; k becomes its rank there
    for (int d = 0; d < 65536; ++d) {
      if (k < h[d]) return d;
      k -= h[d];
    }
    return 65535;
  };
  if (!histogram(-1)) return fail(XB_E_CUDA, "output stage: %s", cudaGetErrorString(cudaGetLastError()));
  const std::vector<unsigned int> high = h;
  float* dst[2] = {&out->median_absolute, &out->p95_absolute};
  const float ps[2] = {0.5f, 0.95f};
  for (int q = 0; q < 2; ++q) {
    uint64_t k = (uint64_t)(size_t)(ps[q] * (float)(count - 1));
    h = high;
    const int hi = pick(k);
    if (!histogram(hi)) return fail(XB_E_CUDA, "output stage: %s", cudaGetErrorString(cudaGetLastError()));
    const int lo = pick(k);
    const uint32_t bits = ((uint32_t)hi << 16) | (uint32_t)lo;
    std::memcpy(dst[q], &bits, 4);
  }
  return XB_OK;
}

}  // namespace xb
