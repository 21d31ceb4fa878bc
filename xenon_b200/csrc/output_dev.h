// output_dev.h — the output stage on the device (output_dev.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/xenon_b200.h"

namespace xb {
// 8-bit pixels (rgb8: host uint8[W*H*3], or nullptr) and noise statistics (out, or nullptr) of
// the device image d_img (float[W*H*3] in xb_resolve's layout), on stream s.
int device_output_stage(const float* d_img, int W, int H, int num_sms, cudaStream_t s, uint8_t* rgb8,
                        xb_noise_stats* out);
}  // namespace xb
