// image_out.cpp — the output stage after accumulation, on the host over the mean image that
// xb_resolve returns: the 8-bit PNG the reference writes when a render ends and its
// blur-residual noise statistics (src/main.cpp:24-52, src/math/image.h:35-118). The image is a
// couple of megapixels handled once per render, not the hot path.
//
// Rows: xb_resolve hands back the reference CPU backend's framebuffer order, whose first row is
// the bottom of the image (src/render/cpu_tiled.cpp:224-236), and the reference flips it on
// write (stbi_flip_vertically_on_write, src/main.cpp:26), so PNG row r is framebuffer row h-1-r.
//
// The statistics follow the reference's float operations in the same order (the host build has
// no FMA contraction), so they come out bit-identical to its strict build.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "capi_common.h"
#include "xenon_b200.h"

namespace {

// 8-bit value of one channel: clamp to [0, 1], gamma 1/2.2, times 255.99, truncated
// (src/main.cpp:28-29).
inline uint8_t to8(float v) {
  const float c = std::pow(std::min(std::max(v, 0.f), 1.f), 1.f / 2.2f);
  return (uint8_t)(255.99f * c);
}

// CRC-32 (ISO-HDLC polynomial, reflected; PNG chunk checksum) and Adler-32 (zlib stream
// checksum), computed from their definitions.
struct Crc32 {
  uint32_t table[256];
  Crc32() {
    for (uint32_t n = 0; n < 256; ++n) {
      uint32_t c = n;
      for (int k = 0; k < 8; ++k) c = (c & 1u) ? 0xEDB88320u ^ (c >> 1) : c >> 1;
      table[n] = c;
    }
  }
  uint32_t update(uint32_t crc, const uint8_t* p, size_t n) const {
    crc = ~crc;
    for (size_t i = 0; i < n; ++i) crc = table[(crc ^ p[i]) & 0xffu] ^ (crc >> 8);
    return ~crc;
  }
};

uint32_t adler32(const uint8_t* p, size_t n) {
  uint32_t a = 1, b = 0;
  for (size_t i = 0; i < n; ++i) {
    a = (a + p[i]) % 65521u;
    b = (b + a) % 65521u;
  }
  return (b << 16) | a;
}

void put32(std::vector<uint8_t>& v, uint32_t x) {
  v.push_back((uint8_t)(x >> 24));
  v.push_back((uint8_t)(x >> 16));
  v.push_back((uint8_t)(x >> 8));
  v.push_back((uint8_t)x);
}

void chunk(std::vector<uint8_t>& png, const Crc32& crc, const char* type, const std::vector<uint8_t>& data) {
  put32(png, (uint32_t)data.size());
  const size_t start = png.size();
  png.insert(png.end(), type, type + 4);
  png.insert(png.end(), data.begin(), data.end());
  put32(png, crc.update(0, png.data() + start, png.size() - start));
}

}  // namespace

extern "C" {

int xb_image_to_rgb8(const float* rgb, int32_t width, int32_t height, uint8_t* out) {
  if (!rgb || !out || width <= 0 || height <= 0) return xb::fail(XB_E_INVALID, "xb_image_to_rgb8: bad arguments");
  const int64_t row = (int64_t)width * 3;
  for (int64_t r = 0; r < height; ++r) {
    const float* src = rgb + (height - 1 - r) * row;
    uint8_t* dst = out + r * row;
    for (int64_t i = 0; i < row; ++i) dst[i] = to8(src[i]);
  }
  return XB_OK;
}

int xb_write_png(const char* path, const float* rgb, int32_t width, int32_t height) {
  if (!path || !rgb || width <= 0 || height <= 0 || (int64_t)width * 3 + 1 > 65535 * 16)
    return xb::fail(XB_E_INVALID, "xb_write_png: bad arguments");
  std::vector<uint8_t> pix((size_t)((int64_t)width * 3 * height));
  xb_image_to_rgb8(rgb, width, height, pix.data());
  return xb_write_png_rgb8(path, pix.data(), width, height);
}

int xb_write_png_rgb8(const char* path, const uint8_t* pix, int32_t width, int32_t height) {
  if (!path || !pix || width <= 0 || height <= 0 || (int64_t)width * 3 + 1 > 65535 * 16)
    return xb::fail(XB_E_INVALID, "xb_write_png_rgb8: bad arguments");
  const int64_t row = (int64_t)width * 3;
  // scanlines with filter type 0, in a zlib stream of stored (uncompressed) deflate blocks
  std::vector<uint8_t> raw;
  raw.reserve((size_t)((row + 1) * height));
  for (int64_t r = 0; r < height; ++r) {
    raw.push_back(0);
    raw.insert(raw.end(), pix + r * row, pix + (r + 1) * row);
  }
  std::vector<uint8_t> z = {0x78, 0x01};
  size_t pos = 0;
  do {
    const size_t n = std::min<size_t>(65535, raw.size() - pos);
    const bool last = pos + n == raw.size();
    z.push_back(last ? 1 : 0);
    z.push_back((uint8_t)n);
    z.push_back((uint8_t)(n >> 8));
    z.push_back((uint8_t)~n);
    z.push_back((uint8_t)(~n >> 8));
    z.insert(z.end(), raw.begin() + pos, raw.begin() + pos + n);
    pos += n;
  } while (pos < raw.size());
  put32(z, adler32(raw.data(), raw.size()));
  static const Crc32 crc;
  std::vector<uint8_t> png = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1a, '\n'};
  std::vector<uint8_t> ihdr;
  put32(ihdr, (uint32_t)width);
  put32(ihdr, (uint32_t)height);
  ihdr.insert(ihdr.end(), {8, 2, 0, 0, 0});   // 8-bit RGB, deflate, adaptive filters, no interlace
  chunk(png, crc, "IHDR", ihdr);
  chunk(png, crc, "IDAT", z);
  chunk(png, crc, "IEND", {});
  FILE* f = std::fopen(path, "wb");
  if (!f) return xb::fail(XB_E_IO, "xb_write_png: cannot open %s", path);
  const size_t written = std::fwrite(png.data(), 1, png.size(), f);
  const int closed = std::fclose(f);
  if (written != png.size() || closed != 0) return xb::fail(XB_E_IO, "xb_write_png: cannot write %s", path);
  return XB_OK;
}

int xb_image_noise_stats(const float* rgb, int32_t width, int32_t height, xb_noise_stats* out) {
  if (!rgb || !out || width <= 0 || height <= 0) return xb::fail(XB_E_INVALID, "xb_image_noise_stats: bad arguments");
  std::memset(out, 0, sizeof(*out));
  if (width <= 2 || height <= 2) return XB_OK;   // no interior pixel
  const int64_t n = (int64_t)width * height;
  out->total_interior_pixel_count = (width - 2) * (height - 2);
  // luminance (Rec. 709 weights) and its mean, summed in FP64 in pixel order
  std::vector<float> lum((size_t)n), blur((size_t)n);
  double sum = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    lum[i] = 0.2126f * rgb[3 * i] + 0.7152f * rgb[3 * i + 1] + 0.0722f * rgb[3 * i + 2];
    sum += lum[i];
  }
  out->avg_luminance = (float)(sum / (double)n);
  // 3x3 binomial blur (1 2 1 / 2 4 2 / 1 2 1) / 16, edges clamped, terms added row by row
  static const float kw[3][3] = {{1.f, 2.f, 1.f}, {2.f, 4.f, 2.f}, {1.f, 2.f, 1.f}};
  for (int y = 0; y < height; ++y)
    for (int x = 0; x < width; ++x) {
      float s = 0.f;
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          const int xx = std::min(std::max(x + dx, 0), width - 1);
          const int yy = std::min(std::max(y + dy, 0), height - 1);
          s += kw[dy + 1][dx + 1] * lum[(size_t)yy * width + xx];
        }
      blur[(size_t)y * width + x] = s / 16.f;
    }
  out->edge_threshold = std::max(1e-6f, out->avg_luminance * 0.1f);
  out->epsilon = std::max(1e-8f, out->avg_luminance * out->avg_luminance * 1e-4f);
  // interior pixels away from strong edges: luminance minus its blur, relative to the blur
  std::vector<float> rel;
  rel.reserve((size_t)out->total_interior_pixel_count);
  double sum_sq = 0.0, sum_abs = 0.0;
  for (int y = 1; y < height - 1; ++y)
    for (int x = 1; x < width - 1; ++x) {
      const size_t i = (size_t)y * width + x;
      const float gx = 0.5f * (lum[i + 1] - lum[i - 1]);
      const float gy = 0.5f * (lum[i + width] - lum[i - width]);
      if (std::sqrt(gx * gx + gy * gy) >= out->edge_threshold) continue;
      const float d = lum[i] - blur[i];
      const float den = blur[i] * blur[i] + out->epsilon;
      const float a = std::fabs(d) / std::sqrt(den);
      sum_sq += (d * d) / den;
      sum_abs += a;
      rel.push_back(a);
      out->max_absolute = std::max(out->max_absolute, a);
    }
  const int count = (int)rel.size();
  out->valid_pixel_count = count;
  out->valid_pixel_ratio = (float)count / (float)out->total_interior_pixel_count;
  if (count == 0) return XB_OK;
  out->mean_squared_score = (float)(sum_sq / (double)count);
  out->rms_score = std::sqrt(out->mean_squared_score);
  out->mean_absolute = (float)(sum_abs / (double)count);
  // order statistics at index floor(p (n - 1)), p computed in float
  auto quantile = [&](float p) {
    const size_t k = (size_t)(p * (float)(count - 1));
    std::nth_element(rel.begin(), rel.begin() + (std::ptrdiff_t)k, rel.end());
    return rel[k];
  };
  out->median_absolute = quantile(0.5f);
  out->p95_absolute = quantile(0.95f);
  return XB_OK;
}

}  // extern "C"
