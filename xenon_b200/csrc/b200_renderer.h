// b200_renderer.h — C++17 face of the C ABI, with xn::CudaRenderer's method set.
//
// A driver written against the reference's CudaRenderer (src/cuda/cuda_renderer.cuh:14-55) or
// the CPU twin WavefrontRenderer (src/render/wavefront.h:19-36) switches to this class under
// `--backend b200` with the same call sequence:
//
//   xb::B200Renderer r(w, h, max_bounces, min_bounces);   // CudaRenderer(w, h, max, min)
//   r.upload_scene(view);                                 // CudaRenderer::upload_scene
//   while (r.spp() < samples) r.render_frame(cam, buf);   // one sample, mean image into buf
//
// Errors raise xb::Error (the reference aborts; the C ABI returns status codes).
#pragma once

#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/xenon_b200.h"

namespace xb {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

inline void check(int rc, const xb_renderer* r = nullptr) {
  if (rc < 0) {
    char buf[512];
    xb_last_error(r, buf, sizeof(buf));
    throw Error(rc, buf);
  }
}

class B200Renderer {
 public:
  B200Renderer(int width, int height, int max_bounces, int min_bounces, int device = 0, int flags = 0) {
    xb_config cfg{};
    cfg.width = width;
    cfg.height = height;
    cfg.max_bounces = max_bounces;
    cfg.min_bounces = min_bounces;
    cfg.device = device;
    cfg.flags = flags;
    check(xb_create(&cfg, &r_));
    w_ = width;
    h_ = height;
  }
  ~B200Renderer() { xb_destroy(r_); }
  B200Renderer(const B200Renderer&) = delete;
  B200Renderer& operator=(const B200Renderer&) = delete;

  void upload_scene(const xb_scene_view& v) { check(xb_upload_scene(r_, &v), r_); }
  void upload_scene(const xb_scene* s) {
    xb_scene_view v;
    check(xb_scene_get_view(s, &v));
    upload_scene(v);
  }
  // Adds one sample per pixel and writes the mean image (float[W*H*3], top-down rows) into
  // `framebuffer`, as CudaRenderer::render_frame does into the swapchain's write buffer.
  void render_frame(const xb_camera& cam, float* framebuffer, int spp_to_add = 1) {
    check(xb_render(r_, &cam, spp_to_add), r_);
    if (framebuffer) check(xb_resolve(r_, framebuffer), r_);
  }
  void set_bounces(int min_b, int max_b) { check(xb_set_bounces(r_, min_b, max_b), r_); }
  void reset_accumulation() { check(xb_reset(r_), r_); }
  int spp() const { return xb_get_spp(r_); }
  int width() const { return w_; }
  int height() const { return h_; }
  xb_renderer* handle() { return r_; }

  // The reference's save_image (src/main.cpp:24-52) on a framebuffer as render_frame fills it:
  // the PNG file, and the noise statistics it prints (host code, no device needed).
  static xb_noise_stats save_image(const std::string& path, const float* framebuffer, int width, int height) {
    check(xb_write_png(path.c_str(), framebuffer, width, height));
    xb_noise_stats s{};
    check(xb_image_noise_stats(framebuffer, width, height, &s));
    return s;
  }

 private:
  xb_renderer* r_ = nullptr;
  int w_ = 0, h_ = 0;
};

}  // namespace xb
