// oracle.h — C API of the CPU restatement of the reference path (test infrastructure).
//
// Used only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs, as the checker.
// It reads the same xb_scene_view the device receives and follows the reference CPU backend:
// traversal (src/geometry/{tlas,blas,prim_blas}.cpp, primitives.h), the BSDF
// (src/material/bsdf.h) and the tiled integrator (src/render/cpu_tiled.cpp).
#pragma once

#include <stdint.h>

#include "../include/xenon_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

void* xo_scene_new(const xb_scene_view* v);
void xo_scene_free(void* s);
/* mode 0 closest, 1 any; work[4] += blas nodes, triangle tests, tlas nodes, instance visits */
int xo_trace(void* s, int64_t n, const xb_ray* rays, xb_hit* hits, int mode, int64_t* work);
void xo_bsdf_eval(const xb_material* m, int64_t n, const float* wo, const float* wi, float* f, float* pdf);
void xo_bsdf_sample(const xb_material* m, int64_t n, const float* wo, uint64_t* states, float* wi,
                    float* f, float* pdf, int32_t* flags);
void xo_material_prepare(const xb_material* m, xb_material_derived* out);
uint64_t xo_seed_pcg(uint64_t seed);
/* Samples [spp_first, spp_first + spp_count) of every pixel, FP64 sums into sum_rgb
 * (double[h*w*3], top-down rows). rays[2] += closest-hit rays, shadow rays traced. */
int xo_render(void* s, const xb_camera* cam, int w, int h, int min_bounces, int max_bounces,
              int spp_first, int spp_count, double* sum_rgb, int64_t* rays, int threads);

#ifdef __cplusplus
}
#endif
