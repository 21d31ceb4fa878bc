/*
 * xenon_b200.h — C ABI of the B200-native wavefront path tracer.
 *
 * This is the drop-in boundary for Xenon's GPU backend. Each entry point names the
 * reference interface it replaces (paths are relative to the Xenon source tree):
 *
 *   xb_create / xb_destroy     xn::CudaRenderer::CudaRenderer / ~CudaRenderer
 *                              (src/cuda/cuda_renderer.cuh:16-17, cuda_renderer.cu:446-456)
 *   xb_upload_scene            xn::CudaRenderer::upload_scene (cuda_renderer.cuh:23) and
 *                              xn::GpuSceneHost::upload (src/cuda/gpu_scene.cu:38)
 *   xb_render                  xn::CudaRenderer::render_frame (cuda_renderer.cuh:26), which adds
 *                              one sample per pixel; here `spp_to_add` samples per call
 *   xb_resolve                 the framebuffer hand-off TripleSwapchain::get_write_buffer()
 *                              + swap_writer() (src/render/swapchain.h:30-46), with the CPU
 *                              backend's top-down row order (src/render/cpu_tiled.cpp:224-236)
 *   xb_get_spp                 xn::CudaRenderer::spp (cuda_renderer.cuh:28)
 *   xb_reset                   xn::WavefrontRenderer::reset_accumulation (src/render/wavefront.h:22)
 *   xb_set_bounces             xn::WavefrontRenderer::set_bounces (src/render/wavefront.h:30)
 *   xb_trace_rays              xn::Scene::intersect / intersects (src/scene/scene.h:124-129)
 *   xb_bsdf_eval               xn::bsdf_eval_for_nee / bsdf_pdf_for_nee (src/material/bsdf.h:601-657)
 *   xb_bsdf_sample             xn::bsdf_sample (src/material/bsdf.h:666-708)
 *   xb_scene_*                 xn::Scene building (src/scene/scene.h:52-121), the .xenon loader
 *                              xn::load_scene (src/scene/scene_file.h:22) and the .mat loader
 *                              xn::load_material (src/material/material.h:81)
 *
 * Conventions: every function returns XB_OK (0) or a negative XB_E_* status and never aborts.
 * xb_last_error() returns the message of the last failure on the calling thread. One renderer
 * is used by one host thread at a time. Host pointers unless a name says `device`.
 */
#ifndef XENON_B200_H
#define XENON_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ── status codes ─────────────────────────────────────────────────────────── */
#define XB_OK             0
#define XB_E_INVALID     -1   /* bad argument */
#define XB_E_CUDA        -2   /* a CUDA runtime call failed */
#define XB_E_OOM         -3   /* device or host allocation failed */
#define XB_E_STATE       -4   /* call out of order (e.g. render before upload) */
#define XB_E_IO          -5   /* file missing or unparsable */
#define XB_E_OVERFLOW    -6   /* a device queue or traversal stack overflowed (work dropped) */
#define XB_E_TIMEOUT     -7   /* a bounded device wait gave up */
#define XB_E_UNSUPPORTED -8

/* ── scene data formats (POD, identical bytes to the reference structs) ─────── */

/* Principled material authoring parameters (src/material/material.h:19-36). */
typedef struct xb_material {
  float base_color[3];
  float roughness;
  float metallic;
  float ior;
  float transmission;
  float subsurface;
  float subsurface_color[3];
  float anisotropy;
  float emission[3];
  float subsurface_mfp[3];
  float clearcoat;
  float clearcoat_roughness;
  float emission_temperature;
} xb_material;

/* Values material_prepare derives (src/material/material.h:55-75). */
#define XB_MAT_CONDUCTOR    1
#define XB_MAT_TRANSMISSIVE 2
#define XB_MAT_SUBSURFACE   4
#define XB_MAT_DELTA        8
#define XB_MAT_EMISSIVE     16
typedef struct xb_material_derived {
  float alpha, alpha_x, alpha_y;
  float f0[3];
  int32_t flags;
} xb_material_derived;

/* BVH node: BLASNode / TLASNode / PrimBLASNode (src/geometry/blas.h:21-27), 32 bytes.
 * count == 0: internal, children at `child` and `child + 1`; count > 0: leaf. */
typedef struct xb_bvh_node {
  float mn[3];
  float mx[3];
  uint32_t child;
  uint32_t count;
} xb_bvh_node;

/* Analytic primitive (src/geometry/primitives.h:54-318). Parameter layout per type:
 *   SPHERE center[3] radius          PLANE normal[3] offset
 *   BOX    center[3] half[3]         DISK  center[3] normal[3] radius
 *   QUAD   origin[3] u[3] v[3] */
#define XB_PRIM_SPHERE 0
#define XB_PRIM_PLANE  1
#define XB_PRIM_BOX    2
#define XB_PRIM_DISK   3
#define XB_PRIM_QUAD   4
typedef struct xb_prim {
  int32_t type;
  int32_t mat_id;
  float p[10];
} xb_prim;

/* Triangle mesh (src/geometry/mesh.h:21-31) with its BLAS (src/geometry/blas.h:61-62). */
typedef struct xb_mesh_view {
  int32_t num_vertices;
  int32_t num_triangles;
  const float *vx, *vy, *vz;          /* positions, SoA */
  const float *nx, *ny, *nz;          /* shading normals, SoA; NULL → geometric normal */
  const int32_t *indices;             /* 3 per triangle */
  const int32_t *mat_ids;             /* 1 per triangle */
  const xb_bvh_node *blas_nodes;
  int32_t num_blas_nodes;
  const uint32_t *blas_prims;         /* num_triangles entries */
} xb_mesh_view;

/* TLAS instance (src/geometry/tlas.h:76-87): column-major 3x4 affine matrices
 * (c0, c1, c2 basis columns, c3 translation; src/geometry/transform.h:32-63). */
#define XB_GEOM_PRIMS (-1)
typedef struct xb_instance_view {
  int32_t geom;                       /* mesh index, or XB_GEOM_PRIMS for the prim group */
  int32_t instance_id;
  float local_to_world[12];
  float world_to_local[12];
} xb_instance_view;

/* Area light: one emitting triangle (src/scene/scene.h:19-24). */
typedef struct xb_light {
  uint32_t mesh_id;
  uint32_t tri_idx;
  float emission[3];
  float area;
} xb_light;

/* Directional light (src/scene/scene.h:43-49). direction points toward the light. */
typedef struct xb_sun {
  float direction[3];
  float color[3];
  float intensity;
} xb_sun;

/* Gradient sky (src/scene/environment.h:14-39). */
typedef struct xb_sky {
  float zenith[3];
  float horizon[3];
  float ground[3];
  float sharpness;
  float intensity;
} xb_sky;

/* Flattened scene: everything the device needs. Pointers are host memory, owned by the
 * caller; xb_upload_scene copies them. */
typedef struct xb_scene_view {
  int32_t num_meshes;
  const xb_mesh_view *meshes;
  int32_t num_prims;
  const xb_prim *prims;
  const xb_bvh_node *prim_nodes;
  int32_t num_prim_nodes;
  const uint32_t *prim_indices;
  int32_t num_instances;
  const xb_instance_view *instances;
  const xb_bvh_node *tlas_nodes;
  int32_t num_tlas_nodes;
  const uint32_t *tlas_inst_indices;
  int32_t num_materials;
  const xb_material *materials;
  int32_t num_lights;
  const xb_light *lights;
  int32_t num_suns;
  const xb_sun *suns;
  xb_sky sky;
} xb_scene_view;

/* Ray (src/math/ray.h:119-126) as two 16-byte halves. */
typedef struct xb_ray {
  float org[3];
  float tmin;
  float dir[3];
  float tmax;
} xb_ray;

/* Hit record (src/math/ray.h:131-143). A miss has t = +inf and ids = -1. */
typedef struct xb_hit {
  float t, u, v;
  int32_t prim_id;
  int32_t instance_id;
  int32_t mat_id;
  int32_t front_face;
  float pos[3];
  float normal[3];
  float geo_normal[3];
} xb_hit;

/* Pinhole camera as the device sees it (Camera::look_at, src/camera/camera.h:15-31). */
typedef struct xb_camera {
  float eye[3];
  float lower_left[3];
  float horizontal[3];
  float vertical[3];
} xb_camera;

/* ── host scene: loaders and the TLAS/BLAS build ──────────────────────────── */

typedef struct xb_scene xb_scene;

typedef struct xb_scene_config {     /* xn::SceneConfig (src/scene/scene_file.h:11-19) */
  int32_t width, height, samples;
  int32_t min_bounces, max_bounces;
} xb_scene_config;

typedef struct xb_camera_desc {      /* the .xenon `camera` line */
  float eye[3];
  float target[3];
  float fov_y_deg;
} xb_camera_desc;

void xb_material_default(xb_material *m);
int  xb_material_prepare(const xb_material *m, xb_material_derived *out);
int  xb_material_load(const char *path, xb_material *out, char *name, size_t name_len);
int  xb_camera_look_at(const float eye[3], const float target[3], const float up[3],
                       float fov_y_deg, float aspect, xb_camera *out);

int  xb_scene_create(xb_scene **out);
void xb_scene_destroy(xb_scene *s);
/* Each add returns the new object's id (>= 0) or a negative status. */
int  xb_scene_add_material(xb_scene *s, const char *name, const xb_material *m);
int  xb_scene_add_mesh(xb_scene *s, int32_t num_vertices, const float *positions,
                       const float *normals, int32_t num_triangles, const int32_t *indices,
                       const int32_t *mat_ids, int32_t default_mat_id);
int  xb_scene_transform_mesh(xb_scene *s, int32_t mesh, const float pos[3], float scale,
                             const float rot_deg[3]);
int  xb_scene_add_prim(xb_scene *s, const xb_prim *p);
int  xb_scene_add_light(xb_scene *s, uint32_t mesh_id, uint32_t tri_idx,
                        const float emission[3], float area);
int  xb_scene_add_sun(xb_scene *s, const float direction[3], const float color[3],
                      float intensity);
int  xb_scene_set_sky(xb_scene *s, const xb_sky *sky);
/* Explicit TLAS instances (AffineTransform::from_trs, src/geometry/transform.h:105). With none,
 * xb_scene_build makes one identity instance per mesh plus one for the prim group, as
 * Scene::build_acceleration does (src/scene/scene.h:79-121). */
int  xb_scene_add_instance(xb_scene *s, int32_t geom, const float translation[3], float scale,
                           const float rot_deg[3], int32_t instance_id);
int  xb_scene_build(xb_scene *s);
/* Threads of the BVH builds (0, the default: the machine's hardware threads; 1: one). Meshes are
 * built side by side and large subtrees split across threads; the node arrays are the same for
 * any count (the reference's, which builds on one thread). No reference counterpart. */
int  xb_scene_set_build_threads(xb_scene *s, int32_t threads);
/* The form of the binned-SAH builds; all give the same node and order arrays.
 *   XB_BUILD_RECURSIVE (default): depth first, one node at a time, as the reference builds.
 *   XB_BUILD_LEVELS: level-synchronous on the host. Every node of a depth is split in one pass,
 *     each step an ordered reduction, a prefix sum or a per-node scan.
 *   XB_BUILD_DEVICE: the level-synchronous form run by the current CUDA device; one pass of
 *     kernels per depth, the host reading each depth's outcome. xb_scene_build returns
 *     XB_E_CUDA when there is no device.
 * No reference counterpart. */
#define XB_BUILD_RECURSIVE 0
#define XB_BUILD_LEVELS    1
#define XB_BUILD_DEVICE    2
int  xb_scene_set_build_mode(xb_scene *s, int32_t mode);
/* Moves the vertices of mesh `mesh` of a built scene and refits its BLAS: the tree keeps its
 * topology and every node box is recomputed bottom-up from the new triangles (a leaf from its
 * triangles in slot order, an interior node from its two children), then the TLAS is rebuilt
 * over the instances' new world boxes as xb_scene_build builds it. positions: float[3 * nv]
 * (nv = the mesh's vertex count); normals: the same, or NULL to keep the mesh's. With unchanged
 * vertices the node boxes equal the build's. Upload the scene again to render it. No reference
 * counterpart: the reference rebuilds (BLAS::build, src/geometry/blas.cpp:183-205). */
int  xb_scene_refit_mesh(xb_scene *s, int32_t mesh, const float *positions, const float *normals);
int  xb_scene_get_view(const xb_scene *s, xb_scene_view *out);
int  xb_scene_load(const char *path, xb_scene **out, xb_scene_config *cfg, xb_camera_desc *cam);

/* ── renderer ─────────────────────────────────────────────────────────────── */

typedef struct xb_renderer xb_renderer;

#define XB_FLAG_FP64_ACCUM      1   /* FP64 per-pixel sum + Welford M2 (oracle renders) */
#define XB_FLAG_THREAD_PER_RAY  2   /* one-ray-per-thread traversal instead of persistent warps */
#define XB_FLAG_SUN_NEE         4   /* directional lights as delta lights in next-event estimation:
                                       contribution f cos E / P(pick), MIS weight 1. Off (parity):
                                       the reference's 1e8 divisor (src/render/cpu_tiled.cpp:166-183),
                                       with which a sun adds about 1e-8 of its light */
#define XB_FLAG_SKY_IS          8   /* sky importance sampling: at non-delta, non-transmissive
                                       vertices seen from the front with a broad lobe (not a
                                       conductor of GGX alpha < 0.25), the next direction comes from
                                       the one-sample MIS mixture of the sky's luminance
                                       distribution (probability 1/2) and the BSDF sampler; the path
                                       carries the importance ratio, so the image converges to the
                                       default one (the sky is weighted by 1 in
                                       src/render/cpu_tiled.cpp:40-54). Ignored while guiding is on.
                                       Changes the random-number draws (not in parity mode). */
#define XB_FLAG_WATERTIGHT      16  /* watertight ray-triangle test (Woop, Benthin and Wald 2013:
                                       shear to ray space, edge functions, FP64 re-evaluation of a
                                       zero edge) in every query of the renderer, instead of the
                                       reference's Moller-Trumbore (src/geometry/primitives.h:25-49),
                                       which can let a ray through the shared edge or vertex of two
                                       triangles. Off (parity): Moller-Trumbore, bit-exact hits */

typedef struct xb_config {
  int32_t width, height;
  int32_t max_bounces, min_bounces;  /* CudaRenderer(width, height, max_bounces, min_bounces) */
  int32_t device;                    /* CUDA device ordinal */
  int32_t flags;                     /* XB_FLAG_* */
  int32_t wave_paths;                /* paths in flight per wave; 0 = automatic */
  int32_t block_size;                /* threads per block of the trace kernels; 0 = automatic */
} xb_config;

int  xb_create(const xb_config *cfg, xb_renderer **out);
void xb_destroy(xb_renderer *r);
int  xb_last_error(const xb_renderer *r, char *buf, size_t len);
int  xb_upload_scene(xb_renderer *r, const xb_scene_view *view);
/* Moves the vertices of uploaded mesh `mesh` and refits its BLAS on the device: the triangles
 * take the new positions, and every node box is recomputed bottom-up by one kernel in which the
 * second child to reach a node folds both children's boxes (no thread waits for another). The
 * passes are those xb_scene_refit_mesh runs on the host, so both give the same node arrays. The
 * TLAS is then rebuilt on the host over the instances' new world boxes and copied up. positions: host
 * float[3 * nv] (nv = the mesh's vertex count in the uploaded view); normals: the same, or NULL
 * to keep the uploaded ones. Meshes that carry area lights are refused (XB_E_UNSUPPORTED: their
 * emitter geometry is built on the host at upload; refit the host scene and upload again).
 * Synchronises the render stream; captured bounce graphs are rebuilt on the next render. The
 * arrays are rewritten in place, so ray queries issued on caller streams (xb_trace_rays_device,
 * xb_trace_rays_noalloc) must have finished before this call. If the uploaded BLAS turns out to
 * be malformed (XB_E_INVALID), some of it has already been rewritten: the renderer then holds no
 * scene (later calls fail with XB_E_STATE) until the scene is uploaded again. The accumulated
 * image is kept: call xb_reset for frames of a moving scene. No reference counterpart: the
 * reference rebuilds its BLAS on the host (src/geometry/blas.cpp:183-205). */
int  xb_refit_mesh(xb_renderer *r, int32_t mesh, const float *positions, const float *normals);
int  xb_set_bounces(xb_renderer *r, int32_t min_bounces, int32_t max_bounces);
/* Adds spp_to_add samples per pixel; sample k of pixel p is seeded exactly as the CPU backend
 * seeds it (seed_pcg(p + k * 0xdeadbeef), src/render/cpu_tiled.cpp:22-23). With guiding on, the
 * samples that train the network are left out of the image unless keep_training_samples is set;
 * xb_get_spp then counts the image's samples. */
int  xb_render(xb_renderer *r, const xb_camera *cam, int32_t spp_to_add);
/* Many views in one call (config 5: dozens of cameras, 256^2 to 1024^2 pixels, 16 to 1024
 * samples, bounce limits 6 to 16): the views share the renderer's scene and are packed together into
 * the same waves, so small views still fill the GPU. Each view renders samples 1..spp, seeded as
 * a render of that view alone (seed_pcg(p + k * 0xdeadbeef)), so its image equals a
 * single-view render of the same size; out_rgb receives the view's mean image (host memory,
 * float[width*height*3], top-down rows). The renderer's own accumulation is untouched. With
 * guiding on, views use the current network without training it. No reference counterpart:
 * the reference renders one view per CudaRenderer. */
typedef struct xb_view {
  xb_camera camera;
  int32_t width, height;
  int32_t spp;
  int32_t max_bounces;     /* this view's bounce limit (0: the renderer's) */
  float *out_rgb;
} xb_view;
int  xb_render_views(xb_renderer *r, const xb_view *views, int32_t count);
/* Mean radiance, float[W*H*3], top-down rows. */
int  xb_resolve(xb_renderer *r, float *out_rgb);
/* xb_resolve without waiting: the mean image of the samples rendered so far is written into
 * out_rgb (host memory, page-locked for the copy to overlap) while later calls proceed; the
 * image is complete when xb_sync returns (or when the next-but-one xb_resolve_async has been
 * enqueued and that call's images were synchronised). Lets a caller hand every sample's image
 * to the host, as CudaRenderer::render_frame does, without stalling the GPU on the copy. */
int  xb_resolve_async(xb_renderer *r, float *out_rgb);
/* Waits for all work of the renderer, including asynchronous resolves. */
int  xb_sync(xb_renderer *r);
/* FP64 per-pixel sums and Welford M2 (needs XB_FLAG_FP64_ACCUM); each double[W*H*3]. */
int  xb_resolve_fp64(xb_renderer *r, double *sum_rgb, double *m2_rgb);
/* The same into device memory of the renderer's GPU (top-down rows; either pointer may be NULL),
 * complete when the call returns: what a multi-GPU caller sums across GPUs (NCCL) without a
 * round trip through the host. No reference counterpart (the reference renders on one device). */
int  xb_resolve_fp64_device(xb_renderer *r, double *sum_rgb, double *m2_rgb);

/* Output stage, on the host over an image as xb_resolve returns it (float[W*H*3], first row the
 * bottom of the image as in the reference's framebuffer). The reference does this inside its
 * main() when a render ends (save_image, src/main.cpp:24-52).
 *   xb_image_to_rgb8: the PNG's 8-bit pixels, top row first: each channel clamped to [0, 1],
 *     raised to 1/2.2, times 255.99, truncated (src/main.cpp:26-30) — uint8[W*H*3].
 *   xb_write_png: those pixels as an 8-bit RGB PNG file (uncompressed deflate blocks).
 *   xb_image_noise_stats: ImageNoiseEstimator::computeResidualNoiseStats
 *     (src/math/image.h:35-118): luminance minus its 3x3 blur, relative to the blur, over the
 *     interior pixels whose luminance gradient is below a tenth of the mean luminance. */
typedef struct xb_noise_stats {
  float mean_squared_score;   /* mean of residual^2 / (blur^2 + epsilon) */
  float rms_score;
  float mean_absolute;        /* mean, median, 95th percentile and maximum of |residual| / */
  float median_absolute;      /* sqrt(blur^2 + epsilon) */
  float p95_absolute;
  float max_absolute;
  float avg_luminance;
  float edge_threshold;       /* max(1e-6, avg_luminance / 10) */
  float epsilon;              /* max(1e-8, 1e-4 avg_luminance^2) */
  int32_t valid_pixel_count;
  int32_t total_interior_pixel_count;
  float valid_pixel_ratio;
} xb_noise_stats;
int  xb_image_to_rgb8(const float *rgb, int32_t width, int32_t height, uint8_t *out_rgb8);
int  xb_write_png(const char *path, const float *rgb, int32_t width, int32_t height);
int  xb_image_noise_stats(const float *rgb, int32_t width, int32_t height, xb_noise_stats *out);
/* The same output stage on the device, over the renderer's current mean image (what xb_resolve
 * would return) right after accumulation, without the image leaving the GPU: rgb8 (host
 * uint8[W*H*3], or NULL) receives xb_image_to_rgb8's pixels, stats (or NULL) the noise
 * statistics. Per-pixel values follow the same float operations as the host forms; the FP64
 * sums are reduced per block, so the mean scores can differ from the host's in the last bit of
 * the float, and the 8-bit values where CUDA's powf and the host's round the gamma differently. */
int  xb_output_stage(xb_renderer *r, uint8_t *rgb8, xb_noise_stats *stats);
/* 8-bit pixels as xb_image_to_rgb8 (or xb_output_stage) returns them, written as xb_write_png writes. */
int  xb_write_png_rgb8(const char *path, const uint8_t *rgb8, int32_t width, int32_t height);
int  xb_get_spp(const xb_renderer *r);
int  xb_reset(xb_renderer *r);
/* Renders samples [spp_first, spp_first + spp_count) of the sequence (1-based), e.g. one shard
 * of a multi-GPU job; xb_render(r, cam, n) equals xb_render_range(r, cam, spp + 1, n). */
int  xb_render_range(xb_renderer *r, const xb_camera *cam, int32_t spp_first, int32_t spp_count);

typedef struct xb_render_stats {
  int64_t rays_closest;   /* closest-hit rays traced (camera + bounce) */
  int64_t rays_shadow;    /* any-hit shadow rays traced */
  int64_t paths;          /* paths started */
  int64_t overflow;       /* items dropped by a full queue or traversal stack (must be 0) */
  float   last_ms;        /* device time of the last xb_render / xb_render_range call */
  int64_t nonfinite;      /* path samples with a NaN or infinite radiance (left out of the image) */
} xb_render_stats;
int  xb_get_render_stats(const xb_renderer *r, xb_render_stats *out);
int  xb_reset_render_stats(xb_renderer *r);

/* Launch tuning (picked per GPU and scene by xenon_b200/autotune.py). Zero fields keep the
 * current value; negative fields restore the default. */
typedef struct xb_tuning {
  int32_t extend_persistent_from_depth; /* closest-hit rays of bounces >= this use persistent
                                           warps, earlier bounces one ray per thread (64: never) */
  int32_t shadow_persistent;            /* 1: persistent warps for shadow rays, 2: one per thread */
  int32_t refill;                       /* persistent warps refill when this many lanes idle */
  int32_t extend_blocks_per_sm;         /* blocks of 128 threads per SM in the grid of the trace */
  int32_t shadow_blocks_per_sm;         /* and shade kernels (1-64); for the persistent ones */
  int32_t shade_blocks_per_sm;          /* bounded by the blocks that fit on an SM at once */
  int32_t wave_paths;                   /* paths in flight per wave (reallocates queues) */
  int32_t shadow_order;                 /* shadow rays: 1 nearer child first, 2 farther first
                                           (the occlusion answer does not depend on it) */
  int32_t overlap;                      /* 1: a bounce's shadow rays run on a second stream,
                                           concurrently with the next bounce's closest hits;
                                           2: one stream */
  int32_t waves;                        /* waves in flight, 1-4 (default 2): a call's consecutive
                                           waves run on that many stream lanes at once (each
                                           lane holds its own queues). Same image either way. */
  int32_t lane_stagger;                 /* a lane's first wave of a call starts once the previous
                                           lane's has shaded this many bounces (1-16) */
  int32_t graph;                        /* 1 (default): the bounce loop of a full, non-training
                                           wave of xb_render replays a CUDA graph captured from
                                           its launches on first use; 2: direct launches. Not
                                           used while profiling. Same image either way. */
  int32_t guided_form;                  /* guided bounces: 1 (default) a plain-form bounce kernel
                                           plus a network pass over the guided vertices; 2 one
                                           fused kernel. Same image either way. */
  int32_t shade_occupancy;              /* shading kernels compiled to fit 4, 8 (default), 12 or
                                           16 blocks of 128 threads per SM: fewer registers per
                                           thread, the rest spilled to L1 (other values: 8; the
                                           guided bounces take 4 or 8, 8 for 12 and 16) */
  int32_t shared_stack;                 /* traversal kernels: 16 = the first 16 entries of each
                                           thread's BLAS stack in shared memory (8 KB per block of
                                           128 threads), the rest in local memory; 1 (default, and
                                           any other value): all in local memory. Same hits. */
  int32_t pixel_order;                  /* camera rays in the queue: 1 scanline order, 2 (default)
                                           each warp's 32 rays from one 8x4 pixel tile (config 3:
                                           5 % faster). Same image either way. */
} xb_tuning;
int  xb_set_tuning(xb_renderer *r, const xb_tuning *t);
int  xb_get_tuning(const xb_renderer *r, xb_tuning *out);

/* Profiling (tracing subsystem): per-stage device time from CUDA events recorded around every
 * stage launch on the renderer's stream, and per-ray traversal work counters. */
#define XB_PROFILE_STAGE_TIMES     1
#define XB_PROFILE_COUNT_TRAVERSAL 2
typedef struct xb_profile {
  double raygen_ms, extend_ms, shade_ms, shadow_ms, accumulate_ms;
  int64_t raygen_launches, extend_launches, shade_launches, shadow_launches, accumulate_launches;
  /* traversal work (XB_PROFILE_COUNT_TRAVERSAL): closest-hit (ext_*) and shadow (sh_*) rays */
  int64_t ext_blas_nodes, ext_tris, ext_tlas_nodes, ext_instances;
  int64_t sh_blas_nodes, sh_tris, sh_tlas_nodes, sh_instances;
  /* guiding: record finalisation and network training after training waves */
  double train_ms;
  int64_t train_launches;
  /* the time during which at least one launch of the stage was running: the union of its launch
   * intervals over all wave lanes and streams (the *_ms sums above count overlapping launches
   * of several lanes once each, so they can exceed the call's duration; these cannot) */
  double extend_busy_ms, shade_busy_ms, shadow_busy_ms;
} xb_profile;
int  xb_set_profiling(xb_renderer *r, int32_t flags);
int  xb_get_profile(const xb_renderer *r, xb_profile *out);
int  xb_reset_profile(xb_renderer *r);

/* Ray queries against the uploaded scene. mode 0 = closest hit (Scene::intersect),
 * 1 = any hit (Scene::intersects: hits[i].t = 0 when occluded, +inf when not). */
#define XB_TRACE_CLOSEST 0
#define XB_TRACE_ANY     1
int  xb_trace_rays(xb_renderer *r, const xb_ray *rays, int64_t n, xb_hit *hits, int32_t mode);
/* Same on device memory and a caller stream (cudaStream_t, NULL = default). Closest-hit queries
 * run on persistent warps when xb_tuning.extend_persistent_from_depth <= 1, any-hit queries when
 * shadow_persistent = 1 (the renderer's own choice for its bounce and shadow rays; both are the
 * defaults), else one ray per thread (also with XB_FLAG_THREAD_PER_RAY); the records are the same
 * either way. Calls on different streams may overlap: they share no device state. */
int  xb_trace_rays_device(xb_renderer *r, const xb_ray *rays, int64_t n, xb_hit *hits,
                          int32_t mode, void *stream);

/* Same as xb_trace_rays_device, but the call allocates nothing (no cudaMalloc, cudaFree or
 * allocating library routine): for callers that cannot allocate device memory while they trace,
 * e.g. a plugin whose host application owns all device memory (its own allocator, or a fixed
 * budget set at start-up). Its scratch (the 64-bit ray cursor and the ray count) is a fixed
 * 256-byte device array inside the library, shared by every call and cleared at the start of
 * each: calls that overlap on the GPU race on it, so issue them on one stream or otherwise one at
 * a time. The first call on a device looks up that array's address (cudaGetSymbolAddress, once
 * per device, with the device current); make that first call before any stream capture. Batches
 * above XB_NOALLOC_MAX_RAYS rays are rejected with XB_E_INVALID. Threads whose traversal stack
 * overflowed (their rays may have lost a hit) are added to the renderer's overflow count
 * (xb_get_render_stats), as for xb_trace_rays_device. It has no counterpart in the reference. */
#define XB_NOALLOC_MAX_RAYS ((int64_t)1 << 40)
int  xb_trace_rays_noalloc(xb_renderer *r, const xb_ray *rays, int64_t n, xb_hit *hits,
                           int32_t mode, void *stream);

/* BSDF on the device, host buffers: wo, wi float[n*3] in the shading frame (z = normal). */
int  xb_bsdf_eval(const xb_material *m, int64_t n, const float *wo, const float *wi,
                  float *f_rgb, float *pdf);
/* rng_state: uint64[n] PCG32 states (increment 1), advanced in place. flags bit0 = sample valid,
 * bit1 = delta lobe. */
int  xb_bsdf_sample(const xb_material *m, int64_t n, const float *wo, uint64_t *rng_state,
                    float *wi, float *f_rgb, float *pdf, int32_t *flags);
/* The true density with which xb_bsdf_sample returns wi (per steradian, over all lobes), for
 * non-delta, non-transmissive materials seen from the front (wo.z > 0; 0 otherwise). For the GGX
 * lobes it is the returned pdf times cos^4 of the half vector's angle: the reference's GGX
 * distribution (bsdf.h:67-76) carries an extra 1/cos^4 while its sampler draws the standard
 * distribution. Guided sampling weighs by this density. No reference counterpart. */
int  xb_bsdf_density(const xb_material *m, int64_t n, const float *wo, const float *wi, float *density);

/* ── learned path guiding (no reference counterpart: the reference has no learned part) ── */

/* A small network maps a surface point (position in the scene bounds, shading normal, outgoing
 * direction) to a mixture of 8 von Mises-Fisher lobes q over incoming directions and a selection
 * probability a. At every non-delta vertex seen from the front of its shading normal the next
 * direction is drawn from
 *     p(w) = a * q(w) + (1 - a) * p_bsdf(w)
 * (p_bsdf: the density of bsdf_sample), the vertex keeps the lobe, f and pdf the plain sampler
 * would have produced for w (so MIS weights, next-event estimation and Russian roulette are the
 * plain tracer's), and the path's radiance is weighted by the product of p_bsdf(w) / p(w) over
 * its guided vertices. The guided image therefore converges to the plain tracer's image for any
 * network and any scene. The network is trained online, on the first train_spp samples per
 * pixel, by Adam on the radiance-weighted negative log-likelihood of p at the sampled directions;
 * keep_training_samples says which of the training samples go into the image. BF16 tensor
 * cores (tcgen05), FP32 accumulation
 * and master weights. */
typedef struct xb_guiding {
  int32_t enabled;          /* 0: plain BSDF sampling (the reference's estimator) */
  int32_t train_spp;        /* train on samples 1..train_spp of each pixel; default 32, -1 = never */
  int32_t steps_per_spp;    /* Adam steps per training sample per pixel; default 64 */
  int32_t batch;            /* records per Adam step (multiple of 128); default 16384 */
  float learning_rate;      /* Adam step size at the start, decaying (cosine) to a tenth of it
                               over train_spp * steps_per_spp steps; default 5e-3 */
  float guide_fraction;     /* probability of sampling the network when fixed_fraction is set;
                               default 0.7 */
  int32_t max_records;      /* training records kept per wave; default 1 << 21 */
  int32_t record_stride;    /* record the vertices of one path in this many; 0 = automatic */
  uint64_t seed;            /* initial weights and batch windows */
  float bounds_min[3];      /* box mapped to [0,1]^3 for the network's position input; */
  float bounds_max[3];      /* an empty box selects the scene's bounds */
  int32_t keep_training_samples;  /* 0: samples 1..train_spp train the network only and stay out
                                   * of the image (xb_get_spp counts image samples); 1: they are
                                   * kept; 2: those after train_spp / 2 (rendered once half of
                                   * the Adam steps are taken) are kept */
  int32_t fixed_fraction;   /* 0: the network also outputs the probability of sampling it at each
                             * vertex (in [0.05, 0.6], trained with the mixture);
                             * 1: guide_fraction everywhere */
  int32_t guided_bounces;   /* the network proposes at bounces 0 .. guided_bounces - 1; later
                             * vertices sample their BSDF (the path's importance ratio carries
                             * on); default: every bounce */
  float ratio_cap;          /* bound on a path's importance ratio prod p_bsdf / p: at a guided
                             * vertex the probability of sampling the network is lowered to
                             * 1 - ratio / ratio_cap (0 once the ratio reaches the cap), so a
                             * path whose guided vertices missed its light cannot carry more than
                             * ratio_cap times the plain estimator's weight; the estimator stays
                             * unbiased. 0: default 2.5; < 0: no bound beyond each vertex's
                             * 1 / (1 - a) */
} xb_guiding;

/* Enables, disables or reconfigures guiding (0 fields take defaults). The first enabling, or a
 * new seed or max_records, creates a freshly initialised network; otherwise the network is kept,
 * across xb_reset too (samples 1..train_spp of every accumulation train it further). */
int  xb_set_guiding(xb_renderer *r, const xb_guiding *g);
int  xb_get_guiding(const xb_renderer *r, xb_guiding *out);

typedef struct xb_guiding_stats {
  int64_t adam_steps;       /* optimizer steps taken */
  int64_t records;          /* training records collected */
  int64_t records_dropped;  /* records beyond max_records */
  float last_loss;          /* mean loss of the last step */
  int32_t training;         /* 1 while spp < train_spp */
} xb_guiding_stats;
int  xb_get_guiding_stats(const xb_renderer *r, xb_guiding_stats *out);

/* The network's parameters: XB_GUIDE_PARAMS floats, W0 b0 W1 b1 W2 b2 W3 b3 with every W
 * row-major [out][in]; layers 64 -> 64 -> 64 -> 64 -> 48. */
#define XB_GUIDE_PARAMS 15600
int  xb_guide_get_params(xb_renderer *r, float *params);
int  xb_guide_set_params(xb_renderer *r, const float *params);

/* Standalone network calls on host buffers (parity tests and diagnostics).
 *   feats: rows x 9 (position in [0,1]^3, normal, outgoing direction)
 *   lobes: rows x 40, per lobe mean direction xyz, concentration kappa, weight; the forward call
 *          writes rows x 41: the lobes, then the selection probability a
 *   recs:  n x 24 training records: feats 9, direction 3, weight c, path, throughput 3,
 *          radiance 3, p_bsdf at the direction (< 0: the loss is that of q alone), 3 unused
 *          (the loss uses feats, direction, c and p_bsdf). */
int  xb_guide_init_params(uint64_t seed, float *params);
int  xb_guide_forward(const float *params, const float *feats, int64_t rows, float *lobes);
/* Loss sum(c * -log p(direction)) / sum(c), p = a q + (1 - a) p_bsdf, and its gradient with
 * respect to the parameters. */
int  xb_guide_loss_grad(const float *params, const float *recs, int64_t n, float *grad, float *loss);
/* `steps` Adam steps (lr, beta 0.9 / 0.99, eps 1e-8) on batches of `batch` records (tiles of 128
 * consecutive records at random starts; all records in order when n <= batch); params_out gets
 * the result, losses[steps] (optional) each step's loss. */
int  xb_guide_train(const float *params, const float *recs, int64_t n, int32_t steps, int32_t batch,
                    float lr, uint64_t seed, float *params_out, float *losses);
/* The device mixture pdf of one direction per row, and directions drawn from it by u (rows x 3). */
int  xb_guide_mixture_pdf(const float *lobes, int64_t rows, const float *dirs, float *pdf);
int  xb_guide_mixture_sample(const float *lobes, int64_t rows, const float *u, float *dirs, float *pdf);

/* ── diagnostics ──────────────────────────────────────────────────────────── */

/* D = A * B^T on the tensor cores (tcgen05, BF16 operands, FP32 accumulation in TMEM): the
 * building block of the guiding network's layers, exposed so it can be checked on its own.
 * A [rows x 64], B [n x 64] row-major bf16 bits, D [rows x n] f32; n in {16, 32, 48, 64}.
 * Host buffers. No reference counterpart (the reference has no tensor-core code). */
int  xb_tc_gemm_bf16(const uint16_t *A, const uint16_t *B, int64_t rows, int32_t n, float *D);

/* The failure path of the bounded device waits (every tensor-core step waits on an mbarrier with
 * a poll limit and reports XB_E_TIMEOUT instead of hanging): one warp waits on an mbarrier that
 * nothing completes (arrive = 0: returns XB_E_TIMEOUT) or that it completes itself (arrive = 1:
 * XB_OK). The context stays usable either way. */
int  xb_selftest_wait(int32_t arrive);

#ifdef __cplusplus
}
#endif
#endif /* XENON_B200_H */
