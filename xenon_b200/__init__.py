"""xenon_b200 — B200-native wavefront path tracer behind Xenon's renderer-backend API.

Python face of the C ABI in include/xenon_b200.h (the C++17 face is csrc/b200_renderer.h):

    scene = HostScene.from_desc(desc)          # or HostScene.load("scene.xenon")
    r = Renderer(width, height, max_bounces, min_bounces)   # CudaRenderer(w, h, max, min)
    r.upload_scene(scene)                      # CudaRenderer::upload_scene
    r.render_frame(camera, spp=1)              # CudaRenderer::render_frame (adds samples)
    img = r.resolve()                          # float32 [H, W, 3], top-down rows
    r.spp                                      # CudaRenderer::spp

Every call goes to libxenon_b200.so; there is no CPU path. Failures raise XenonError.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import abi
from .native import XenonError, check, lib

__all__ = ["HostScene", "Renderer", "XenonError", "camera", "abi", "lib"]


def _p(a):
    # data_as keeps a reference to the array for as long as the pointer object lives
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def camera(eye, target, fov: float, aspect: float, up=(0.0, 1.0, 0.0)) -> abi.Camera:
    """Camera::look_at (src/camera/camera.h:15-31) → the device camera."""
    c = abi.Camera()
    e = np.asarray(eye, np.float32)
    t = np.asarray(target, np.float32)
    u = np.asarray(up, np.float32)
    check(lib().xb_camera_look_at(_p(e), _p(t), _p(u), float(fov), float(aspect), ctypes.byref(c)))
    return c


def material_prepare(m: np.ndarray) -> abi.MaterialDerived:
    out = abi.MaterialDerived()
    mm = np.ascontiguousarray(m, np.float32)
    check(lib().xb_material_prepare(_p(mm), ctypes.byref(out)))
    return out


class HostScene:
    """Host-side scene: meshes, prims, materials, lights, sky and the TLAS/BLAS build."""

    def __init__(self):
        h = ctypes.c_void_p()
        check(lib().xb_scene_create(ctypes.byref(h)))
        self.h = h
        self.config = None
        self.camera_desc = None

    def __del__(self):
        try:
            if getattr(self, "h", None) is not None and self.h.value:
                lib().xb_scene_destroy(self.h)
                self.h = None
        except Exception:       # interpreter shutdown: the library handle may be gone already
            pass

    @classmethod
    def from_desc(cls, desc, build_threads: int = 0, build_mode: int = abi.XB_BUILD_RECURSIVE,
                  build: bool = True) -> "HostScene":
        """Builds the scene's BVHs with `build_threads` threads (0: all hardware threads), in the
        recursive or the level-synchronous form (build_mode); the arrays are the same for any
        count and either form. build=False: the scene is filled but not built (build() does it)."""
        s = cls()
        L = lib()
        for name, m in zip(desc.material_names, desc.materials):
            arr = np.ascontiguousarray(m, np.float32)
            check(L.xb_scene_add_material(s.h, name.encode(), _p(arr)))
        for mesh in desc.meshes:
            pos = np.ascontiguousarray(mesh.positions, np.float32)
            nrm = None if mesh.normals is None else np.ascontiguousarray(mesh.normals, np.float32)
            idx = np.ascontiguousarray(mesh.indices, np.int32)
            mat = None if mesh.mat_ids is None else np.ascontiguousarray(mesh.mat_ids, np.int32)
            mid = check(L.xb_scene_add_mesh(s.h, len(pos), _p(pos), _p(nrm), len(idx), _p(idx), _p(mat),
                                            int(mesh.default_mat)))
            if mesh.transform is not None:
                t, sc, r = mesh.transform
                check(L.xb_scene_transform_mesh(s.h, mid, _p(np.asarray(t, np.float32)), float(sc),
                                                _p(np.asarray(r, np.float32))))
        for p in desc.prims:
            arr = np.ascontiguousarray(p)
            check(L.xb_scene_add_prim(s.h, _p(arr)))
        for (mesh_id, tri, e, area) in desc.lights:
            check(L.xb_scene_add_light(s.h, mesh_id, tri, _p(np.asarray(e, np.float32)), float(area)))
        for (d, c, inten) in desc.suns:
            check(L.xb_scene_add_sun(s.h, _p(np.asarray(d, np.float32)), _p(np.asarray(c, np.float32)),
                                     float(inten)))
        sky = np.ascontiguousarray(desc.sky, np.float32)
        check(L.xb_scene_set_sky(s.h, _p(sky)))
        for (geom, t, sc, r, iid) in desc.instances:
            check(L.xb_scene_add_instance(s.h, int(geom), _p(np.asarray(t, np.float32)), float(sc),
                                          _p(np.asarray(r, np.float32)), int(iid)))
        if build:
            s.build(build_threads, build_mode)
        return s

    def build(self, build_threads: int = 0, build_mode: int = abi.XB_BUILD_RECURSIVE) -> None:
        """xb_scene_build: the BVHs (BLAS per mesh, PrimBLAS, TLAS) and the flattened arrays."""
        L = lib()
        check(L.xb_scene_set_build_threads(self.h, int(build_threads)))
        check(L.xb_scene_set_build_mode(self.h, int(build_mode)))
        check(L.xb_scene_build(self.h))

    @classmethod
    def load(cls, path: str) -> "HostScene":
        """The .xenon loader (src/scene/scene_file.cpp:49-231), builds the BVHs too."""
        s = cls.__new__(cls)
        h = ctypes.c_void_p()
        cfg = abi.SceneConfig()
        cam = abi.CameraDesc()
        check(lib().xb_scene_load(str(path).encode(), ctypes.byref(h), ctypes.byref(cfg), ctypes.byref(cam)))
        s.h = h
        s.config = cfg
        s.camera_desc = cam
        return s

    def refit_mesh(self, mesh: int, positions, normals=None) -> None:
        """Moves mesh `mesh`'s vertices and refits its BLAS with the topology kept, then
        rebuilds the TLAS (xb_scene_refit_mesh). positions, normals: (num_vertices, 3)."""
        pos = np.ascontiguousarray(positions, np.float32)
        nrm = None if normals is None else np.ascontiguousarray(normals, np.float32)
        v = self.view()
        if not 0 <= mesh < v.num_meshes:
            raise XenonError(abi.XB_E_INVALID, f"refit_mesh: no mesh {mesh}")
        nv = v.meshes[mesh].num_vertices
        if pos.shape != (nv, 3) or (nrm is not None and nrm.shape != (nv, 3)):
            raise XenonError(abi.XB_E_INVALID, f"refit_mesh: mesh {mesh} has {nv} vertices")
        check(lib().xb_scene_refit_mesh(self.h, int(mesh), _p(pos), _p(nrm)))

    def view(self) -> abi.SceneView:
        """The flattened arrays; they belong to this scene, which the view keeps alive."""
        v = abi.SceneView()
        check(lib().xb_scene_get_view(self.h, ctypes.byref(v)))
        v._owner = self
        return v


class Renderer:
    """Mirrors xn::CudaRenderer (src/cuda/cuda_renderer.cuh:14-55) over the C ABI."""

    def __init__(self, width: int, height: int, max_bounces: int = 8, min_bounces: int = 3,
                 device: int = 0, fp64: bool = False, wave_paths: int = 0, flags: int = 0):
        cfg = abi.Config(width, height, max_bounces, min_bounces, device,
                         (abi.XB_FLAG_FP64_ACCUM if fp64 else 0) | flags, wave_paths, 0)
        h = ctypes.c_void_p()
        check(lib().xb_create(ctypes.byref(cfg), ctypes.byref(h)))
        self.h = h
        self.width, self.height = width, height
        self.fp64 = fp64

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            lib().xb_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:   # interpreter shutdown: the library handle may be gone already
            pass

    def _check(self, rc):
        return check(rc, self.h)

    def upload_scene(self, scene) -> None:
        """Accepts a HostScene or an abi.SceneView (e.g. exported from another builder)."""
        v = scene.view() if isinstance(scene, HostScene) else scene
        self._check(lib().xb_upload_scene(self.h, ctypes.byref(v)))
        self._mesh_vertices = [v.meshes[i].num_vertices for i in range(v.num_meshes)]

    def refit_mesh(self, mesh: int, positions, normals=None) -> None:
        """Moves an uploaded mesh's vertices and refits its BLAS on the device (xb_refit_mesh);
        positions, normals: (num_vertices, 3) float32 in host memory."""
        pos = np.ascontiguousarray(positions, np.float32)
        nrm = None if normals is None else np.ascontiguousarray(normals, np.float32)
        counts = getattr(self, "_mesh_vertices", [])
        if not 0 <= mesh < len(counts):
            raise XenonError(abi.XB_E_INVALID, f"refit_mesh: no uploaded mesh {mesh}")
        nv = counts[mesh]
        if pos.shape != (nv, 3) or (nrm is not None and nrm.shape != (nv, 3)):
            raise XenonError(abi.XB_E_INVALID, f"refit_mesh: mesh {mesh} has {nv} vertices")
        self._check(lib().xb_refit_mesh(self.h, int(mesh), _p(pos), _p(nrm)))

    def set_bounces(self, min_bounces: int, max_bounces: int) -> None:
        self._check(lib().xb_set_bounces(self.h, min_bounces, max_bounces))

    def render_frame(self, cam: abi.Camera, spp: int = 1) -> None:
        self._check(lib().xb_render(self.h, ctypes.byref(cam), int(spp)))

    def render_range(self, cam: abi.Camera, spp_first: int, spp_count: int) -> None:
        self._check(lib().xb_render_range(self.h, ctypes.byref(cam), int(spp_first), int(spp_count)))

    def render_views(self, views) -> list:
        """xb_render_views: views = [(camera, width, height, spp[, max_bounces]), ...] rendered
        together in shared waves; returns each view's mean image (height, width, 3), top-down."""
        arr = (abi.View * len(views))()
        outs = []
        for i, v in enumerate(views):
            cam, w, h, spp = v[:4]
            o = np.empty((h, w, 3), np.float32)
            outs.append(o)
            arr[i].camera = cam
            arr[i].width, arr[i].height, arr[i].spp = int(w), int(h), int(spp)
            arr[i].max_bounces = int(v[4]) if len(v) > 4 else 0
            arr[i].out_rgb = o.ctypes.data
        self._check(lib().xb_render_views(self.h, arr, len(views)))
        return outs

    def resolve(self, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.empty((self.height, self.width, 3), np.float32)
        self._check(lib().xb_resolve(self.h, _p(out)))
        return out

    def resolve_async(self, out: np.ndarray) -> None:
        """xb_resolve_async into `out` (float32 [H, W, 3], ideally page-locked); complete after sync()."""
        assert out.dtype == np.float32 and out.size == self.width * self.height * 3
        self._check(lib().xb_resolve_async(self.h, out.ctypes.data_as(ctypes.c_void_p)))

    def sync(self) -> None:
        self._check(lib().xb_sync(self.h))

    def resolve_fp64(self):
        s = np.empty((self.height, self.width, 3), np.float64)
        m2 = np.empty_like(s)
        self._check(lib().xb_resolve_fp64(self.h, _p(s), _p(m2)))
        return s, m2

    def output_stage(self, rgb8: bool = True, stats: bool = True):
        """xb_output_stage: the PNG's 8-bit pixels (H, W, 3) and the noise statistics of the current
        mean image, computed on the device; returns (rgb8 or None, stats dict or None)."""
        pix = np.empty((self.height, self.width, 3), np.uint8) if rgb8 else None
        st = abi.NoiseStats() if stats else None
        self._check(lib().xb_output_stage(self.h, _p(pix) if pix is not None else None,
                                          ctypes.byref(st) if st is not None else None))
        return pix, (st.as_dict() if st is not None else None)

    def resolve_fp64_device(self, sum_ptr: int, m2_ptr: int = 0) -> None:
        """xb_resolve_fp64_device: FP64 sums and Welford M2 (top-down rows) into device buffers
        of W*H*3 doubles on the renderer's GPU (e.g. torch tensors' data_ptr(); 0 skips one)."""
        self._check(lib().xb_resolve_fp64_device(self.h, ctypes.c_void_p(sum_ptr) if sum_ptr else None,
                                                 ctypes.c_void_p(m2_ptr) if m2_ptr else None))

    @property
    def spp(self) -> int:
        return int(lib().xb_get_spp(self.h))

    def reset(self) -> None:
        self._check(lib().xb_reset(self.h))

    def stats(self) -> abi.RenderStats:
        st = abi.RenderStats()
        self._check(lib().xb_get_render_stats(self.h, ctypes.byref(st)))
        return st

    def reset_stats(self) -> None:
        self._check(lib().xb_reset_render_stats(self.h))

    def set_tuning(self, **kw) -> None:
        """xb_set_tuning: fields of abi.Tuning; unnamed fields keep their value."""
        t = abi.Tuning(**kw)
        self._check(lib().xb_set_tuning(self.h, ctypes.byref(t)))

    def tuning(self) -> dict:
        t = abi.Tuning()
        self._check(lib().xb_get_tuning(self.h, ctypes.byref(t)))
        return t.as_dict()

    def set_profiling(self, flags: int) -> None:
        self._check(lib().xb_set_profiling(self.h, int(flags)))

    def profile(self) -> abi.Profile:
        p = abi.Profile()
        self._check(lib().xb_get_profile(self.h, ctypes.byref(p)))
        return p

    def reset_profile(self) -> None:
        self._check(lib().xb_reset_profile(self.h))

    def set_guiding(self, enabled: bool = True, **kw) -> None:
        """xb_set_guiding: learned path guiding; keyword fields of abi.Guiding (0 = default)."""
        g = abi.Guiding()
        g.enabled = 1 if enabled else 0
        for k, v in kw.items():
            if k in ("bounds_min", "bounds_max"):
                getattr(g, k)[:] = [float(x) for x in v]
            else:
                setattr(g, k, v)
        self._check(lib().xb_set_guiding(self.h, ctypes.byref(g)))

    def guiding(self) -> dict:
        g = abi.Guiding()
        self._check(lib().xb_get_guiding(self.h, ctypes.byref(g)))
        return g.as_dict()

    def guiding_stats(self) -> dict:
        st = abi.GuidingStats()
        self._check(lib().xb_get_guiding_stats(self.h, ctypes.byref(st)))
        return st.as_dict()

    def guide_params(self) -> np.ndarray:
        out = np.empty(abi.GUIDE_PARAMS, np.float32)
        self._check(lib().xb_guide_get_params(self.h, _p(out)))
        return out

    def set_guide_params(self, params: np.ndarray) -> None:
        p = np.ascontiguousarray(params, np.float32)
        assert p.shape == (abi.GUIDE_PARAMS,)
        self._check(lib().xb_guide_set_params(self.h, _p(p)))

    def trace_rays(self, rays: np.ndarray, mode: int = abi.XB_TRACE_CLOSEST) -> np.ndarray:
        rays = np.ascontiguousarray(rays)
        assert rays.dtype == abi.RAY_DTYPE
        hits = np.empty(len(rays), abi.HIT_DTYPE)
        self._check(lib().xb_trace_rays(self.h, _p(rays), len(rays), _p(hits), int(mode)))
        return hits

    def trace_rays_device(self, rays_ptr: int, n: int, hits_ptr: int, mode: int = 0, stream: int = 0) -> None:
        """xb_trace_rays_device on `stream` (a cudaStream_t handle; 0: the renderer's own stream,
        which does not wait for the legacy default stream — pass torch's stream explicitly)."""
        self._check(lib().xb_trace_rays_device(self.h, ctypes.c_void_p(rays_ptr), int(n),
                                               ctypes.c_void_p(hits_ptr), int(mode),
                                               ctypes.c_void_p(stream) if stream else None))


def image_to_rgb8(rgb: np.ndarray) -> np.ndarray:
    """xb_image_to_rgb8: the PNG's 8-bit pixels (top row first) of an image as resolve() returns it."""
    img = np.ascontiguousarray(rgb, np.float32)
    h, w = img.shape[:2]
    out = np.empty((h, w, 3), np.uint8)
    check(lib().xb_image_to_rgb8(_p(img), w, h, _p(out)))
    return out


def write_png(path: str, rgb: np.ndarray) -> None:
    """xb_write_png: an image as resolve() returns it, written as the reference's save_image does."""
    img = np.ascontiguousarray(rgb, np.float32)
    h, w = img.shape[:2]
    check(lib().xb_write_png(str(path).encode(), _p(img), w, h))


def write_png_rgb8(path: str, rgb8: np.ndarray) -> None:
    """xb_write_png_rgb8: 8-bit pixels (H, W, 3), top row first, as a PNG file."""
    pix = np.ascontiguousarray(rgb8, np.uint8)
    h, w = pix.shape[:2]
    check(lib().xb_write_png_rgb8(str(path).encode(), _p(pix), w, h))


def noise_stats(rgb: np.ndarray) -> dict:
    """xb_image_noise_stats: the reference's blur-residual noise statistics of an image."""
    img = np.ascontiguousarray(rgb, np.float32)
    h, w = img.shape[:2]
    st = abi.NoiseStats()
    check(lib().xb_image_noise_stats(_p(img), w, h, ctypes.byref(st)))
    return st.as_dict()


def bsdf_eval(mat: np.ndarray, wo: np.ndarray, wi: np.ndarray):
    """GPU eval/pdf for NEE (bsdf_eval_for_nee / bsdf_pdf_for_nee)."""
    wo = np.ascontiguousarray(wo, np.float32)
    wi = np.ascontiguousarray(wi, np.float32)
    n = len(wo)
    f = np.empty((n, 3), np.float32)
    pdf = np.empty(n, np.float32)
    m = np.ascontiguousarray(mat, np.float32)
    check(lib().xb_bsdf_eval(_p(m), n, _p(wo), _p(wi), _p(f), _p(pdf)))
    return f, pdf


def bsdf_density(mat: np.ndarray, wo: np.ndarray, wi: np.ndarray) -> np.ndarray:
    """True density of bsdf_sample's directions (xb_bsdf_density)."""
    wo = np.ascontiguousarray(wo, np.float32)
    wi = np.ascontiguousarray(wi, np.float32)
    out = np.empty(len(wo), np.float32)
    m = np.ascontiguousarray(mat, np.float32)
    check(lib().xb_bsdf_density(_p(m), len(wo), _p(wo), _p(wi), _p(out)))
    return out


def bsdf_sample(mat: np.ndarray, wo: np.ndarray, states):
    wo = np.ascontiguousarray(wo, np.float32)
    n = len(wo)
    st = np.array(states, dtype=np.uint64, copy=True)
    wi = np.empty((n, 3), np.float32)
    f = np.empty((n, 3), np.float32)
    pdf = np.empty(n, np.float32)
    flags = np.empty(n, np.int32)
    m = np.ascontiguousarray(mat, np.float32)
    check(lib().xb_bsdf_sample(_p(m), n, _p(wo), _p(st), _p(wi), _p(f), _p(pdf), _p(flags)))
    return wi, f, pdf, flags, st


# ── the guiding network on its own (xb_guide_*) ────────────────────────────────────
def guide_init_params(seed: int = 1) -> np.ndarray:
    out = np.empty(abi.GUIDE_PARAMS, np.float32)
    check(lib().xb_guide_init_params(int(seed), _p(out)))
    return out


def guide_forward(params: np.ndarray, feats: np.ndarray, with_selection: bool = False):
    """feats [rows, 9] (position in [0,1]^3, normal, outgoing direction) -> lobes [rows, 8, 5]
    (and the selection probabilities [rows] with with_selection)."""
    p = np.ascontiguousarray(params, np.float32)
    f = np.ascontiguousarray(feats, np.float32)
    out = np.empty((len(f), abi.GUIDE_OUT_FLOATS), np.float32)
    check(lib().xb_guide_forward(_p(p), _p(f), len(f), _p(out)))
    lobes = np.ascontiguousarray(out[:, :40]).reshape(len(f), 8, 5)
    return (lobes, out[:, 40].copy()) if with_selection else lobes


def guide_loss_grad(params: np.ndarray, recs: np.ndarray):
    p = np.ascontiguousarray(params, np.float32)
    r = np.ascontiguousarray(recs, np.float32)
    g = np.empty(abi.GUIDE_PARAMS, np.float32)
    loss = np.zeros(1, np.float32)
    check(lib().xb_guide_loss_grad(_p(p), _p(r), len(r), _p(g), _p(loss)))
    return float(loss[0]), g


def guide_train(params: np.ndarray, recs: np.ndarray, steps: int, batch: int, lr: float = 5e-3, seed: int = 1):
    p = np.ascontiguousarray(params, np.float32)
    r = np.ascontiguousarray(recs, np.float32)
    out = np.empty(abi.GUIDE_PARAMS, np.float32)
    losses = np.empty(steps, np.float32)
    check(lib().xb_guide_train(_p(p), _p(r), len(r), int(steps), int(batch), float(lr), int(seed), _p(out),
                               _p(losses)))
    return out, losses


def guide_mixture_pdf(lobes: np.ndarray, dirs: np.ndarray) -> np.ndarray:
    L = np.ascontiguousarray(lobes, np.float32).reshape(-1, abi.GUIDE_LOBE_FLOATS)
    d = np.ascontiguousarray(dirs, np.float32)
    out = np.empty(len(L), np.float32)
    check(lib().xb_guide_mixture_pdf(_p(L), len(L), _p(d), _p(out)))
    return out


def guide_mixture_sample(lobes: np.ndarray, u: np.ndarray):
    L = np.ascontiguousarray(lobes, np.float32).reshape(-1, abi.GUIDE_LOBE_FLOATS)
    uu = np.ascontiguousarray(u, np.float32)
    d = np.empty((len(L), 3), np.float32)
    pdf = np.empty(len(L), np.float32)
    check(lib().xb_guide_mixture_sample(_p(L), len(L), _p(uu), _p(d), _p(pdf)))
    return d, pdf
