"""ctypes binding of oracle/_ref (the reference's own CPU code behind ref_driver.cpp).

Test infrastructure: only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use
it, as the checker or as the timed CPU baseline. Two flavours are built by oracle/Makefile:
``strict`` (IEEE, no FMA contraction: the bit-exact checker) and ``fast`` (the reference's
Release flags: the CPU baseline).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_P = ctypes.c_void_p
_I = ctypes.c_int
_I64 = ctypes.c_int64
_F = ctypes.c_float

_SIGS = {
    "xr_scene_new": ([], _P),
    "xr_scene_free": ([_P], None),
    "xr_scene_add_material": ([_P, _P], _I),
    "xr_scene_add_mesh": ([_P, _I, _P, _P, _I, _P, _P, _I], _I),
    "xr_scene_transform_mesh": ([_P, _I, _P, _F, _P], _I),
    "xr_scene_mesh_arrays": ([_P, _I, _P, _P], _I),
    "xr_scene_add_prim": ([_P, _P], _I),
    "xr_scene_add_light": ([_P, ctypes.c_uint, ctypes.c_uint, _P, _F], _I),
    "xr_scene_add_sun": ([_P, _P, _P, _F], _I),
    "xr_scene_set_sky": ([_P, _P], None),
    "xr_scene_add_instance": ([_P, _I, _P, _F, _P, _I], _I),
    "xr_scene_build": ([_P], _I),
    "xr_scene_load_xenon": ([ctypes.c_char_p, ctypes.POINTER(_P), _P, _P], _I),
    "xr_material_prepare": ([_P, _P], None),
    "xr_material_load": ([ctypes.c_char_p, _P, ctypes.c_char_p, _I], _I),
    "xr_scene_view": ([_P, _P], _I),
    "xr_trace": ([_P, _I64, _P, _P, _I], _I),
    "xr_bsdf_eval": ([_P, _I64, _P, _P, _P, _P], None),
    "xr_bsdf_sample": ([_P, _I64, _P, _P, _P, _P, _P, _P], None),
    "xr_seed_pcg": ([ctypes.c_uint64], ctypes.c_uint64),
    "xr_camera": ([_P, _P, _F, _F, _P], None),
    "xr_renderer_new": ([_I, _I, _I, _I], _P),
    "xr_renderer_free": ([_P], None),
    "xr_render": ([_P, _P, _P, _I, _I, _P], ctypes.c_double),
    "xr_hardware_threads": ([], _I),
    "xr_noise_stats": ([_P, _I, _I, _P, _P], None),
    "xr_image_rgb8": ([_P, _I64, _P], None),
}

_LIBS: dict[str, ctypes.CDLL] = {}


def lib(flavour: str = "strict") -> ctypes.CDLL:
    if flavour not in _LIBS:
        path = os.path.join(HERE, "_ref", f"libxnref_{flavour}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle ref` where the reference sources are")
        L = ctypes.CDLL(path)
        for name, (args, res) in _SIGS.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _LIBS[flavour] = L
    return _LIBS[flavour]


def available(flavour: str = "strict") -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", f"libxnref_{flavour}.so"))


def ptr(a: np.ndarray | None):
    # data_as keeps a reference to the array for as long as the pointer object lives
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


class RefScene:
    """A reference Scene built from a scene description (see xenon_b200.scenes.SceneDesc)."""

    def __init__(self, desc, flavour: str = "strict"):
        self.L = lib(flavour)
        self.h = self.L.xr_scene_new()
        self._keep = []
        L = self.L
        for m in desc.materials:
            arr = np.ascontiguousarray(m, dtype=np.float32)
            L.xr_scene_add_material(self.h, ptr(arr))
        for mesh in desc.meshes:
            pos = np.ascontiguousarray(mesh.positions, np.float32)
            nrm = None if mesh.normals is None else np.ascontiguousarray(mesh.normals, np.float32)
            idx = np.ascontiguousarray(mesh.indices, np.int32)
            mat = None if mesh.mat_ids is None else np.ascontiguousarray(mesh.mat_ids, np.int32)
            mid = L.xr_scene_add_mesh(self.h, len(pos), ptr(pos), ptr(nrm), len(idx), ptr(idx), ptr(mat),
                                      int(mesh.default_mat))
            if mesh.transform is not None:
                t, s, r = mesh.transform
                L.xr_scene_transform_mesh(self.h, mid, ptr(np.asarray(t, np.float32)), float(s),
                                          ptr(np.asarray(r, np.float32)))
        for p in desc.prims:
            arr = np.ascontiguousarray(p)
            L.xr_scene_add_prim(self.h, ptr(arr))
        for (mesh_id, tri, e, area) in desc.lights:
            L.xr_scene_add_light(self.h, mesh_id, tri, ptr(np.asarray(e, np.float32)), float(area))
        for (d, c, inten) in desc.suns:
            L.xr_scene_add_sun(self.h, ptr(np.asarray(d, np.float32)), ptr(np.asarray(c, np.float32)), float(inten))
        sky = np.ascontiguousarray(desc.sky, np.float32)
        L.xr_scene_set_sky(self.h, ptr(sky))
        for (geom, t, s, r, iid) in desc.instances:
            L.xr_scene_add_instance(self.h, int(geom), ptr(np.asarray(t, np.float32)), float(s),
                                    ptr(np.asarray(r, np.float32)), int(iid))
        if L.xr_scene_build(self.h) != 0:
            raise RuntimeError("reference scene build failed")

    def __del__(self):
        if getattr(self, "h", None):
            self.L.xr_scene_free(self.h)
            self.h = None

    def trace(self, rays: np.ndarray, mode: int = 0) -> np.ndarray:
        from xenon_b200.abi import HIT_DTYPE
        rays = np.ascontiguousarray(rays)
        hits = np.zeros(len(rays), dtype=HIT_DTYPE)
        self.L.xr_trace(self.h, len(rays), ptr(rays), ptr(hits), int(mode))
        return hits

    def view(self):
        """(xb_scene_view bytes, keepalive) of the reference-built scene."""
        from xenon_b200.abi import SceneView
        v = SceneView()
        if self.L.xr_scene_view(self.h, ctypes.byref(v)) != 0:
            raise RuntimeError("xr_scene_view failed")
        v._owner = self
        return v

    def mesh_arrays(self, mesh: int, nv: int):
        pos = np.zeros((nv, 3), np.float32)
        nrm = np.zeros((nv, 3), np.float32)
        self.L.xr_scene_mesh_arrays(self.h, mesh, ptr(pos), ptr(nrm))
        return pos, nrm


class RefRenderer:
    """WavefrontRenderer::render_frame_tiled, one sample index at a time, summed in FP64."""

    def __init__(self, w: int, h: int, min_bounces: int, max_bounces: int, flavour: str = "strict"):
        self.L = lib(flavour)
        self.w, self.h = w, h
        self.r = self.L.xr_renderer_new(w, h, min_bounces, max_bounces)

    def __del__(self):
        if getattr(self, "r", None):
            self.L.xr_renderer_free(self.r)
            self.r = None

    def render(self, scene: RefScene, eye, target, fov, spp_first: int, spp_count: int, out_sum=None):
        """Adds samples [spp_first, spp_first+spp_count) into out_sum (float64 [H,W,3], top-down).
        Returns (out_sum, seconds spent in render_frame_tiled)."""
        if out_sum is None:
            out_sum = np.zeros((self.h, self.w, 3), np.float64)
        cam = np.array(list(eye) + list(target) + [fov], np.float32)
        secs = self.L.xr_render(self.r, scene.h, ptr(cam), int(spp_first), int(spp_count), ptr(out_sum))
        return out_sum, secs


def bsdf_eval(mat: np.ndarray, wo: np.ndarray, wi: np.ndarray):
    L = lib("strict")
    wo = np.ascontiguousarray(wo, np.float32)
    wi = np.ascontiguousarray(wi, np.float32)
    n = len(wo)
    f = np.zeros((n, 3), np.float32)
    pdf = np.zeros(n, np.float32)
    m = np.ascontiguousarray(mat, np.float32)
    L.xr_bsdf_eval(ptr(m), n, ptr(wo), ptr(wi), ptr(f), ptr(pdf))
    return f, pdf


def bsdf_sample(mat: np.ndarray, wo: np.ndarray, states: np.ndarray):
    L = lib("strict")
    wo = np.ascontiguousarray(wo, np.float32)
    n = len(wo)
    st = np.array(states, dtype=np.uint64, copy=True)
    wi = np.zeros((n, 3), np.float32)
    f = np.zeros((n, 3), np.float32)
    pdf = np.zeros(n, np.float32)
    flags = np.zeros(n, np.int32)
    m = np.ascontiguousarray(mat, np.float32)
    L.xr_bsdf_sample(ptr(m), n, ptr(wo), ptr(st), ptr(wi), ptr(f), ptr(pdf), ptr(flags))
    return wi, f, pdf, flags, st


def seed_pcg(seed: int) -> int:
    return int(lib("strict").xr_seed_pcg(seed))


def camera(eye, target, fov, aspect) -> np.ndarray:
    out = np.zeros(12, np.float32)
    lib("strict").xr_camera(ptr(np.asarray(eye, np.float32)), ptr(np.asarray(target, np.float32)),
                            float(fov), float(aspect), ptr(out))
    return out


def noise_stats(rgb: np.ndarray):
    """The reference's ImageNoiseEstimator on an (h, w, 3) float32 image: (10 floats, 2 counts)."""
    img = np.ascontiguousarray(rgb, np.float32)
    h, w = img.shape[:2]
    out = np.zeros(10, np.float32)
    counts = np.zeros(2, np.int32)
    lib().xr_noise_stats(ptr(img), w, h, ptr(out), ptr(counts))
    return out, counts


def image_rgb8(rgb: np.ndarray) -> np.ndarray:
    """save_image's 8-bit values of an (h, w, 3) float32 image (before its vertical flip)."""
    img = np.ascontiguousarray(rgb, np.float32)
    out = np.zeros(img.shape, np.uint8)
    lib().xr_image_rgb8(ptr(img), img.size, ptr(out))
    return out
