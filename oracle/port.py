"""ctypes binding of oracle/build/liboracle.so, this repo's CPU restatement of the reference path.

Test infrastructure (the checker): used by tests/, __graft_entry__.smoke() and bench.py's
reference leg (rays per path for the reference's Mrays/s, which the reference does not count).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "build", "liboracle.so")
_P, _I, _I64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64
_SIGS = {
    "xo_scene_new": ([_P], _P),
    "xo_scene_free": ([_P], None),
    "xo_trace": ([_P, _I64, _P, _P, _I, _P], _I),
    "xo_bsdf_eval": ([_P, _I64, _P, _P, _P, _P], None),
    "xo_bsdf_sample": ([_P, _I64, _P, _P, _P, _P, _P, _P], None),
    "xo_material_prepare": ([_P, _P], None),
    "xo_seed_pcg": ([ctypes.c_uint64], ctypes.c_uint64),
    "xo_render": ([_P, _P, _I, _I, _I, _I, _I, _I, _P, _P, _I], _I),
}
_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    return LIB


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        for k, (a, r) in _SIGS.items():
            getattr(L, k).argtypes = a
            getattr(L, k).restype = r
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


class PortScene:
    """The restatement's scene, copied from an xb_scene_view (abi.SceneView)."""

    def __init__(self, view):
        self.h = lib().xo_scene_new(ctypes.byref(view))

    def __del__(self):
        if getattr(self, "h", None):
            lib().xo_scene_free(self.h)
            self.h = None

    def trace(self, rays: np.ndarray, mode: int = 0):
        from xenon_b200.abi import HIT_DTYPE
        rays = np.ascontiguousarray(rays)
        hits = np.zeros(len(rays), HIT_DTYPE)
        work = np.zeros(4, np.int64)
        lib().xo_trace(self.h, len(rays), _p(rays), _p(hits), int(mode), _p(work))
        return hits, work

    def render(self, cam, w: int, h: int, min_b: int, max_b: int, spp_first: int, spp_count: int,
               threads: int = 0):
        s = np.zeros((h, w, 3), np.float64)
        rays = np.zeros(2, np.int64)
        lib().xo_render(self.h, ctypes.byref(cam), w, h, min_b, max_b, spp_first, spp_count, _p(s), _p(rays),
                        threads)
        return s, rays


def bsdf_eval(mat, wo, wi):
    wo = np.ascontiguousarray(wo, np.float32)
    wi = np.ascontiguousarray(wi, np.float32)
    f = np.zeros((len(wo), 3), np.float32)
    pdf = np.zeros(len(wo), np.float32)
    m = np.ascontiguousarray(mat, np.float32)
    lib().xo_bsdf_eval(_p(m), len(wo), _p(wo), _p(wi), _p(f), _p(pdf))
    return f, pdf


def bsdf_sample(mat, wo, states):
    wo = np.ascontiguousarray(wo, np.float32)
    n = len(wo)
    st = np.array(states, np.uint64, copy=True)
    wi = np.zeros((n, 3), np.float32)
    f = np.zeros((n, 3), np.float32)
    pdf = np.zeros(n, np.float32)
    fl = np.zeros(n, np.int32)
    m = np.ascontiguousarray(mat, np.float32)
    lib().xo_bsdf_sample(_p(m), n, _p(wo), _p(st), _p(wi), _p(f), _p(pdf), _p(fl))
    return wi, f, pdf, fl, st


def material_prepare(mat):
    from xenon_b200.abi import MaterialDerived
    out = MaterialDerived()
    m = np.ascontiguousarray(mat, np.float32)
    lib().xo_material_prepare(_p(m), ctypes.byref(out))
    return out


def seed_pcg(seed: int) -> int:
    return int(lib().xo_seed_pcg(seed))


def rays_per_path(view, cam, width: int, height: int, min_bounces: int, max_bounces: int,
                  paths: int = 4096) -> float:
    """Closest + shadow rays per path of the estimator on a coarse grid over a view: `view` is an
    xb_scene_view (e.g. the reference-built one, oracle/ref.py RefScene.view()) and `cam` the
    camera's four vectors (eye, lower-left, horizontal, vertical: float[12], e.g. oracle/ref.py
    camera()) for a width x height image."""
    from xenon_b200.abi import Camera
    ps = PortScene(view)
    side = max(8, int(paths ** 0.5))
    w = side
    h = max(1, int(side * height / width))
    _, rays = ps.render(Camera.from_array(cam), w, h, min_bounces, max_bounces, 7, 1)
    return float(rays.sum()) / (w * h)
