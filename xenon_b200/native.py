"""Loads libxenon_b200.so and declares the C ABI (include/xenon_b200.h) for ctypes.

There is no fallback: if the library is missing or no CUDA device exists, the calls fail with
an exception naming the problem.
"""
from __future__ import annotations

import ctypes
import os

from . import abi

_P = ctypes.c_void_p
_I = ctypes.c_int
_I32 = ctypes.c_int32
_I64 = ctypes.c_int64
_F = ctypes.c_float

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib", "libxenon_b200.so")

SIGNATURES = {
    "xb_material_default": ([_P], None),
    "xb_material_prepare": ([_P, _P], _I),
    "xb_material_load": ([ctypes.c_char_p, _P, ctypes.c_char_p, ctypes.c_size_t], _I),
    "xb_camera_look_at": ([_P, _P, _P, _F, _F, _P], _I),
    "xb_scene_create": ([ctypes.POINTER(_P)], _I),
    "xb_scene_destroy": ([_P], None),
    "xb_scene_add_material": ([_P, ctypes.c_char_p, _P], _I),
    "xb_scene_add_mesh": ([_P, _I32, _P, _P, _I32, _P, _P, _I32], _I),
    "xb_scene_transform_mesh": ([_P, _I32, _P, _F, _P], _I),
    "xb_scene_add_prim": ([_P, _P], _I),
    "xb_scene_add_light": ([_P, ctypes.c_uint32, ctypes.c_uint32, _P, _F], _I),
    "xb_scene_add_sun": ([_P, _P, _P, _F], _I),
    "xb_scene_set_sky": ([_P, _P], _I),
    "xb_scene_add_instance": ([_P, _I32, _P, _F, _P, _I32], _I),
    "xb_scene_build": ([_P], _I),
    "xb_scene_set_build_threads": ([_P, _I], _I),
    "xb_scene_set_build_mode": ([_P, _I], _I),
    "xb_scene_refit_mesh": ([_P, _I, _P, _P], _I),
    "xb_scene_get_view": ([_P, _P], _I),
    "xb_scene_load": ([ctypes.c_char_p, ctypes.POINTER(_P), _P, _P], _I),
    "xb_create": ([_P, ctypes.POINTER(_P)], _I),
    "xb_destroy": ([_P], None),
    "xb_last_error": ([_P, ctypes.c_char_p, ctypes.c_size_t], _I),
    "xb_upload_scene": ([_P, _P], _I),
    "xb_refit_mesh": ([_P, _I, _P, _P], _I),
    "xb_set_bounces": ([_P, _I32, _I32], _I),
    "xb_render": ([_P, _P, _I32], _I),
    "xb_render_range": ([_P, _P, _I32, _I32], _I),
    "xb_resolve": ([_P, _P], _I),
    "xb_resolve_fp64": ([_P, _P, _P], _I),
    "xb_resolve_fp64_device": ([_P, _P, _P], _I),
    "xb_get_spp": ([_P], _I),
    "xb_reset": ([_P], _I),
    "xb_get_render_stats": ([_P, _P], _I),
    "xb_reset_render_stats": ([_P], _I),
    "xb_trace_rays": ([_P, _P, _I64, _P, _I32], _I),
    "xb_trace_rays_device": ([_P, _P, _I64, _P, _I32, _P], _I),
    "xb_trace_rays_noalloc": ([_P, _P, _I64, _P, _I32, _P], _I),
    "xb_set_tuning": ([_P, _P], _I),
    "xb_get_tuning": ([_P, _P], _I),
    "xb_set_profiling": ([_P, _I32], _I),
    "xb_get_profile": ([_P, _P], _I),
    "xb_reset_profile": ([_P], _I),
    "xb_bsdf_eval": ([_P, _I64, _P, _P, _P, _P], _I),
    "xb_bsdf_sample": ([_P, _I64, _P, _P, _P, _P, _P, _P], _I),
    "xb_bsdf_density": ([_P, _I64, _P, _P, _P], _I),
    "xb_tc_gemm_bf16": ([_P, _P, _I64, _I32, _P], _I),
    "xb_selftest_wait": ([_I32], _I),
    "xb_render_views": ([_P, _P, _I32], _I),
    "xb_resolve_async": ([_P, _P], _I),
    "xb_sync": ([_P], _I),
    "xb_image_to_rgb8": ([_P, _I, _I, _P], _I),
    "xb_write_png": ([ctypes.c_char_p, _P, _I, _I], _I),
    "xb_image_noise_stats": ([_P, _I, _I, _P], _I),
    "xb_output_stage": ([_P, _P, _P], _I),
    "xb_write_png_rgb8": ([ctypes.c_char_p, _P, _I, _I], _I),
    "xb_set_guiding": ([_P, _P], _I),
    "xb_get_guiding": ([_P, _P], _I),
    "xb_get_guiding_stats": ([_P, _P], _I),
    "xb_guide_get_params": ([_P, _P], _I),
    "xb_guide_set_params": ([_P, _P], _I),
    "xb_guide_init_params": ([ctypes.c_uint64, _P], _I),
    "xb_guide_forward": ([_P, _P, _I64, _P], _I),
    "xb_guide_loss_grad": ([_P, _P, _I64, _P, _P], _I),
    "xb_guide_train": ([_P, _P, _I64, _I32, _I32, _F, ctypes.c_uint64, _P, _P], _I),
    "xb_guide_mixture_pdf": ([_P, _I64, _P, _P], _I),
    "xb_guide_mixture_sample": ([_P, _I64, _P, _P, _P], _I),
}

_lib = None


class XenonError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{abi.STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: the CUDA extension is not built "
                               "(run `python -m xenon_b200.build` or __graft_entry__.build())")
        L = ctypes.CDLL(LIB_PATH)
        for name, (args, res) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def last_error(handle=None) -> str:
    buf = ctypes.create_string_buffer(1024)
    lib().xb_last_error(handle, buf, len(buf))
    return buf.value.decode(errors="replace")


def check(rc: int, handle=None) -> int:
    if rc < 0:
        raise XenonError(rc, last_error(handle))
    return rc


def exported_symbols() -> list[str]:
    return sorted(SIGNATURES)
