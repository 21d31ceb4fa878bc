"""The C-ABI library loads and exports every function include/xenon_b200.h declares; without
a GPU the renderer entry points fail with a status, never abort."""
import ctypes
import os
import re

import pytest

import xenon_b200 as xb
from xenon_b200 import abi

HEADER = os.path.join(os.path.dirname(os.path.dirname(__file__)), "include", "xenon_b200.h")


def declared_functions() -> list[str]:
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:int|void|int64_t)\s+\**(xb_\w+)\s*\(", src, flags=re.M)))


def test_header_declares_the_boundary():
    names = declared_functions()
    for required in ("xb_create", "xb_destroy", "xb_upload_scene", "xb_render", "xb_resolve", "xb_get_spp",
                     "xb_reset", "xb_last_error", "xb_trace_rays", "xb_bsdf_eval", "xb_scene_load"):
        assert required in names


def test_library_exports_every_declared_symbol():
    L = xb.lib()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing
    # the Python binding declares the same set
    assert set(declared_functions()) <= set(xb.native.SIGNATURES)


def test_no_gpu_means_a_status_not_a_crash():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    cfg = abi.Config(64, 64, 8, 3, 0, 0, 0, 0)
    h = ctypes.c_void_p()
    rc = xb.lib().xb_create(ctypes.byref(cfg), ctypes.byref(h))
    assert rc == abi.XB_E_CUDA and not h.value
    assert "CUDA" in xb.native.last_error() or "device" in xb.native.last_error()


def test_invalid_arguments():
    L = xb.lib()
    assert L.xb_create(None, None) == abi.XB_E_INVALID
    bad = abi.Config(0, 64, 8, 3, 0, 0, 0, 0)
    h = ctypes.c_void_p()
    assert L.xb_create(ctypes.byref(bad), ctypes.byref(h)) == abi.XB_E_INVALID
    assert L.xb_render(None, None, 1) == abi.XB_E_INVALID
    assert L.xb_get_spp(None) == abi.XB_E_INVALID
    assert L.xb_bsdf_eval(None, 1, None, None, None, None) == abi.XB_E_INVALID
