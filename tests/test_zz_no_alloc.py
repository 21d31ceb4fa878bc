"""xb_trace_rays_noalloc: tracing for callers that cannot allocate device memory (a plugin
whose host application owns all device memory through its own allocator or a fixed budget).

The entry point must give exactly the hit records of xb_trace_rays_device, on two calls in a
row (its scratch is a fixed array shared by all calls, cleared at the start of each), and
must leave the device's free memory unchanged. This file is collected last on purpose."""
import ctypes
import os
import re

import numpy as np
import pytest

import xenon_b200 as xb
from tests.helpers import deep_chain_scene
from xenon_b200 import HostScene, Renderer, abi, scenes

_HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "xenon_b200.h")
NOALLOC_MAX_RAYS = 1 << int(re.search(r"#define XB_NOALLOC_MAX_RAYS \(\(int64_t\)1 << (\d+)\)",
                                         open(_HEADER).read()).group(1))


def _device_bytes(torch, arr: np.ndarray):
    t = torch.empty(arr.nbytes, dtype=torch.uint8, device="cuda")
    t.copy_(torch.from_numpy(arr.view(np.uint8).reshape(-1)))
    return t


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [abi.XB_TRACE_CLOSEST, abi.XB_TRACE_ANY])
def test_noalloc_trace_matches_trace_device(mode):
    import torch
    desc = scenes.instanced_grid(grid=3, levels=(3, 3, 4, 4), with_prims=True)
    r = Renderer(16, 16)
    r.upload_scene(HostScene.from_desc(desc))
    lo, hi = scenes.scene_bounds(desc)
    rays = scenes.random_rays((lo, hi), 50_000, seed=21)
    n = len(rays)
    d_rays = _device_bytes(torch, rays)
    d_ref = torch.zeros(n * abi.HIT_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    d_a = torch.zeros_like(d_ref)
    d_b = torch.zeros_like(d_ref)
    torch.cuda.synchronize()                 # the buffers' fills (torch's stream) before the traces
    ts = torch.cuda.Stream()                 # an explicit stream (kept alive): handle 0 means the renderer's own
    stream = ts.cuda_stream
    L = xb.lib()
    xb.native.check(L.xb_trace_rays_device(r.h, ctypes.c_void_p(d_rays.data_ptr()), n,
                                           ctypes.c_void_p(d_ref.data_ptr()), mode, ctypes.c_void_p(stream)), r.h)
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    for out in (d_a, d_b):     # two calls in a row share the scratch array
        xb.native.check(L.xb_trace_rays_noalloc(r.h, ctypes.c_void_p(d_rays.data_ptr()), n,
                                                ctypes.c_void_p(out.data_ptr()), mode, ctypes.c_void_p(stream)), r.h)
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    want = d_ref.cpu().numpy().view(abi.HIT_DTYPE)
    for out in (d_a, d_b):
        got = out.cpu().numpy().view(abi.HIT_DTYPE)
        assert np.array_equal(got["prim_id"], want["prim_id"])
        assert np.array_equal(got["instance_id"], want["instance_id"])
        assert got.tobytes() == want.tobytes()
    assert np.isfinite(want["t"]).sum() > n // 10
    assert free_after == free_before


@pytest.mark.gpu
def test_noalloc_rejects_bad_requests():
    desc = scenes.cornell()
    r = Renderer(16, 16)
    L = xb.lib()
    # no scene yet
    assert L.xb_trace_rays_noalloc(r.h, None, 0, None, 0, None) == abi.XB_E_STATE
    r.upload_scene(HostScene.from_desc(desc))
    # one ray over the limit is refused before anything is launched (the pointers are never read)
    too_many = NOALLOC_MAX_RAYS + 1
    assert L.xb_trace_rays_noalloc(r.h, ctypes.c_void_p(16), too_many, ctypes.c_void_p(16), 0, None) == abi.XB_E_INVALID
    assert f"maximum batch of {NOALLOC_MAX_RAYS}" in xb.native.last_error(r.h)
    assert L.xb_trace_rays_noalloc(r.h, ctypes.c_void_p(16), 4, ctypes.c_void_p(16), 7, None) == abi.XB_E_INVALID
    assert L.xb_trace_rays_noalloc(r.h, None, 0, None, 0, None) == abi.XB_OK


def test_noalloc_cursor_cannot_wrap():
    """The 64-bit work cursor ends at most 32 rays past the batch per warp of the grid (each warp's
    last fetch lands past the end). With the largest accepted batch and far more warps than any
    launch has (2^31: the grid is at most SMs x resident blocks x 4 warps), it stays below 2^63."""
    max_warps = 1 << 31
    assert NOALLOC_MAX_RAYS + 32 * (max_warps + 1) < (1 << 63)
    assert NOALLOC_MAX_RAYS >= (1 << 40)


@pytest.mark.gpu
def test_noalloc_reports_stack_overflow():
    """A BLAS deeper than the traversal stack: the rays that lose entries are counted in the
    renderer's overflow statistic, as xb_trace_rays_device counts them."""
    import torch
    hs, view, rays = deep_chain_scene(depth=100)
    r = Renderer(16, 16)
    r.upload_scene(view)
    n = len(rays)
    d_rays = _device_bytes(torch, rays)
    d_hits = torch.zeros(n * abi.HIT_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    L = xb.lib()
    torch.cuda.synchronize()
    ts = torch.cuda.Stream()
    stream = ts.cuda_stream
    counts = []
    for fn in (L.xb_trace_rays_device, L.xb_trace_rays_noalloc):
        before = r.stats().overflow
        xb.native.check(fn(r.h, ctypes.c_void_p(d_rays.data_ptr()), n, ctypes.c_void_p(d_hits.data_ptr()),
                           abi.XB_TRACE_CLOSEST, ctypes.c_void_p(stream)), r.h)
        torch.cuda.synchronize()
        counts.append(r.stats().overflow - before)
    assert counts[0] > 0, counts
    assert counts[1] > 0, counts
