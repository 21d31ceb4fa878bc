"""GPU path against the committed golden vectors (computed by the reference itself; no
reference code runs here): closest / any hit records, BSDF eval grids, and the converged
config-1 image (64x64, 4096 samples of the reference's render_frame_tiled)."""
import os

import numpy as np
import pytest

import xenon_b200 as xb
from tests.golden.gen_golden import BSDF_MATERIALS, TRACE_SCENES
from tests.helpers import compare_hits, prim_instance_ids
from tests.test_gpu_render import relmse
from xenon_b200 import HostScene, Renderer, abi, camera, scenes

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(TRACE_SCENES))
def test_trace_matches_golden(name):
    g = np.load(os.path.join(GOLD, "trace_bvh.npz"))
    desc = TRACE_SCENES[name]()
    r = Renderer(16, 16)
    r.upload_scene(HostScene.from_desc(desc))
    rays = g[f"trace_{name}_rays"]
    got = r.trace_rays(rays, abi.XB_TRACE_CLOSEST)
    d = compare_hits(got, g[f"trace_{name}_closest"], prim_ids=prim_instance_ids(desc))
    assert d["hit_mismatch"] == 0 and d["prim_id_mismatch"] == 0 and d["instance_id_mismatch"] == 0, d
    assert d["t_ulp_max"] <= 4 and d["u_ulp_max"] <= 4 and d["v_ulp_max"] <= 4, d
    got_any = r.trace_rays(rays, abi.XB_TRACE_ANY)
    assert np.array_equal(np.isfinite(got_any["t"]), g[f"trace_{name}_any"])


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(BSDF_MATERIALS))
def test_bsdf_matches_golden(name):
    g = np.load(os.path.join(GOLD, "bsdf.npz"))
    f, p = xb.bsdf_eval(g[f"{name}_material"], g["wo"], g["wi"])
    fw, pw = g[f"{name}_f"], g[f"{name}_pdf"]
    assert np.max(np.abs(f - fw) / np.maximum(np.abs(fw), 1e-6)) < 1e-5
    assert np.max(np.abs(p - pw) / np.maximum(np.abs(pw), 1e-6)) < 1e-5


@pytest.mark.gpu
def test_converged_config1_matches_golden():
    g = np.load(os.path.join(GOLD, "render.npz"))
    want = g["cornell64_mean"]
    spp = int(g["cornell64_spp"])
    desc = scenes.cornell()
    r = Renderer(64, 64, desc.max_bounces, desc.min_bounces)
    r.upload_scene(HostScene.from_desc(desc))
    r.render_frame(camera(desc.eye, desc.target, desc.fov, 1.0), spp)
    got = r.resolve()
    e = relmse(got, want)
    assert e < 1e-3, e
