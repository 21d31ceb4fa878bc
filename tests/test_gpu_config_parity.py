"""Parity on the benchmarked configurations at their own sizes.

* Traversal (parity check (a)): closest-hit and any-hit answers against the reference's strict
  build (Scene::intersect / Scene::intersects, src/geometry/tlas.cpp:172-290,
  src/geometry/blas.cpp:211-307) on config 2's level-8 mesh (1.31 M triangles, BVH depth 26),
  config 3's full 16x16 instance grid and config 4's 500k-triangle glass sphere in the room;
  rays: 2^16 incoherent rays (origins uniform in the world bounds, directions uniform on the
  sphere) and 2^16 secondary rays harvested from bounce 2 of the path tracer's own sampling.
  Ids bit-exact; t, u, v within 4 ulp.
* Images (parity check (c)): config 2's view at 240x135 (1/64 of its pixels) per pixel against
  render_frame_tiled (src/render/cpu_tiled.cpp:13-237) with the same seeds; config 1 at its
  own 256x256 converged over samples 1..16384 against the reference's render of the same
  samples (tests/golden/config1_256.npz, made by tests/golden/gen_golden.py config1).
"""
import os

import numpy as np
import pytest

from tests.helpers import compare_hits, prim_instance_ids
from tests.test_gpu_render import per_pixel_agreement, relmse
from xenon_b200 import HostScene, Renderer, abi, camera, raybatch, scenes

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

CONFIGS = {
    "config2_L8": lambda: scenes.icosphere_scene(),
    "config3_grid": lambda: scenes.instanced_grid(),
    "config4_room": lambda: scenes.guiding_room(),
}


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CONFIGS))
def test_traversal_matches_reference_at_full_size(name, ref):
    desc = CONFIGS[name]()
    hs = HostScene.from_desc(desc)
    r = Renderer(64, 64)
    r.upload_scene(hs)
    cam = camera(desc.eye, desc.target, desc.fov, desc.width / desc.height)
    inc = raybatch.incoherent_rays(hs.view(), 1 << 16, seed=31)
    sec = raybatch.secondary_rays(r, desc.materials, cam, desc.width, desc.height, 1 << 16, seed=32, bounce=2)
    rs = ref.RefScene(desc)
    for label, rays in (("incoherent", inc), ("bounce2", sec)):
        got = r.trace_rays(rays, abi.XB_TRACE_CLOSEST)
        want = rs.trace(rays, abi.XB_TRACE_CLOSEST)
        d = compare_hits(got, want, prim_ids=prim_instance_ids(desc))
        print(name, label, d)
        assert d["hits"] > len(rays) // 20, d
        assert d["hit_mismatch"] == 0, (label, d)
        assert d["prim_id_mismatch"] == 0 and d["instance_id_mismatch"] == 0 and d["mat_id_mismatch"] == 0, (label, d)
        assert d["t_ulp_max"] <= 4 and d["u_ulp_max"] <= 4 and d["v_ulp_max"] <= 4, (label, d)
        assert d["front_mismatch"] == 0, (label, d)
        assert d["normal_maxabs"] < 1e-5 and d["geo_normal_maxabs"] < 1e-5, (label, d)
        got_any = r.trace_rays(rays, abi.XB_TRACE_ANY)
        want_any = rs.trace(rays, abi.XB_TRACE_ANY)
        assert np.array_equal(np.isfinite(got_any["t"]), np.isfinite(want_any["t"])), label
    assert r.stats().overflow == 0


@pytest.mark.gpu
def test_config2_view_agrees_per_pixel(ref):
    """The bench's config-2 view (level-8 mesh, sun + sky, depth 10) at 240x135, samples 1 and 2."""
    desc = scenes.icosphere_scene()
    w, h = desc.width // 8, desc.height // 8
    rr = ref.RefRenderer(w, h, desc.min_bounces, desc.max_bounces)
    s, _ = rr.render(ref.RefScene(desc), desc.eye, desc.target, desc.fov, 1, 2)
    want = s / 2
    r = Renderer(w, h, desc.max_bounces, desc.min_bounces)
    r.upload_scene(HostScene.from_desc(desc))
    r.render_range(camera(desc.eye, desc.target, desc.fov, w / h), 1, 2)
    got = r.resolve()
    assert r.stats().overflow == 0
    frac = per_pixel_agreement(got, want)
    print("config2 240x135 per-pixel agreement", frac, "relmse", relmse(got, want))
    assert frac > 0.97, frac
    assert relmse(got, want) < 1e-2


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["config3_grid", "config4_room"])
def test_config_views_agree_per_pixel(name, ref):
    """Config 3 (the full 16x16 instance grid, random diffuse / conductor / dielectric materials,
    sky + 4 quad lights, depth 12) and config 4 (the closed room, the light behind the baffle, the
    500k-triangle glass sphere, depth 16) at 1/8 of their pixels, samples 1 and 2, per pixel
    against the reference's render_frame_tiled with the same seeds."""
    desc = CONFIGS[name]()
    w, h = desc.width // 8, desc.height // 8
    rr = ref.RefRenderer(w, h, desc.min_bounces, desc.max_bounces)
    s, _ = rr.render(ref.RefScene(desc), desc.eye, desc.target, desc.fov, 1, 2)
    want = s / 2
    ok = np.isfinite(want).all(-1)   # the reference keeps non-finite path radiance
    r = Renderer(w, h, desc.max_bounces, desc.min_bounces)
    r.upload_scene(HostScene.from_desc(desc))
    r.render_range(camera(desc.eye, desc.target, desc.fov, w / h), 1, 2)
    got = r.resolve()
    assert r.stats().overflow == 0
    frac = per_pixel_agreement(got[ok], want[ok])
    print(name, f"{w}x{h} per-pixel agreement", frac, "relmse", relmse(got[ok], want[ok]),
          "reference non-finite pixels", int((~ok).sum()))
    assert (~ok).sum() <= 0.001 * ok.size
    assert frac > 0.97, frac


@pytest.mark.gpu
def test_config1_converged_at_full_size():
    """Config 1 (256x256 Cornell box) over samples 1..16384 against the reference's own render of
    the same samples: per-pixel relMSE below 1e-3."""
    g = np.load(os.path.join(GOLD, "config1_256.npz"))
    want, spp = g["mean"], int(g["spp"])
    desc = scenes.cornell()
    r = Renderer(desc.width, desc.height, desc.max_bounces, desc.min_bounces, fp64=True)
    r.upload_scene(HostScene.from_desc(desc))
    cam = camera(desc.eye, desc.target, desc.fov, desc.width / desc.height)
    for first in range(1, spp + 1, 1024):
        r.render_range(cam, first, min(1024, spp + 1 - first))
    got = r.resolve()
    # the reference accumulates non-finite path radiance (it has no guard): the few pixels where
    # one of its 16k samples was NaN are NaN in its image and are left out, as the parity rules
    # for NaN say; this library drops such samples and counts them (stats().nonfinite)
    ok = np.isfinite(want).all(-1)
    assert (~ok).sum() <= 8, (~ok).sum()
    e = relmse(got[ok], want[ok])
    print("config1 256x256 16k spp relMSE", e, "mean", got[ok].mean(), want[ok].mean(),
          "reference NaN pixels", int((~ok).sum()), "dropped samples", r.stats().nonfinite)
    assert r.stats().overflow == 0
    assert np.isfinite(got).all()
    assert e < 1e-3, e
    assert abs(got[ok].mean() / want[ok].mean() - 1) < 1e-3
