"""Parity (c): the GPU wavefront render against the reference CPU backend
(WavefrontRenderer::render_frame_tiled, src/render/cpu_tiled.cpp:13-237) on the same scene,
camera, bounces and per-pixel seeds.

Both sides seed sample k of pixel p with seed_pcg(p + k * 0xdeadbeef) and draw random numbers
in the same order, so low-spp images agree pixel by pixel except where a float transcendental
(CUDA's sinf/cosf/powf vs glibc's, both within 2 ulp) tips a discrete decision; converged
images agree to relMSE < 1e-3.
"""
import numpy as np
import pytest

from xenon_b200 import HostScene, Renderer, camera, scenes


def relmse(a: np.ndarray, b: np.ndarray, eps: float = 1e-2) -> float:
    """Per-pixel relative MSE, averaged: mean((a - b)^2 / (b^2 + eps)) over finite pixels of b."""
    lum_a, lum_b = a.mean(-1), b.mean(-1)
    ok = np.isfinite(lum_b)
    return float(np.mean((lum_a[ok] - lum_b[ok]) ** 2 / (lum_b[ok] ** 2 + eps)))


def gpu_render(desc, spp_first, spp_count, w, h, fp64=False):
    r = Renderer(w, h, desc.max_bounces, desc.min_bounces, fp64=fp64)
    r.upload_scene(HostScene.from_desc(desc))
    cam = camera(desc.eye, desc.target, desc.fov, w / h)
    r.render_range(cam, spp_first, spp_count)
    return r


def ref_render(ref, desc, spp_first, spp_count, w, h):
    rr = ref.RefRenderer(w, h, desc.min_bounces, desc.max_bounces)
    s, _ = rr.render(ref.RefScene(desc), desc.eye, desc.target, desc.fov, spp_first, spp_count)
    return s / spp_count


def per_pixel_agreement(a, b, tol=1e-3):
    d = np.abs(a - b).max(-1)
    scale = np.maximum(np.abs(b).max(-1), 1e-3)
    return float(np.mean(d / scale < tol))


@pytest.mark.gpu
@pytest.mark.parametrize("name,builder,w,h", [
    ("cornell", lambda: scenes.cornell(), 96, 96),
    ("prims", lambda: scenes.prim_showcase(), 96, 72),
    ("icosphere_sun", lambda: scenes.icosphere_scene(level=4), 96, 54),
    ("instanced", lambda: scenes.instanced_grid(grid=3, levels=(3, 3, 3, 3), with_prims=True), 96, 54),
])
def test_low_spp_images_agree_per_pixel(name, builder, w, h, ref):
    desc = builder()
    want = ref_render(ref, desc, 1, 2, w, h)
    r = gpu_render(desc, 1, 2, w, h)
    got = r.resolve()
    st = r.stats()
    assert st.overflow == 0
    frac = per_pixel_agreement(got, want)
    assert frac > 0.97, (name, frac)
    assert relmse(got, want) < 1e-2, (name, relmse(got, want))


@pytest.mark.gpu
def test_render_accumulates_like_render_frame(ref):
    """render_frame adds samples 1, 2, 3...: two calls of 2 equal one call of 4."""
    desc = scenes.cornell()
    cam = camera(desc.eye, desc.target, desc.fov, 1.0)
    r1 = Renderer(48, 48, desc.max_bounces, desc.min_bounces)
    r1.upload_scene(HostScene.from_desc(desc))
    r1.render_frame(cam, 2)
    r1.render_frame(cam, 2)
    r2 = Renderer(48, 48, desc.max_bounces, desc.min_bounces)
    r2.upload_scene(HostScene.from_desc(desc))
    r2.render_frame(cam, 4)
    assert r1.spp == 4 and r2.spp == 4
    assert np.array_equal(r1.resolve(), r2.resolve())


@pytest.mark.gpu
@pytest.mark.parametrize("builder", [lambda: scenes.cornell(), lambda: scenes.icosphere_scene(level=5),
                                     lambda: scenes.instanced_grid(grid=3, levels=(3, 3, 3, 3), with_prims=True)])
def test_traversal_variants_render_identically(builder):
    """Persistent-warp traversal and one-ray-per-thread traversal visit each ray's nodes in the
    same order (closest hit) or return the same occlusion answer (any hit): images are equal."""
    from xenon_b200 import abi
    desc = builder()
    imgs = []
    for flags, tune in ((0, {}), (abi.XB_FLAG_THREAD_PER_RAY, {}), (0, {"overlap": 2}),
                        (0, {"shade_occupancy": 4}), (0, {"shade_occupancy": 12}), (0, {"shade_occupancy": 16}),
                        (0, {"extend_persistent_from_depth": 1, "shadow_order": 2, "refill": 4}),
                        (0, {"shared_stack": 16}),
                        (0, {"shared_stack": 16, "extend_persistent_from_depth": 1, "shadow_persistent": 2}),
                        (0, {"pixel_order": 1}), (0, {"pixel_order": 1, "waves": 3})):
        r = Renderer(64, 48, desc.max_bounces, desc.min_bounces, flags=flags)
        r.upload_scene(HostScene.from_desc(desc))
        if tune:
            r.set_tuning(**tune)
        r.render_frame(camera(desc.eye, desc.target, desc.fov, 64 / 48), 3)
        imgs.append(r.resolve())
    for img in imgs[1:]:
        assert np.array_equal(imgs[0], img)


@pytest.mark.gpu
@pytest.mark.parametrize("flags", [0, 1])
def test_opaque_scene_bounce_renders_like_the_general_one(flags):
    """A scene without delta, transmissive or subsurface materials shades with the bounce kernel
    compiled without those lobes; adding an unused glass material selects the general kernel, and
    the images are equal."""
    from xenon_b200 import abi
    imgs = []
    for extra in (False, True):
        desc = scenes.icosphere_scene(level=5)
        if extra:   # listed, never referenced by a triangle
            desc.add_material("unused_glass", abi.material(base_color=(1.0, 1.0, 1.0), transmission=1.0,
                                                           roughness=0.0, ior=1.5))
        r = Renderer(64, 48, desc.max_bounces, desc.min_bounces,
                     flags=abi.XB_FLAG_THREAD_PER_RAY if flags else 0)
        r.upload_scene(HostScene.from_desc(desc))
        r.render_frame(camera(desc.eye, desc.target, desc.fov, 64 / 48), 3)
        imgs.append(r.resolve())
    assert np.array_equal(imgs[0], imgs[1])


@pytest.mark.gpu
def test_two_waves_in_flight_render_identically():
    """Consecutive waves on two to four stream lanes accumulate in sample order: the images (FP32
    and FP64 sums, plain and guided, one view and many) equal the one-lane images bit for bit."""
    desc = scenes.instanced_grid(grid=3, levels=(3, 3, 3, 3), with_prims=True)
    hs = HostScene.from_desc(desc)
    W, H = 64, 48
    cam = camera(desc.eye, desc.target, desc.fov, W / H)
    views = [(camera(desc.eye, desc.target, f, 1.0), s, s, spp, mb)
             for f, s, spp, mb in ((40.0, 32, 3, 0), (55.0, 48, 2, 4), (30.0, 40, 4, 6))]
    params = None
    out = {}
    for waves in (1, 2, 3, 4):
        r = Renderer(W, H, desc.max_bounces, desc.min_bounces, fp64=True, wave_paths=W * H)
        r.upload_scene(hs)
        r.set_tuning(waves=waves)
        assert r.tuning()["waves"] == waves
        r.render_frame(cam, 5)                   # five waves of one sample each
        s64, m2 = r.resolve_fp64()
        res = [r.resolve(), s64, m2]
        r.set_guiding(True, train_spp=-1)
        if params is None:
            params = r.guide_params()
        r.set_guide_params(params)
        r.reset()
        r.render_frame(cam, 4)
        res.append(r.resolve())
        res += r.render_views(views)             # views split over several waves
        r.close()
        out[waves] = res
    for waves in (2, 3, 4):
        for a, b in zip(out[1], out[waves]):
            assert np.array_equal(a, b)


@pytest.mark.gpu
def test_captured_bounce_loops_render_identically():
    """Replayed CUDA graphs of the bounce loop give the direct launches' images, and a change of
    bounces, guiding or scene drops the captured graphs (the next render matches a fresh one)."""
    desc = scenes.instanced_grid(grid=3, levels=(3, 3, 3, 3), with_prims=True)
    hs = HostScene.from_desc(desc)
    other = HostScene.from_desc(scenes.cornell())
    W, H = 64, 48
    cam = camera(desc.eye, desc.target, desc.fov, W / H)

    def fresh(graph, bounces=None, guided=False, scene=hs, spp=4):
        r = Renderer(W, H, desc.max_bounces, desc.min_bounces, wave_paths=W * H)
        r.upload_scene(scene)
        r.set_tuning(graph=graph)
        if bounces:
            r.set_bounces(desc.min_bounces, bounces)
        if guided:
            r.set_guiding(True, train_spp=-1)
        r.render_frame(cam, spp)
        img = r.resolve().copy()
        r.close()
        return img

    for kw in ({}, {"guided": True}):
        assert np.array_equal(fresh(1, **kw), fresh(2, **kw))
    views = [(camera(desc.eye, desc.target, f, 1.0), sz, sz, spp, mb)
             for f, sz, spp, mb in ((40.0, 32, 3, 0), (55.0, 48, 2, 4), (30.0, 40, 4, 6))]
    vimgs = []
    for graph in (1, 2):
        r = Renderer(W, H, desc.max_bounces, desc.min_bounces, wave_paths=W * H)
        r.upload_scene(hs)
        r.set_tuning(graph=graph)
        vimgs.append(r.render_views(views) + r.render_views(views))   # the second call replays
        r.close()
    for a, b in zip(*vimgs):
        assert np.array_equal(a, b)
    r = Renderer(W, H, desc.max_bounces, desc.min_bounces, wave_paths=W * H)
    r.upload_scene(hs)
    r.set_tuning(graph=1)
    r.render_frame(cam, 4)                      # captures the graphs
    assert np.array_equal(r.resolve(), fresh(2))
    r.reset()
    r.set_bounces(desc.min_bounces, 3)
    r.render_frame(cam, 4)
    assert np.array_equal(r.resolve(), fresh(2, bounces=3))
    r.reset()
    r.set_guiding(True, train_spp=-1)
    r.render_frame(cam, 4)
    assert np.array_equal(r.resolve(), fresh(2, bounces=3, guided=True))
    r.set_guiding(False)
    r.set_bounces(desc.min_bounces, desc.max_bounces)
    r.upload_scene(other)
    r.reset()
    r.render_frame(cam, 4)
    assert np.array_equal(r.resolve(), fresh(2, scene=other))
    r.close()


@pytest.mark.gpu
def test_sun_nee_flag_lights_a_lambertian_ground():
    """XB_FLAG_SUN_NEE: a Lambertian ground of albedo a under a sun of irradiance E at angle t
    and no sky shows a E cos t / pi in every pixel at one bounce; without the flag (the
    reference's 1e8 divisor) it shows 1e-8 of that."""
    from xenon_b200 import abi
    d = scenes.SceneDesc(name="sun", width=32, height=24, spp=1, max_bounces=1)
    ground = d.add_material("g", abi.material(base_color=(0.5, 0.4, 0.3), roughness=1.0, ior=1.0))
    d.add_mesh(scenes.quad_mesh((-50, 0, 50), (100, 0, 0), (0, 0, -100), ground))
    sun = np.array([0.3, 0.8, -0.2])
    sun /= np.linalg.norm(sun)
    d.suns.append((tuple(sun), (1.0, 0.9, 0.8), 2.0))
    d.sky = scenes.sky_array(intensity=0.0)
    d.eye, d.target, d.fov = (0.0, 10.0, 10.0), (0.0, 0.0, 0.0), 20.0
    hs = HostScene.from_desc(d)
    want = np.array([0.5, 0.4, 0.3]) * np.array([1.0, 0.9, 0.8]) * 2.0 * sun[1] / np.pi
    for flags, scale in ((abi.XB_FLAG_SUN_NEE, 1.0), (0, 1e-8)):
        r = Renderer(32, 24, 1, 3, flags=flags)
        r.upload_scene(hs)
        r.render_frame(camera(d.eye, d.target, d.fov, 32 / 24), 4)
        img = r.resolve()
        r.close()
        assert np.allclose(img.reshape(-1, 3), want * scale, rtol=1e-4, atol=0), (img.reshape(-1, 3)[:3], want * scale)


@pytest.mark.gpu
def test_converged_cornell_matches_cpu_render(ref):
    desc = scenes.cornell(max_bounces=8)
    w = h = 64
    spp = 512
    want = ref_render(ref, desc, 1, spp, w, h)
    r = gpu_render(desc, 1, spp, w, h, fp64=True)
    got = r.resolve()
    s64, m2 = r.resolve_fp64()
    print("relmse", relmse(got, want), "max fp32/fp64 diff", np.abs(s64 / spp - got).max())
    assert relmse(got, want) < 1e-3, relmse(got, want)
    assert np.allclose(s64 / spp, got, rtol=1e-3, atol=1e-4)


@pytest.mark.gpu
def test_resolve_async_matches_resolve():
    desc = scenes.cornell()
    r = Renderer(48, 40, desc.max_bounces, desc.min_bounces)
    r.upload_scene(HostScene.from_desc(desc))
    cam = camera(desc.eye, desc.target, desc.fov, 48 / 40)
    outs = []
    for k in range(3):
        r.render_frame(cam, 1)
        o = np.zeros((40, 48, 3), np.float32)
        r.resolve_async(o)
        outs.append(o)
    r.sync()
    assert np.array_equal(outs[-1], r.resolve())
    assert not np.array_equal(outs[0], outs[-1])
    r.close()


@pytest.mark.gpu
def test_fp64_sums_on_the_device_equal_the_host_copy():
    """xb_resolve_fp64_device (the multi-GPU exchange's input) gives the bytes xb_resolve_fp64
    gives, and the per-rank moments of the device path equal those of the host path."""
    import torch

    from xenon_b200 import distributed
    desc = scenes.cornell()
    r = gpu_render(desc, 1, 5, 40, 24, fp64=True)
    s, m2 = r.resolve_fp64()
    ds = torch.empty((24, 40, 3), dtype=torch.float64, device="cuda")
    dm = torch.empty_like(ds)
    r.resolve_fp64_device(ds.data_ptr(), dm.data_ptr())
    assert ds.cpu().numpy().tobytes() == s.tobytes()
    assert dm.cpu().numpy().tobytes() == m2.tobytes()
    dev = distributed._local_moments(r, 5, "cuda").cpu().numpy()
    host = distributed._local_moments(_HostOnly(r), 5, "cpu").numpy()
    assert np.isfinite(dev).all() and np.isfinite(host).all()
    assert np.allclose(dev, host, rtol=1e-12, atol=0.0), float(np.abs(dev - host).max())


class _HostOnly:
    """A renderer seen without its device resolve (the host path of the exchange)."""

    def __init__(self, r):
        self.r, self.fp64, self.width, self.height = r, True, r.width, r.height

    def resolve_fp64(self):
        return self.r.resolve_fp64()
