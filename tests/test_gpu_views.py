"""xb_render_views: many cameras packed into shared waves give, view by view, exactly the image
a renderer of that view's size renders on its own (same seeds, same sample order)."""
import numpy as np
import pytest

import xenon_b200 as xb
from xenon_b200 import scenes


def _single(sc, cam, w, h, spp, bounces):
    r = xb.Renderer(w, h, max_bounces=bounces, min_bounces=3)
    r.upload_scene(sc)
    r.render_frame(cam, spp)
    img = r.resolve().copy()
    r.close()
    return img


@pytest.mark.gpu
@pytest.mark.parametrize("scene", ["cornell", "prims"])
def test_views_equal_single_view_renders(scene):
    desc = scenes.cornell() if scene == "cornell" else scenes.prim_showcase()
    sc = xb.HostScene.from_desc(desc)
    specs = [((0.0, 5.0, 18.7), (0.0, 5.0, 0.0), 40.0, 40, 30, 3),
             ((3.0, 6.0, 15.0), (0.0, 4.0, 0.0), 50.0, 64, 48, 2),
             ((-4.0, 3.0, 16.0), (0.5, 5.0, -1.0), 35.0, 33, 17, 5),
             ((0.0, 9.0, 12.0), (0.0, 2.0, 0.0), 60.0, 17, 33, 1)]
    if scene == "prims":
        specs = [(tuple(np.add(desc.eye, (dx, 0.5 * dx, 0))), desc.target, desc.fov, w, h, spp)
                 for (dx, (_, _, _, w, h, spp)) in zip((0.0, 1.0, -1.5, 2.0), specs)]
    cams = [xb.camera(e, t, f, w / h) for (e, t, f, w, h, _) in specs]
    r = xb.Renderer(64, 64, max_bounces=desc.max_bounces, min_bounces=3)
    r.upload_scene(sc)
    imgs = r.render_views([(c, w, h, spp) for c, (_, _, _, w, h, spp) in zip(cams, specs)])
    st = r.stats()
    assert st.paths == sum(w * h * spp for (_, _, _, w, h, spp) in specs)
    assert r.spp == 0                     # the renderer's own image is untouched
    r.close()
    for img, cam, (_, _, _, w, h, spp) in zip(imgs, cams, specs):
        want = _single(sc, cam, w, h, spp, desc.max_bounces)
        assert img.shape == (h, w, 3)
        assert np.array_equal(img, want)


@pytest.mark.gpu
def test_views_larger_than_the_wave_and_many_pieces():
    desc = scenes.cornell()
    sc = xb.HostScene.from_desc(desc)
    cam = xb.camera(desc.eye, desc.target, desc.fov, 1.0)
    # a tiny wave forces every view to span several waves
    r = xb.Renderer(32, 32, max_bounces=4, min_bounces=3, wave_paths=3000)
    r.upload_scene(sc)
    views = [(cam, 70, 70, 2), (cam, 16, 16, 40), (cam, 8, 8, 3)] + [(cam, 4, 4, 1)] * 70
    imgs = r.render_views(views)
    r.close()
    for img, (c, w, h, spp) in zip(imgs[:4], views[:4]):
        assert np.array_equal(img, _single(sc, c, w, h, spp, 4))
    assert all(np.array_equal(imgs[3], i) for i in imgs[4:])


@pytest.mark.gpu
def test_views_reject_bad_input():
    desc = scenes.cornell()
    r = xb.Renderer(16, 16)
    cam = xb.camera(desc.eye, desc.target, desc.fov, 1.0)
    with pytest.raises(xb.XenonError):
        r.render_views([(cam, 8, 8, 1)])          # no scene uploaded
    r.upload_scene(xb.HostScene.from_desc(desc))
    with pytest.raises(xb.XenonError):
        r.render_views([(cam, 0, 8, 1)])
    r.close()


@pytest.mark.gpu
def test_views_with_their_own_bounce_limits():
    desc = scenes.cornell()
    sc = xb.HostScene.from_desc(desc)
    cam = xb.camera(desc.eye, desc.target, desc.fov, 1.0)
    r = xb.Renderer(32, 32, max_bounces=8, min_bounces=3)
    r.upload_scene(sc)
    views = [(cam, 40, 40, 3, 2), (cam, 24, 24, 5, 5), (cam, 16, 16, 2, 0), (cam, 33, 21, 2, 12)]
    imgs = r.render_views(views)
    r.close()
    for img, (c, w, h, spp, mb) in zip(imgs, views):
        want = _single(sc, c, w, h, spp, mb or 8)
        assert np.array_equal(img, want), (w, h, mb)


@pytest.mark.gpu
def test_guided_views_converge_to_plain_views():
    """One network, trained on the renderer's own view, serves every view of the batch; the
    guided views estimate the same images as plain ones."""
    desc = scenes.cornell()
    sc = xb.HostScene.from_desc(desc)
    cam = xb.camera(desc.eye, desc.target, desc.fov, 1.0)
    cam2 = xb.camera((2.0, 6.0, 16.0), (0.0, 4.0, 0.0), 45.0, 1.0)
    views = [(cam, 48, 48, 1024, 8), (cam2, 40, 40, 1024, 6)]
    plain = xb.Renderer(48, 48, max_bounces=8, min_bounces=3)
    plain.upload_scene(sc)
    pimgs = plain.render_views(views)
    plain.close()
    g = xb.Renderer(48, 48, max_bounces=8, min_bounces=3)
    g.upload_scene(sc)
    g.set_guiding(True, train_spp=32, steps_per_spp=16, batch=4096)
    g.render_frame(cam, 32)                            # trains the shared network
    assert g.guiding_stats()["adam_steps"] == 32 * 16
    gimgs = g.render_views(views)
    g.close()
    for gi, pi in zip(gimgs, pimgs):
        assert np.all(np.isfinite(gi))
        assert abs(gi.mean() / pi.mean() - 1.0) < 0.02, (gi.mean(), pi.mean())
