"""Sky importance sampling (XB_FLAG_SKY_IS) against the default estimator, which weights the
sky by 1 on every escaping path (src/render/cpu_tiled.cpp:40-54): the sky proposal changes the
random draws and the per-pixel noise, but not the converged image."""
import numpy as np
import pytest

import xenon_b200 as xb
from xenon_b200 import abi, scenes

W, H = 96, 54


def _render(desc, spp, flags):
    r = xb.Renderer(W, H, desc.max_bounces, desc.min_bounces, fp64=True, flags=flags)
    r.upload_scene(xb.HostScene.from_desc(desc))
    r.render_frame(xb.camera(desc.eye, desc.target, desc.fov, W / H), spp)
    s, m2 = r.resolve_fp64()
    st = r.stats()
    r.close()
    return s / spp, m2 / (spp - 1), st


@pytest.mark.gpu
@pytest.mark.parametrize("name,heavy", [("icosphere", False), ("instanced", True)])
def test_sky_importance_sampling_converges_to_the_default_image(name, heavy):
    desc = {"icosphere": lambda: scenes.icosphere_scene(level=5, width=W, height=H),
            "instanced": lambda: scenes.instanced_grid(grid=4, levels=(3, 3, 4, 4), width=W, height=H)}[name]()
    spp = 2048
    mp, vp, stp = _render(desc, spp, 0)
    ms, vs, sts = _render(desc, spp, abi.XB_FLAG_SKY_IS)
    assert stp.overflow == 0 and sts.overflow == 0
    # non-finite samples (dropped and counted; the reference's estimator makes a few per million
    # paths on this scene, the plain render too) stay as rare as in the default render
    assert sts.nonfinite <= 2 * stp.nonfinite + 10, (sts.nonfinite, stp.nonfinite)
    assert not np.array_equal(ms, mp)                    # the proposal is in use
    # the image means agree within the guided tests' gate (6 estimated standard errors)
    d = ms.sum() - mp.sum()
    se = np.sqrt(vs.sum() / spp + vp.sum() / spp)
    assert abs(d) < 6 * se, (ms.mean(), mp.mean(), d / se)
    # per pixel the differences are centred; their scale is not checked (the two estimators'
    # per-pixel variance estimates differ several-fold, and heavy tails make them unreliable)
    z = (ms.mean(2) - mp.mean(2)) / (np.sqrt(vs.mean(2) / spp + vp.mean(2) / spp) + 1e-12)
    assert abs(np.median(z)) < 0.1, np.median(z)
    assert np.mean(np.abs(z) > 4) < (0.02 if heavy else 0.002), np.mean(np.abs(z) > 4)
    print(name, "median per-pixel variance sky/default:",
          float(np.median(vs.mean(2)) / max(np.median(vp.mean(2)), 1e-30)))


@pytest.mark.gpu
def test_sky_importance_sampling_needs_a_sky():
    """A black sky has no distribution: the flag then leaves the default estimator in place."""
    desc = scenes.cornell()
    a, _, _ = _render(desc, 4, 0)
    b, _, _ = _render(desc, 4, abi.XB_FLAG_SKY_IS)
    assert np.array_equal(a, b)
