"""Device BLAS refit (xb_refit_mesh) against the host refit (xb_scene_refit_mesh) + upload, on a
B200: rays traced through both scenes give bit-identical hits; an unchanged refit changes no hit;
meshes with area lights are refused."""
import numpy as np
import pytest

import xenon_b200 as xb
from xenon_b200 import HostScene, abi, scenes

pytestmark = pytest.mark.gpu


def _moved(pos, seed):
    rng = np.random.default_rng(seed)
    w = rng.normal(size=(3, 3)) * 0.3
    return (pos + np.sin(pos @ w) * 0.4 + rng.normal(size=3)).astype(np.float32)


def _renderer(scene):
    r = xb.Renderer(64, 64)
    r.upload_scene(scene)
    return r


@pytest.mark.parametrize("make", [lambda: scenes.icosphere_scene(level=5),
                                  lambda: scenes.instanced_grid(grid=3, levels=(4, 4, 3, 3), with_prims=True)])
def test_device_refit_equals_host_refit(make):
    desc = make()
    rays = scenes.random_rays(scenes.scene_bounds(desc), 1 << 16, seed=7)
    host = HostScene.from_desc(desc)
    dev = _renderer(host)
    before = dev.trace_rays(rays)
    lit = {l[0] for l in desc.lights}
    targets = [m for m in range(len(desc.meshes)) if m not in lit][:3]
    for m in targets:                        # unchanged vertices: no hit changes
        dev.refit_mesh(m, abi.view_arrays(host.view())["meshes"][m]["pos"])
    assert dev.trace_rays(rays).tobytes() == before.tobytes()
    for m in targets:
        pos = abi.view_arrays(host.view())["meshes"][m]["pos"]
        new = _moved(pos, m)
        dev.refit_mesh(m, new)
        host.refit_mesh(m, new)
    ref = _renderer(host).trace_rays(rays)
    got = dev.trace_rays(rays)
    assert (ref["prim_id"] >= 0).mean() > 0.2
    assert got.tobytes() == ref.tobytes()


def test_device_refit_refuses_light_meshes_and_bad_input():
    desc = scenes.cornell()
    host = HostScene.from_desc(desc)
    r = _renderer(host)
    light_mesh = desc.lights[0][0]
    pos = abi.view_arrays(host.view())["meshes"][light_mesh]["pos"]
    with pytest.raises(xb.XenonError) as e:
        r.refit_mesh(light_mesh, pos)
    assert e.value.code == abi.XB_E_UNSUPPORTED
    with pytest.raises(xb.XenonError):
        r.refit_mesh(99, pos)
