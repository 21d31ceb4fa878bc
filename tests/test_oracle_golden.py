"""The oracle (oracle/oracle.cpp, the CPU restatement) pinned against the golden vectors the
reference itself produced (tests/golden/gen_golden.py): traversal, BSDF and renders must be
bit-identical, since both are scalar CPU code with the same float operations and libm."""
import os

import numpy as np
import pytest

from xenon_b200 import HostScene, abi
from tests.golden.gen_golden import BSDF_MATERIALS, TRACE_SCENES
from tests.test_host_scene import golden_view_scene

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def port():
    from oracle import port as p
    p.lib()
    return p


@pytest.fixture(scope="module")
def trace_gold():
    return np.load(os.path.join(GOLD, "trace_bvh.npz"))


@pytest.mark.parametrize("name", list(TRACE_SCENES))
def test_trace_bit_exact(name, port, trace_gold):
    desc = TRACE_SCENES[name]()
    ps = port.PortScene(HostScene.from_desc(desc).view())
    rays = trace_gold[f"trace_{name}_rays"]
    got, _ = ps.trace(rays, 0)
    want = trace_gold[f"trace_{name}_closest"]
    assert got.tobytes() == want.tobytes()
    got_any, _ = ps.trace(rays, 1)
    assert np.array_equal(np.isfinite(got_any["t"]), trace_gold[f"trace_{name}_any"])


def test_trace_on_reference_built_arrays(port, trace_gold):
    """The oracle also runs on the reference's own node arrays (as committed), not only on this
    repo's build of them."""
    view, keep = golden_view_scene("instanced", trace_gold)
    ps = port.PortScene(view)
    rays = trace_gold["trace_instanced_rays"]
    got, _ = ps.trace(rays, 0)
    assert got.tobytes() == trace_gold["trace_instanced_closest"].tobytes()


@pytest.fixture(scope="module")
def bsdf_gold():
    return np.load(os.path.join(GOLD, "bsdf.npz"))


@pytest.mark.parametrize("name", list(BSDF_MATERIALS))
def test_bsdf_bit_exact(name, port, bsdf_gold):
    g = bsdf_gold
    m = g[f"{name}_material"]
    f, p = port.bsdf_eval(m, g["wo"], g["wi"])
    assert f.tobytes() == g[f"{name}_f"].tobytes() and p.tobytes() == g[f"{name}_pdf"].tobytes()
    wi, sf, sp, fl, st = port.bsdf_sample(m, g["wo"], g["states"])
    assert np.array_equal(st, g[f"{name}_s_states"]) and np.array_equal(fl, g[f"{name}_s_flags"])
    assert wi.tobytes() == g[f"{name}_s_wi"].tobytes()
    assert sf.tobytes() == g[f"{name}_s_f"].tobytes() and sp.tobytes() == g[f"{name}_s_pdf"].tobytes()
    d = port.material_prepare(m)
    want = g[f"{name}_derived"]
    assert np.array_equal(np.array([d.alpha, d.alpha_x, d.alpha_y, *d.f0, float(d.flags)], np.float32), want)


def test_pcg_seeding(port, bsdf_gold):
    seeds = (0, 1, 2, 12345, 2**40 + 7)
    assert [port.seed_pcg(s) for s in seeds] == [int(x) for x in bsdf_gold["seed_pcg"]]


@pytest.mark.parametrize("name", ["cornell", "icosphere", "prims", "instanced"])
def test_render_bit_exact(name, port):
    from xenon_b200 import camera, scenes
    g = np.load(os.path.join(GOLD, "render.npz"))
    builders = {"cornell": scenes.cornell, "icosphere": lambda: scenes.icosphere_scene(level=4),
                "prims": scenes.prim_showcase,
                "instanced": lambda: scenes.instanced_grid(grid=3, levels=(3, 3, 3, 3), with_prims=True)}
    desc = builders[name]()
    want = g[f"{name}_sum"]
    h, w = want.shape[:2]
    spp = int(g[f"{name}_spp"])
    ps = port.PortScene(HostScene.from_desc(desc).view())
    s, rays = ps.render(camera(desc.eye, desc.target, desc.fov, w / h), w, h, desc.min_bounces,
                        desc.max_bounces, 1, spp)
    assert np.array_equal(s, want)
    assert rays[0] >= w * h * spp
