"""Parity (a): hit primitive / instance ids bit-exact against the reference CPU traversal for
identical seeded ray batches; t and barycentrics within 4 ulp (Scene::intersect /
Scene::intersects, src/scene/scene.h:124-129)."""
import numpy as np
import pytest

from tests.helpers import compare_hits, mixed_rays, prim_instance_ids
from xenon_b200 import HostScene, Renderer, abi, scenes

SCENES = {
    "cornell": lambda: scenes.cornell(),
    "prims": lambda: scenes.prim_showcase(),
    "instanced": lambda: scenes.instanced_grid(grid=4, levels=(3, 3, 4, 4), with_prims=True),
    "icosphere": lambda: scenes.icosphere_scene(level=6),
    "room": lambda: scenes.guiding_room(level=5),
}


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(SCENES))
def test_closest_and_any_hit_match_reference(name, ref):
    desc = SCENES[name]()
    rays = mixed_rays(desc, 1 << 15, seed=11)
    want = ref.RefScene(desc).trace(rays, abi.XB_TRACE_CLOSEST)
    want_any = ref.RefScene(desc).trace(rays, abi.XB_TRACE_ANY)
    r = Renderer(64, 64)
    r.upload_scene(HostScene.from_desc(desc))
    got = r.trace_rays(rays, abi.XB_TRACE_CLOSEST)
    got_any = r.trace_rays(rays, abi.XB_TRACE_ANY)
    d = compare_hits(got, want, prim_ids=prim_instance_ids(desc))
    print(name, d)
    assert d["hits"] > len(rays) // 10, d
    assert d["hit_mismatch"] == 0, d
    assert d["prim_id_mismatch"] == 0 and d["instance_id_mismatch"] == 0 and d["mat_id_mismatch"] == 0, d
    assert d["t_ulp_max"] <= 4 and d["u_ulp_max"] <= 4 and d["v_ulp_max"] <= 4, d
    assert d["u_prim_maxabs"] < 1e-5 and d["v_prim_maxabs"] < 1e-5, d
    assert d["front_mismatch"] == 0, d
    assert d["normal_maxabs"] < 1e-5 and d["geo_normal_maxabs"] < 1e-5, d
    assert np.array_equal(np.isfinite(got_any["t"]), np.isfinite(want_any["t"]))


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(SCENES))
def test_query_forms_return_the_same_records(name):
    """xb_trace_rays runs its queries on persistent warps (the default tuning) or one ray per
    thread (XB_FLAG_THREAD_PER_RAY, or a tuning without persistent bounce/shadow rays): the hit
    records are equal byte for byte."""
    desc = SCENES[name]()
    rays = mixed_rays(desc, 1 << 15, seed=12)
    hs = HostScene.from_desc(desc)
    out = []
    for flags, tune in ((0, {}), (abi.XB_FLAG_THREAD_PER_RAY, {}),
                        (0, {"extend_persistent_from_depth": 64, "shadow_persistent": 2}),
                        (0, {"refill": 1}), (0, {"refill": 32})):
        r = Renderer(64, 64, flags=flags)
        r.upload_scene(hs)
        if tune:
            r.set_tuning(**tune)
        out.append((r.trace_rays(rays, abi.XB_TRACE_CLOSEST).tobytes(), r.trace_rays(rays, abi.XB_TRACE_ANY).tobytes()))
        r.close()
    for o in out[1:]:
        assert o == out[0]


@pytest.mark.gpu
def test_reference_built_view_uploads_as_is(ref):
    """The drop-in path: the reference's own BLAS/TLAS arrays go through xb_upload_scene."""
    desc = scenes.instanced_grid(grid=3, levels=(3, 3, 3, 3), with_prims=True)
    rs = ref.RefScene(desc)
    rays = mixed_rays(desc, 1 << 14, seed=5)
    want = rs.trace(rays)
    r = Renderer(32, 32)
    r.upload_scene(rs.view())
    got = r.trace_rays(rays)
    d = compare_hits(got, want, prim_ids=prim_instance_ids(desc))
    assert d["prim_id_mismatch"] == 0 and d["instance_id_mismatch"] == 0 and d["hit_mismatch"] == 0, d
    assert d["t_ulp_max"] <= 4, d


@pytest.mark.gpu
def test_empty_and_degenerate_batches(ref):
    """Edge cases the reference handles in its own way: zero direction components (infinite
    reciprocals, NaN slabs), tmin > tmax (closest hit ignores tmax, tlas.cpp:172-245; any hit
    honours it), rays outside the scene, rays along a wall."""
    desc = scenes.cornell()
    r = Renderer(16, 16)
    r.upload_scene(HostScene.from_desc(desc))
    assert len(r.trace_rays(np.zeros(0, abi.RAY_DTYPE))) == 0
    org = np.array([[0, 5, 0], [0, 5, 0], [0, 5, 0], [100, 100, 100], [-5, 5, 0], [0, 0, 0]], np.float32)
    dirs = np.array([[0, 0, -1], [1, 0, 0], [0, -1, 0], [0, 0, 1], [0, 1, 0], [0, 0, -1]], np.float32)
    rays = abi.make_rays(org, dirs)
    rays["tmin"][2], rays["tmax"][2] = 5.0, 1.0
    rs = ref.RefScene(desc)
    for mode in (abi.XB_TRACE_CLOSEST, abi.XB_TRACE_ANY):
        h = r.trace_rays(rays, mode)
        w = rs.trace(rays, mode)
        assert np.array_equal(np.isfinite(h["t"]), np.isfinite(w["t"])), (mode, h["t"], w["t"])
        assert np.array_equal(h["prim_id"], w["prim_id"]) and np.array_equal(h["instance_id"], w["instance_id"])


@pytest.mark.gpu
def test_stack_overflow_is_reported():
    """A BLAS deeper than the 64-entry traversal stack: xb_trace_rays reports XB_E_OVERFLOW
    (the hit may be lost) instead of writing past the stack."""
    import xenon_b200 as xb
    from tests.helpers import deep_chain_scene
    hs, view, rays = deep_chain_scene(depth=100)
    r = Renderer(16, 16)
    r.upload_scene(view)
    with pytest.raises(xb.XenonError) as e:
        r.trace_rays(rays, abi.XB_TRACE_CLOSEST)
    assert e.value.code == abi.XB_E_OVERFLOW
    # a chain the stack holds traces without overflow
    hs2, view2, rays2 = deep_chain_scene(depth=40)
    r2 = Renderer(16, 16)
    r2.upload_scene(view2)
    h = r2.trace_rays(rays2, abi.XB_TRACE_CLOSEST)
    assert np.isfinite(h["t"]).any()
