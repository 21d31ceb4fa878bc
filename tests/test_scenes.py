"""The seeded workloads stand in for the configs' scenes: their shapes, sizes and the config-5 view
list are checked here on the CPU (numpy only; the renders are the GPU tests' business)."""
import numpy as np

from xenon_b200 import abi, scenes


def _tris(desc):
    return sum(len(m.indices) // 3 if np.ndim(m.indices) == 1 else len(m.indices) for m in desc.meshes)


def test_config2_scene_shape():
    d = scenes.icosphere_scene(level=8)
    assert (d.width, d.height, d.max_bounces) == (1920, 1080, 10)
    assert _tris(d) == 1_310_722                # 20 * 4^8 sphere triangles + the 2 of the ground
    assert len(d.suns) == 1


def test_config4_room_shape():
    d = scenes.guiding_room()
    assert (d.width, d.height, d.max_bounces) == (1280, 720, 16)
    # the only light: two triangles covering 0.5 % of the 10 x 10 ceiling
    area = sum(l[3] for l in d.lights)
    assert len(d.lights) == 2 and abs(area / (10.0 * 10.0) - 0.005) < 1e-9
    assert _tris(d) - 18 == 499_280              # the geodesic sphere (20 * 158^2) + 9 quads: walls, baffle, light
    assert _tris(scenes.guiding_room(level=7)) - 18 == 327_680   # the level-7 icosphere form (20 * 4^7)
    glass = [m for m in d.materials if m[abi.MATERIAL_FIELDS["transmission"]] == 1.0]
    assert len(glass) == 1 and glass[0][abi.MATERIAL_FIELDS["ior"]] == np.float32(1.5)
    assert d.sky[10] == 0.0                      # closed room: the sky's intensity is zero


def test_config5_views_are_seeded_and_in_range():
    d = scenes.instanced_grid(grid=2, levels=(2, 2, 2, 2))
    a = scenes.config5_views(d, 32, seed=1)
    b = scenes.config5_views(d, 32, seed=1)
    assert a == b and len(a) == 32
    assert scenes.config5_views(d, 32, seed=2) != a
    lo, hi = scenes.scene_bounds(d)
    for eye, target, fov, w, h, spp, mb in a:
        assert w == h and 256 <= w <= 1024
        assert spp in scenes.VIEW_SPP
        assert 6 <= mb <= 16
        assert np.allclose(target, (np.asarray(lo) + np.asarray(hi)) / 2)
        assert eye[1] > target[1]                  # from the upper hemisphere
    # sizes spread over the log-uniform range, and the spp cap applies to every view
    sides = np.array([v[3] for v in a])
    assert sides.min() < 400 and sides.max() > 700
    capped = scenes.config5_views(d, 32, seed=1, max_spp=64)
    assert [v[:5] + v[6:] for v in capped] == [v[:5] + v[6:] for v in a]
    assert all(v[5] == min(o[5], 64) for v, o in zip(capped, a))
