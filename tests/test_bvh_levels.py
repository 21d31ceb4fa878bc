"""The level-synchronous BVH build (XB_BUILD_LEVELS, csrc/bvh_levels.cpp) on CPU. The form is
data-parallel: every node of a depth is split in one pass, bounds come from chunked ordered
folds, the partition from prefix-sum ranks, and node indices from subtree sizes. It must give
the recursive build's node and order arrays bit for bit, and so the reference's. Tie-breaks
between +0 and -0 included."""
import numpy as np
import pytest

from xenon_b200 import HostScene, abi, scenes

SCENES = {
    "cornell": scenes.cornell,
    "prims": scenes.prim_showcase,
    "icosphere_l7": lambda: scenes.icosphere_scene(level=7),
    "room_l7": lambda: scenes.guiding_room(level=7),
    "instanced": lambda: scenes.instanced_grid(grid=5, levels=(5, 5, 4, 4), with_prims=True),
}


def _arrays(scene):
    a = abi.view_arrays(scene.view())
    out = {"tlas": a["tlas_nodes"].tobytes(), "tlas_inst": a["tlas_inst"].tobytes(),
           "prim_nodes": a["prim_nodes"].tobytes(), "prim_indices": a["prim_indices"].tobytes()}
    for i, m in enumerate(a["meshes"]):
        out[f"mesh{i}_nodes"] = m["nodes"].tobytes()
        out[f"mesh{i}_prims"] = m["prims"].tobytes()
    return out


@pytest.mark.parametrize("name", list(SCENES))
def test_level_build_equals_recursive_build(name):
    desc = SCENES[name]()
    rec = _arrays(HostScene.from_desc(desc, build_threads=1))
    lev = _arrays(HostScene.from_desc(desc, build_threads=1, build_mode=abi.XB_BUILD_LEVELS))
    assert rec.keys() == lev.keys()
    for k in rec:
        assert lev[k] == rec[k], k


def _signed_zero_mesh():
    """Triangles whose coordinate extremes are reached by both +0 and -0, in both orders, so a
    fold that kept the wrong one of two equal values would change a node's bytes."""
    rng = np.random.default_rng(4)
    tris = []
    for k in range(400):
        p = rng.uniform(-1, 1, size=(3, 3)).astype(np.float32)
        a = k % 3
        p[:, a] = np.abs(p[:, a])                    # the minimum along axis a is a zero
        p[k % 2, a] = np.float32(0.0)
        p[(k + 1) % 2, a] = np.float32(-0.0)
        tris.append(p)
    pos = np.concatenate(tris)
    idx = np.arange(len(pos), dtype=np.int32).reshape(-1, 3)
    d = scenes.SceneDesc(name="signed_zeros")
    d.add_material("m", abi.material())
    d.add_mesh(scenes.MeshDesc(pos, idx, None, None, 0))
    return d


def test_signed_zero_ties(ref):
    d = _signed_zero_mesh()
    p = d.meshes[0].positions
    assert (np.signbit(p) & (p == 0)).sum() == 400 and (~np.signbit(p) & (p == 0)).sum() >= 400
    rec = _arrays(HostScene.from_desc(d, build_threads=1))
    lev = _arrays(HostScene.from_desc(d, build_threads=1, build_mode=abi.XB_BUILD_LEVELS))
    theirs = abi.view_arrays(ref.RefScene(d).view())
    assert lev == rec
    assert lev["mesh0_nodes"] == theirs["meshes"][0]["nodes"].tobytes()
    assert lev["mesh0_prims"] == theirs["meshes"][0]["prims"].tobytes()


def test_level_build_equals_the_reference_on_a_large_mesh(ref):
    """The 327,680-triangle sphere of the config-4 room: every node as the reference builds it."""
    desc = scenes.guiding_room(level=7)
    mine = abi.view_arrays(HostScene.from_desc(desc, build_mode=abi.XB_BUILD_LEVELS).view())
    theirs = abi.view_arrays(ref.RefScene(desc).view())
    for a, b in zip(mine["meshes"], theirs["meshes"]):
        assert a["nodes"].tobytes() == b["nodes"].tobytes()
        assert a["prims"].tobytes() == b["prims"].tobytes()
    assert mine["tlas_nodes"].tobytes() == theirs["tlas_nodes"].tobytes()


def test_bad_build_mode():
    import xenon_b200 as xb
    s = HostScene()
    assert xb.lib().xb_scene_set_build_mode(s.h, 7) == abi.XB_E_INVALID


def test_device_build_fails_loudly_without_a_device():
    """XB_BUILD_DEVICE has no host fallback: with no usable CUDA device the build is an error."""
    import torch
    import xenon_b200 as xb
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(xb.XenonError) as e:
        HostScene.from_desc(scenes.cornell(), build_mode=abi.XB_BUILD_DEVICE)
    assert e.value.code == abi.XB_E_CUDA and "device BVH build" in str(e.value)
