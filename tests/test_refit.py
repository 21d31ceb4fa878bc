"""BLAS refit on the host (xb_scene_refit_mesh, bvh_refit.h), CPU only.

With unchanged vertices, the refit gives the build's node arrays bit for bit. With moved vertices, every
leaf box is its triangles' bounds and every interior box is the union of its children's boxes.
The TLAS equals a fresh build's: it depends only on the instances' root boxes, which are the
bounds of all their triangles whatever the tree. Rays traced through the refitted tree by the
oracle's traversal find what they find in a tree built for the moved mesh."""
import numpy as np
import pytest

import xenon_b200 as xb
from xenon_b200 import HostScene, abi, scenes

SCENES = {
    "cornell": scenes.cornell,
    "icosphere": lambda: scenes.icosphere_scene(level=5),
    "room": lambda: scenes.guiding_room(level=4),
    "instanced": lambda: scenes.instanced_grid(grid=3, levels=(4, 4, 3, 3), with_prims=True),
}


def _boxes(nodes):
    return np.concatenate([nodes["mn"], nodes["mx"]], 1) if len(nodes) else np.zeros((0, 6), np.float32)


def _mesh_vertices(scene, mesh):
    a = abi.view_arrays(scene.view())["meshes"][mesh]
    return a["pos"].copy(), a["nrm"]


@pytest.mark.parametrize("name", list(SCENES))
def test_refit_of_unchanged_vertices_gives_the_build(name):
    desc = SCENES[name]()
    built = abi.view_arrays(HostScene.from_desc(desc).view())
    s = HostScene.from_desc(desc)
    for m in range(len(desc.meshes)):
        pos, _ = _mesh_vertices(s, m)
        s.refit_mesh(m, pos)
    refit = abi.view_arrays(s.view())
    # bit for bit: these scenes have no box coordinate reached by both +0 and -0 (bvh_refit.h)
    for a, b in zip(refit["meshes"], built["meshes"]):
        assert a["nodes"].tobytes() == b["nodes"].tobytes()
        assert a["prims"].tobytes() == b["prims"].tobytes()
    assert refit["tlas_nodes"].tobytes() == built["tlas_nodes"].tobytes()
    assert refit["tlas_inst"].tobytes() == built["tlas_inst"].tobytes()


def _moved(pos, seed):
    """A smooth deformation plus a shift: the tree's topology no longer fits it well."""
    rng = np.random.default_rng(seed)
    w = rng.normal(size=(3, 3)) * 0.3
    return (pos + np.sin(pos @ w) * 0.4 + rng.normal(size=3)).astype(np.float32)


def test_refit_of_moved_vertices_bounds_every_subtree():
    desc = scenes.icosphere_scene(level=5)
    s = HostScene.from_desc(desc)
    pos, _ = _mesh_vertices(s, 0)
    new = _moved(pos, 1)
    s.refit_mesh(0, new)
    a = abi.view_arrays(s.view())["meshes"][0]
    nodes, prims, idx = a["nodes"], a["prims"], a["indices"]
    assert np.array_equal(a["pos"], new)
    tri = new[idx[prims]]                                   # (slots, 3 vertices, xyz)
    tmin, tmax = tri.min(1), tri.max(1)
    box = _boxes(nodes)
    for i, n in enumerate(nodes):
        if n["count"] > 0:
            sl = slice(n["child"], n["child"] + n["count"])
            assert np.array_equal(box[i, :3], tmin[sl].min(0)) and np.array_equal(box[i, 3:], tmax[sl].max(0)), i
        else:
            l, r = box[n["child"]], box[n["child"] + 1]
            assert np.array_equal(box[i, :3], np.minimum(l[:3], r[:3])), i
            assert np.array_equal(box[i, 3:], np.maximum(l[3:], r[3:])), i


def test_refit_tlas_and_hits_match_a_fresh_build():
    from oracle import port
    port.lib()
    desc = scenes.instanced_grid(grid=3, levels=(4, 4, 3, 3), with_prims=True)
    s = HostScene.from_desc(desc)
    moved = {}
    for m in (0, 4, 9):                                      # instanced meshes of several variants
        pos, _ = _mesh_vertices(s, m)
        moved[m] = _moved(pos, m)
        s.refit_mesh(m, moved[m])
    # the same scene built from scratch with the moved vertices (vertex order is the loader's)
    fresh_desc = scenes.instanced_grid(grid=3, levels=(4, 4, 3, 3), with_prims=True)
    for m, p in moved.items():
        old = fresh_desc.meshes[m]
        fresh_desc.meshes[m] = scenes.MeshDesc(p, old.indices, None, old.mat_ids, old.default_mat, None)
    fresh = HostScene.from_desc(fresh_desc)
    a, b = abi.view_arrays(s.view()), abi.view_arrays(fresh.view())
    assert np.array_equal(_boxes(a["tlas_nodes"]), _boxes(b["tlas_nodes"]))
    assert a["tlas_inst"].tobytes() == b["tlas_inst"].tobytes()
    for m in moved:
        assert np.array_equal(_boxes(a["meshes"][m]["nodes"][:1]), _boxes(b["meshes"][m]["nodes"][:1]))
    rays = scenes.random_rays(scenes.scene_bounds(desc), 20000, seed=5)
    h1, _ = port.PortScene(s.view()).trace(rays)
    h2, _ = port.PortScene(fresh.view()).trace(rays)
    assert (h1["prim_id"] >= 0).mean() > 0.2
    assert np.array_equal(h1["t"], h2["t"])
    same = (h1["prim_id"] == h2["prim_id"]) & (h1["instance_id"] == h2["instance_id"])
    assert same.mean() > 0.999                               # ties at shared edges may differ


def test_refit_errors():
    s = HostScene.from_desc(scenes.cornell())
    pos, _ = _mesh_vertices(s, 0)
    with pytest.raises(xb.XenonError):
        s.refit_mesh(99, pos)
    with pytest.raises(xb.XenonError):
        s.refit_mesh(0, pos[:-1])
    bad = pos.copy()
    bad[0, 0] = np.inf
    with pytest.raises(xb.XenonError) as e:
        s.refit_mesh(0, bad)
    assert e.value.code == abi.XB_E_INVALID


def test_refit_signed_zero_ties_differ_only_in_sign():
    """Where a box coordinate's extreme is reached by both +0 and -0, an interior node's refit
    box can keep the other zero than the build's (bvh_refit.h): equal values, leaves identical."""
    from tests.test_bvh_levels import _signed_zero_mesh
    d = _signed_zero_mesh()
    built = abi.view_arrays(HostScene.from_desc(d).view())["meshes"][0]["nodes"]
    s = HostScene.from_desc(d)
    s.refit_mesh(0, d.meshes[0].positions)
    refit = abi.view_arrays(s.view())["meshes"][0]["nodes"]
    assert np.array_equal(_boxes(refit), _boxes(built))
    leaves = built["count"] > 0
    assert refit[leaves].tobytes() == built[leaves].tobytes()
    assert np.array_equal(refit["child"], built["child"]) and np.array_equal(refit["count"], built["count"])
