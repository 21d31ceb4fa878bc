"""Host side of the library (no GPU needed): the TLAS/BLAS build reproduces the reference's
node arrays bit for bit, the camera, material preparation and loaders match the reference, and
the C ABI reports errors as status codes."""
import ctypes
import os

import numpy as np
import pytest

import xenon_b200 as xb
from xenon_b200 import HostScene, abi, camera, scenes
from tests.golden.gen_golden import BSDF_MATERIALS, TRACE_SCENES

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def gold():
    return np.load(os.path.join(GOLD, "trace_bvh.npz"))


def golden_view_scene(name, gold):
    """An xb_scene_view whose BVH arrays are the reference's committed ones (for `name`)."""
    desc = TRACE_SCENES[name]()
    hs = HostScene.from_desc(desc)
    v = hs.view()
    keep = [hs]
    for i in range(v.num_meshes):
        nodes = np.ascontiguousarray(gold[f"bvh_{name}_mesh{i}_nodes"])
        prims = np.ascontiguousarray(gold[f"bvh_{name}_mesh{i}_prims"])
        keep += [nodes, prims]
        v.meshes[i].blas_nodes = nodes.ctypes.data
        v.meshes[i].blas_prims = prims.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))
    tl = np.ascontiguousarray(gold[f"bvh_{name}_tlas"])
    ti = np.ascontiguousarray(gold[f"bvh_{name}_tlas_inst"])
    keep += [tl, ti]
    v.tlas_nodes = tl.ctypes.data
    v.tlas_inst_indices = ti.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))
    if v.num_prims:
        pn = np.ascontiguousarray(gold[f"bvh_{name}_prim_nodes"])
        pi = np.ascontiguousarray(gold[f"bvh_{name}_prim_indices"])
        keep += [pn, pi]
        v.prim_nodes = pn.ctypes.data
        v.prim_indices = pi.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))
    return v, keep


@pytest.mark.parametrize("name", list(TRACE_SCENES))
def test_bvh_build_matches_reference(name, gold):
    desc = TRACE_SCENES[name]()
    a = abi.view_arrays(HostScene.from_desc(desc).view())
    for i, m in enumerate(a["meshes"]):
        assert m["nodes"].tobytes() == gold[f"bvh_{name}_mesh{i}_nodes"].tobytes(), (name, i)
        assert m["prims"].tobytes() == gold[f"bvh_{name}_mesh{i}_prims"].tobytes(), (name, i)
        key = f"bvh_{name}_mesh{i}_normals"
        if key in gold:
            assert m["nrm"].tobytes() == gold[key].tobytes(), (name, i)
    assert a["tlas_nodes"].tobytes() == gold[f"bvh_{name}_tlas"].tobytes()
    assert a["tlas_inst"].tobytes() == gold[f"bvh_{name}_tlas_inst"].tobytes()
    assert a["prim_nodes"].tobytes() == gold[f"bvh_{name}_prim_nodes"].tobytes()
    assert a["prim_indices"].tobytes() == gold[f"bvh_{name}_prim_indices"].tobytes()


@pytest.mark.parametrize("name", list(TRACE_SCENES))
def test_camera_matches_reference(name, gold):
    desc = TRACE_SCENES[name]()
    c = camera(desc.eye, desc.target, desc.fov, desc.width / desc.height).to_array()
    assert c.tobytes() == gold[f"camera_{name}"].tobytes()


@pytest.mark.parametrize("name", list(BSDF_MATERIALS))
def test_material_prepare_matches_reference(name):
    g = np.load(os.path.join(GOLD, "bsdf.npz"))
    d = xb.material_prepare(g[f"{name}_material"])
    got = np.array([d.alpha, d.alpha_x, d.alpha_y, *d.f0, float(d.flags)], np.float32)
    assert np.array_equal(got, g[f"{name}_derived"])


def test_xenon_loader_matches_reference(monkeypatch):
    g = np.load(os.path.join(GOLD, "loader.npz"))
    monkeypatch.chdir(os.path.join(GOLD, "scenes"))
    hs = HostScene.load("loader_test.xenon")
    assert [hs.config.width, hs.config.height, hs.config.samples] == list(g["config"])
    cd = hs.camera_desc
    cam = camera(list(cd.eye), list(cd.target), cd.fov_y_deg, hs.config.width / hs.config.height).to_array()
    assert cam.tobytes() == g["camera"].tobytes()
    v = hs.view()
    mats = np.frombuffer((ctypes.c_char * (v.num_materials * 84)).from_address(v.materials), np.float32).reshape(-1, 21)
    # the reference keeps only the fields its Material has; compare those (all of xb_material)
    assert np.array_equal(mats, g["materials"])
    prims = np.frombuffer((ctypes.c_char * (v.num_prims * 48)).from_address(v.prims), abi.PRIM_DTYPE)
    assert prims.tobytes() == g["prims"].tobytes()
    suns = np.frombuffer((ctypes.c_char * (v.num_suns * 28)).from_address(v.suns), np.float32).reshape(-1, 7)
    assert np.array_equal(suns, g["suns"])
    sky = np.array(list(v.sky.zenith) + list(v.sky.horizon) + list(v.sky.ground) + [v.sky.sharpness, v.sky.intensity], np.float32)
    assert np.array_equal(sky, g["sky"])
    a = abi.view_arrays(v)
    assert a["prim_nodes"].tobytes() == g["prim_nodes"].tobytes()
    assert a["tlas_nodes"].tobytes() == g["tlas_nodes"].tobytes()


def test_mat_file_loader():
    m = abi.Camera  # noqa: F841 (keeps import order obvious)
    out = np.zeros(21, np.float32)
    name = ctypes.create_string_buffer(64)
    rc = xb.lib().xb_material_load(os.path.join(GOLD, "scenes", "materials", "brass.mat").encode(),
                                   out.ctypes.data_as(ctypes.c_void_p), name, 64)
    assert rc == 0 and name.value == b"brass"
    assert np.allclose(out[0:3], [0.91, 0.78, 0.42]) and out[4] == 1.0 and np.isclose(out[11], 0.4)
    rc = xb.lib().xb_material_load(b"/nonexistent/x.mat", out.ctypes.data_as(ctypes.c_void_p), name, 64)
    assert rc == abi.XB_E_IO


def test_scene_errors_are_status_codes():
    L = xb.lib()
    with pytest.raises(xb.XenonError) as e:
        HostScene.load("/nonexistent/scene.xenon")
    assert e.value.code == abi.XB_E_IO
    s = HostScene()
    pos = np.zeros((3, 3), np.float32)
    idx = np.array([[0, 1, 5]], np.int32)           # index out of range
    rc = L.xb_scene_add_mesh(s.h, 3, pos.ctypes.data_as(ctypes.c_void_p), None, 1,
                             idx.ctypes.data_as(ctypes.c_void_p), None, 0)
    assert rc == abi.XB_E_INVALID and "out of range" in xb.native.last_error()
    # a light on a mesh that does not exist is caught at build time
    e3 = np.ones(3, np.float32)
    L.xb_scene_add_light(s.h, 7, 0, e3.ctypes.data_as(ctypes.c_void_p), 1.0)
    assert L.xb_scene_build(s.h) == abi.XB_E_INVALID
    v = abi.SceneView()
    assert L.xb_scene_get_view(s.h, ctypes.byref(v)) == abi.XB_E_STATE
    assert L.xb_scene_add_instance(s.h, 3, e3.ctypes.data_as(ctypes.c_void_p), 1.0,
                                   e3.ctypes.data_as(ctypes.c_void_p), 0) == abi.XB_E_INVALID


def test_mesh_transform_matches_reference(ref):
    desc = scenes.SceneDesc()
    desc.add_material("m", abi.material())
    mesh = scenes.box_mesh((0.3, 0.2, -0.1), (1.0, 2.0, 0.5), 0.0, 0)
    mesh.transform = ((1.5, -2.0, 0.25), 1.7, (12.0, -33.0, 71.0))
    desc.add_mesh(mesh)
    rs = ref.RefScene(desc)
    pos, nrm = rs.mesh_arrays(0, len(mesh.positions))
    a = abi.view_arrays(HostScene.from_desc(desc).view())
    assert a["meshes"][0]["pos"].tobytes() == pos.tobytes()
    assert a["meshes"][0]["nrm"].tobytes() == nrm.tobytes()


def test_scene_generators_are_deterministic():
    import hashlib

    def digest(d):
        h = hashlib.sha256()
        for m in d.meshes:
            h.update(m.positions.tobytes()); h.update(m.indices.tobytes())
        for t in d.instances:
            h.update(repr(t).encode())
        return h.hexdigest()

    assert digest(scenes.icosphere_scene(level=3)) == digest(scenes.icosphere_scene(level=3))
    assert digest(scenes.instanced_grid(grid=2, levels=(2, 2, 2, 2))) == \
        digest(scenes.instanced_grid(grid=2, levels=(2, 2, 2, 2)))
    v, f = scenes.icosphere(8)
    assert len(f) == 1310720 and len(v) == 655362


def test_xenon_instance_command(tmp_path, monkeypatch):
    """`instance` (this library's addition to the .xenon format): the loaded scene's TLAS and
    instances equal those of the same scene built through xb_scene_add_instance."""
    obj = tmp_path / "tri.obj"
    obj.write_text("v 0 0 0\nv 1 0 0\nv 0 1 0\nv 1 1 0.5\nf 1 2 3\nf 2 4 3\n")
    (tmp_path / "s.xenon").write_text(
        "config 64 48 4\ncamera 0 3 10  0 0 0  45\n"
        "material m 0.7 0.6 0.5 0.0 0.9\n"
        "mesh tri.obj\nmesh tri.obj\n"
        "light 1 0 5 5 5 0.5\n"
        "instance 0  -2 0 0  1.0  0 30 0\n"
        "instance 0   2 0 0  0.5  0 -45 10  77\n"
        "instance 1   0 4 0  1.0  0 0 0\n"
        "sphere 0 1 0 0.5 m\n"
        "instance prims  0 0 1  1.0  0 0 0\n"
        "instance 5  0 0 0  1 0 0 0\n"        # no such mesh: skipped with a warning
        "instance 0  0 0 0  0 0 0 0\n")       # zero scale: skipped
    monkeypatch.chdir(tmp_path)                # mesh paths are relative to the working directory
    loaded = HostScene.load("s.xenon")
    got = abi.view_arrays(loaded.view())

    d = scenes.SceneDesc()
    d.add_material("m", abi.material(base_color=(0.7, 0.6, 0.5), roughness=0.9))
    pos = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [1, 1, 0.5]], np.float32)
    idx = np.array([[0, 1, 2], [1, 3, 2]], np.int32)
    for _ in range(2):
        d.add_mesh(scenes.MeshDesc(pos, idx, None, None, 0))
    d.lights.append((1, 0, (5.0, 5.0, 5.0), 0.5))
    p = np.zeros(1, abi.PRIM_DTYPE)
    p["type"], p["mat_id"], p["p"][0, :4] = abi.XB_PRIM_SPHERE, 0, (0, 1, 0, 0.5)
    d.prims.append(p)
    d.instances += [(0, (-2, 0, 0), 1.0, (0, 30, 0), 0), (0, (2, 0, 0), 0.5, (0, -45, 10), 77),
                    (1, (0, 4, 0), 1.0, (0, 0, 0), 1), (abi.XB_GEOM_PRIMS, (0, 0, 1), 1.0, (0, 0, 0), 2)]
    want = abi.view_arrays(HostScene.from_desc(d).view())

    assert [(g, i) for g, i, *_ in got["instances"]] == [(0, 0), (0, 77), (1, 1), (-1, 2)]
    for a, b in zip(got["instances"], want["instances"]):
        assert a[0] == b[0] and a[1] == b[1]
        for x, y in zip(a[2:], b[2:]):
            assert np.array_equal(x, y)
    assert np.array_equal(got["tlas_nodes"], want["tlas_nodes"])
    assert np.array_equal(got["tlas_inst"], want["tlas_inst"])


def _arrays(scene):
    a = abi.view_arrays(scene.view())
    out = [a["tlas_nodes"], a["tlas_inst"], a["prim_nodes"], a["prim_indices"]]
    for m in a["meshes"]:
        out += [m["nodes"], m["prims"]]
    return [np.ascontiguousarray(x).tobytes() for x in out]


def test_parallel_bvh_build_equals_one_thread_and_the_reference(ref):
    """Meshes built side by side and large subtrees split across threads: the node and index
    arrays equal the one-thread build's, and on a 327,680-triangle mesh the reference's own."""
    import time
    big = scenes.guiding_room(level=7)                              # the sphere crosses every split size
    inst = scenes.instanced_grid(grid=3, levels=(5, 5, 4, 4), with_prims=True)   # several meshes
    for desc in (big, inst):
        t0 = time.perf_counter()
        one = _arrays(HostScene.from_desc(desc, build_threads=1))
        t1 = time.perf_counter()
        many = _arrays(HostScene.from_desc(desc, build_threads=8))
        t2 = time.perf_counter()
        print(desc.name, "1 thread %.3f s, 8 threads %.3f s" % (t1 - t0, t2 - t1))
        assert one == many
    mine = abi.view_arrays(HostScene.from_desc(big, build_threads=8).view())
    theirs = abi.view_arrays(ref.RefScene(big).view())
    sphere = len(big.meshes) - 1
    assert mine["meshes"][sphere]["nodes"].tobytes() == theirs["meshes"][sphere]["nodes"].tobytes()
    assert mine["meshes"][sphere]["prims"].tobytes() == theirs["meshes"][sphere]["prims"].tobytes()
    assert mine["tlas_nodes"].tobytes() == theirs["tlas_nodes"].tobytes()
