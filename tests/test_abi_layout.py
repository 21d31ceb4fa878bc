"""The Python bindings' view of the C ABI: every ctypes structure and numpy record type in
xenon_b200/abi.py has the size and field offsets that a C compiler gives the declarations in
include/xenon_b200.h (gcc on a generated program; no GPU, no library load)."""
import ctypes
import os
import shutil
import subprocess

import pytest

from xenon_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

STRUCTS = {
    "MeshView": "xb_mesh_view", "InstanceView": "xb_instance_view", "Sky": "xb_sky",
    "SceneView": "xb_scene_view", "Camera": "xb_camera", "Config": "xb_config",
    "RenderStats": "xb_render_stats", "Tuning": "xb_tuning", "Profile": "xb_profile",
    "Guiding": "xb_guiding", "GuidingStats": "xb_guiding_stats", "SceneConfig": "xb_scene_config",
    "View": "xb_view", "CameraDesc": "xb_camera_desc", "MaterialDerived": "xb_material_derived",
    "NoiseStats": "xb_noise_stats",
}
DTYPES = {"PRIM_DTYPE": "xb_prim", "RAY_DTYPE": "xb_ray", "HIT_DTYPE": "xb_hit", "NODE_DTYPE": "xb_bvh_node"}


def _python_layout():
    out = {}
    for cls, cname in STRUCTS.items():
        c = getattr(abi, cls)
        out[cname] = (ctypes.sizeof(c), {f[0]: getattr(c, f[0]).offset for f in c._fields_})
    for dname, cname in DTYPES.items():
        d = getattr(abi, dname)
        out[cname] = (d.itemsize, {k: d.fields[k][1] for k in d.names})
    out["xb_material"] = (4 * abi.MATERIAL_FLOATS, {})
    return out


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_bindings_match_the_header(tmp_path):
    want = _python_layout()
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "xenon_b200.h"', "int main(void) {"]
    for cname, (_, fields) in want.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for f in fields:
            lines.append(f'  printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                   check=True)
    got = {}
    for line in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines():
        name, field, value = line.split()
        got[(name, field)] = int(value)
    for cname, (size, fields) in want.items():
        assert got[(cname, "size")] == size, cname
        for f, off in fields.items():
            assert got[(cname, f)] == off, (cname, f)
