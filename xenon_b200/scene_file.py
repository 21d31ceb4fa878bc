"""Writes a SceneDesc as files in the reference's scene format: a `.xenon` scene file, one
`.mat` file per material and one Wavefront `.obj` per mesh. This is the inverse of the loader
(xenon_b200.HostScene.load, csrc/loaders.cpp). The format is the one the reference's parser
reads (src/scene/scene_file.cpp:49-231, src/material/material.cpp load_material,
src/geometry/mesh.cpp load_obj), so the reference's own command-line renderer can load the same
seeded scenes. The one exception is the `instance` command, which that parser lacks; with
bake_instances the writer expresses instances as transformed `mesh` lines instead.

Layout under the scene file's directory:

    <name>.xenon                 config, camera, matfile, mesh, light, sunlight, sky,
                                 analytic primitives, instance lines
    materials/<name>_<nnn>_<material>.mat   every xb_material field under the .mat key that sets it
    meshes/<name>_<nnn>.obj      v (+ vn) and f lines, with `usemtl` wherever the material changes

Conventions the reference imposes, which the writer follows:
  * `mesh` paths are opened relative to the working directory (scene_file.cpp:107-111), so the
    file is loaded from its own directory. write_xenon returns that directory with the argv.
  * `matfile` paths are prefixed with `materials/` (scene_file.cpp:80-90). Materials are found
    by name, and where two share a name the last wins, so names must be unique single tokens.
  * Minimum and maximum bounce counts have no scene-file command. They go on the command line
    (`--min-bounces`, `--max-bounces`, src/main.cpp:82-87) and are part of the returned argv.
  * Floats are written with 9 significant digits, which parse back to the same float32.
  * The loader normalises `vn` lines and disk/plane normals, and the API does not. A mesh given
    explicit normals, or a disk or plane given a normal one ulp off unit length, therefore loads
    with normals within an ulp or two of the description's. Positions, indices, BVHs, materials,
    lights, suns, sky and instances load bit-identical.
"""
from __future__ import annotations

import os
import re

import numpy as np

from . import abi

# the .mat key for each xb_material field, in the reference's key spelling (material.cpp)
MAT_KEYS = (("baseColor", "base_color"), ("roughness", "roughness"), ("metallic", "metallic"),
            ("ior", "ior"), ("transmission", "transmission"), ("subsurface", "subsurface"),
            ("subsurfaceColor", "subsurface_color"), ("subsurfaceMFP", "subsurface_mfp"),
            ("clearcoat", "clearcoat"), ("clearcoatRoughness", "clearcoat_roughness"),
            ("anisotropy", "anisotropy"), ("emission", "emission"),
            ("emissionTemperature", "emission_temperature"))
# number of parameters each primitive line carries before its material name (scene_file.cpp:171-229)
PRIM_LINES = {abi.XB_PRIM_SPHERE: ("sphere", 4), abi.XB_PRIM_BOX: ("box", 6),
              abi.XB_PRIM_DISK: ("disk", 7), abi.XB_PRIM_QUAD: ("quad", 9),
              abi.XB_PRIM_PLANE: ("plane", 4)}
_TOKEN = re.compile(r"^[A-Za-z0-9_.\-]{1,127}$")


def _f(x) -> str:
    v = np.float32(x)
    if not np.isfinite(v):
        raise ValueError(f"scene file: non-finite value {x!r} cannot be written")
    return "%.9g" % float(v)


def _fs(xs) -> str:
    return " ".join(_f(x) for x in np.asarray(xs, np.float32).ravel())


def _check_names(desc) -> None:
    seen = set()
    for n in desc.material_names:
        if not _TOKEN.match(n):
            raise ValueError(f"scene file: material name {n!r} is not a single token of [A-Za-z0-9_.-]")
        if n in seen:
            raise ValueError(f"scene file: material name {n!r} is used twice (the loader keeps the last)")
        seen.add(n)


def _write_mat(path: str, name: str, m: np.ndarray) -> None:
    m = np.asarray(m, np.float32)
    lines = [f"name {name}"]
    for key, field in MAT_KEYS:
        lines.append(f"{key} {_fs(m[abi.MATERIAL_FIELDS[field]])}")
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")


def _write_obj(path: str, mesh, names: list) -> None:
    pos = np.asarray(mesh.positions, np.float32).reshape(-1, 3)
    idx = np.asarray(mesh.indices, np.int64).reshape(-1, 3)
    nt = len(idx)
    if not np.all(np.isfinite(pos)):
        raise ValueError(f"scene file: non-finite vertex in {path}")
    if nt and (idx.min() < 0 or idx.max() >= len(pos)):
        raise ValueError(f"scene file: index out of range in {path}")
    mats = np.full(nt, int(mesh.default_mat), np.int64)
    if mesh.mat_ids is not None:
        given = np.asarray(mesh.mat_ids, np.int64)
        mats = np.where(given >= 0, given, mats)        # xb_scene_add_mesh's rule for -1
    if nt and (mats.min() < 0 or mats.max() >= len(names)):
        raise ValueError(f"scene file: material id out of range in {path}")
    with open(path, "w") as fh:
        np.savetxt(fh, pos.astype(np.float64), fmt="v %.9g %.9g %.9g")
        face = "f %d %d %d"
        if mesh.normals is not None:
            nrm = np.asarray(mesh.normals, np.float32).reshape(-1, 3)
            if nrm.shape != pos.shape or not np.all(np.isfinite(nrm)):
                raise ValueError(f"scene file: normals do not match the vertices in {path}")
            np.savetxt(fh, nrm.astype(np.float64), fmt="vn %.9g %.9g %.9g")
            face = "f %d//%d %d//%d %d//%d"
        # the loader starts every mesh on material 0, so a run on another material opens with usemtl
        starts = np.flatnonzero(np.r_[True, mats[1:] != mats[:-1]]) if nt else np.zeros(0, np.int64)
        ends = np.r_[starts[1:], nt]
        one = idx + 1
        if mesh.normals is not None:
            one = np.repeat(one, 2, axis=1)
        for a, b in zip(starts, ends):
            if not (a == 0 and mats[a] == 0):
                fh.write(f"usemtl {names[int(mats[a])]}\n")
            np.savetxt(fh, one[a:b], fmt=face)


def _argv(scene: str, min_bounces: int, max_bounces: int) -> list:
    return ["xenon", "--scene", scene, "--min-bounces", str(int(min_bounces)),
            "--max-bounces", str(int(max_bounces)), "--backend", "cuda"]


def _baked(desc, mesh_files: list):
    """The reference's parser has no `instance` command: it places every `mesh` line once, at
    the transform baked into its vertices, and the analytic primitives at the identity. So each
    mesh instance becomes a `mesh` line with the instance's transform, and each light moves to
    the line of the instance whose id it names. Returns (mesh lines, lights)."""
    lines, line_of = [], {}
    prims_placed = False
    for (geom, t, s, r, iid) in desc.instances:
        t, r = np.asarray(t, np.float32), np.asarray(r, np.float32)
        identity = not t.any() and np.float32(s) == 1 and not r.any()
        if int(geom) == abi.XB_GEOM_PRIMS:
            if not identity or prims_placed:
                raise ValueError("scene file: analytic primitives bake only as one instance at the identity")
            prims_placed = True
            continue
        mesh = desc.meshes[int(geom)]
        if mesh.transform is not None and not identity:
            raise ValueError("scene file: a transformed mesh cannot be baked under another transform")
        if int(iid) in line_of:
            raise ValueError(f"scene file: instance id {int(iid)} is used twice")
        line_of[int(iid)] = len(lines)
        lines.append((mesh_files[int(geom)], mesh.transform if identity else (t, s, r)))
    if desc.prims and not prims_placed:
        raise ValueError("scene file: the primitives have no instance, which the reference always places")
    lights = []
    for (mesh_id, tri, e, area) in desc.lights:
        if int(mesh_id) not in line_of:
            raise ValueError(f"scene file: a light names instance id {int(mesh_id)}, which no instance has")
        lights.append((line_of[int(mesh_id)], tri, e, area))
    return lines, lights


def _scene_lines(desc, mesh_lines: list, lights: list, instances: list, mat_files: list, eye, target,
                 fov, w, h, spp) -> list:
    names = desc.material_names
    out = [f"# {desc.name}: written by xenon_b200.scene_file.write_xenon",
           f"config {int(w)} {int(h)} {int(spp)}",
           f"camera {_fs(eye)} {_fs(target)} {_f(fov)}"]
    out += [f"matfile {f}" for f in mat_files]
    for f, transform in mesh_lines:
        line = f"mesh {f}"
        if transform is not None:
            t, s, r = transform
            line += f" {_fs(t)} {_f(s)} {_fs(r)}"
        out.append(line)
    for (mesh_id, tri, e, area) in lights:
        out.append(f"light {int(mesh_id)} {int(tri)} {_fs(e)} {_f(area)}")
    for (d, c, inten) in desc.suns:
        out.append(f"sunlight {_fs(d)} {_fs(c)} {_f(inten)}")
    sky = np.asarray(desc.sky, np.float32)
    out.append(f"sky {_fs(sky[0:9])} {_f(sky[10])} {_f(sky[9])}")   # intensity before sharpness
    for p in desc.prims:
        q = np.asarray(p, abi.PRIM_DTYPE).reshape(-1)[0]
        kind, n = PRIM_LINES[int(q["type"])]
        out.append(f"{kind} {_fs(q['p'][:n])} {names[int(q['mat_id'])]}")
    for (geom, t, s, r, iid) in instances:
        what = "prims" if int(geom) == abi.XB_GEOM_PRIMS else str(int(geom))
        out.append(f"instance {what} {_fs(t)} {_f(s)} {_fs(r)} {int(iid)}")
    return out


def write_xenon(desc, path: str, views: list | None = None, bake_instances: bool = False) -> list:
    """Writes `desc` to `path` (a .xenon file), its materials under materials/ and its meshes
    under meshes/ beside it. With `views`, a list of (eye, target, fov, width, height, spp
    [, max_bounces]) tuples as scenes.config5_views returns, it also writes one
    `<stem>_viewNN.xenon` per view, sharing the same material and mesh files.

    Instances are written as `instance` lines, which only this library's loader reads. With
    `bake_instances`, each one is written instead as a `mesh` line carrying its transform, which
    the reference's parser reads too. The scene then has one BLAS per instance, and the
    reference's loader reads the shared .obj once per line.

    Returns one entry per scene file written, the main one first:
    {"scene": path, "cwd": directory to load it from, "argv": the reference CLI's arguments}."""
    if desc.instances and any(int(g) != abi.XB_GEOM_PRIMS and not 0 <= int(g) < len(desc.meshes)
                              for (g, *_) in desc.instances):
        raise ValueError("scene file: an instance names a mesh that does not exist")
    _check_names(desc)
    for p in desc.prims:
        q = np.asarray(p, abi.PRIM_DTYPE).reshape(-1)[0]
        if int(q["type"]) not in PRIM_LINES or not 0 <= int(q["mat_id"]) < len(desc.materials):
            raise ValueError("scene file: primitive with a bad type or material")
    root = os.path.dirname(os.path.abspath(path))
    stem = os.path.splitext(os.path.basename(path))[0]
    os.makedirs(os.path.join(root, "materials"), exist_ok=True)
    os.makedirs(os.path.join(root, "meshes"), exist_ok=True)
    mat_files = []
    for i, (name, m) in enumerate(zip(desc.material_names, desc.materials)):
        f = f"{stem}_{i:03d}_{name}.mat"
        _write_mat(os.path.join(root, "materials", f), name, m)
        mat_files.append(f)
    mesh_files = []
    for i, mesh in enumerate(desc.meshes):
        f = f"meshes/{stem}_{i:03d}.obj"
        _write_obj(os.path.join(root, f), mesh, desc.material_names)
        mesh_files.append(f)

    if bake_instances and desc.instances:
        mesh_lines, lights = _baked(desc, mesh_files)
        instances = []
    else:
        mesh_lines = [(f, m.transform) for f, m in zip(mesh_files, desc.meshes)]
        lights, instances = desc.lights, desc.instances

    def emit(file, eye, target, fov, w, h, spp, max_b):
        lines = _scene_lines(desc, mesh_lines, lights, instances, mat_files, eye, target, fov, w, h, spp)
        lines.insert(1, f"# bounces {desc.min_bounces}..{max_b}: --min-bounces {desc.min_bounces} "
                        f"--max-bounces {max_b} on the command line")
        with open(file, "w") as fh:
            fh.write("\n".join(lines) + "\n")
        return {"scene": file, "cwd": root, "argv": _argv(os.path.basename(file), desc.min_bounces, max_b)}

    out = [emit(os.path.abspath(path), desc.eye, desc.target, desc.fov, desc.width, desc.height,
                desc.spp, desc.max_bounces)]
    for k, v in enumerate(views or []):
        eye, target, fov, w, h, spp = v[:6]
        max_b = v[6] if len(v) > 6 else desc.max_bounces
        out.append(emit(os.path.join(root, f"{stem}_view{k:02d}.xenon"), eye, target, fov, w, h, spp, max_b))
    return out


def main(argv=None) -> int:
    """python -m xenon_b200.scene_file <scene> <out.xenon>: cornell (256x256 box, 64 spp),
    icosphere (1.31 M-triangle conductor, sun and sky), instanced (16x16 instances of 4 meshes),
    room (closed room with a baffled light and a glass sphere), prims (the five analytic
    primitives), views (the instanced scene plus 32 seeded views, one file each)."""
    import argparse
    import json
    from . import scenes
    makers = {"cornell": scenes.cornell, "icosphere": scenes.icosphere_scene,
              "instanced": scenes.instanced_grid, "room": scenes.guiding_room,
              "prims": scenes.prim_showcase, "views": scenes.instanced_grid}
    ap = argparse.ArgumentParser(description="Write a seeded scene as .xenon/.mat/.obj files.")
    ap.add_argument("scene", choices=sorted(makers))
    ap.add_argument("out")
    ap.add_argument("--bake-instances", action="store_true",
                    help="one mesh line per instance, for the reference's parser (no instance lines)")
    a = ap.parse_args(argv)
    desc = makers[a.scene]()
    views = scenes.config5_views(desc, 32, seed=1) if a.scene == "views" else None
    for e in write_xenon(desc, a.out, views, bake_instances=a.bake_instances):
        print(json.dumps(e))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
