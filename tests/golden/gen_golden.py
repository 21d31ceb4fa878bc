#!/usr/bin/env python3
"""Generates the golden vectors under tests/golden/ from the reference's own CPU code.

Run where the reference sources exist (`make -C oracle ref` first): every expected value here
is computed by the reference itself (oracle/_ref/libxnref_strict.so: its BLAS/TLAS build,
Scene::intersect / intersects, bsdf_eval_for_nee / bsdf_pdf_for_nee / bsdf_sample,
Camera::look_at, material_prepare, the .xenon / .mat loaders and render_frame_tiled), and for
the output stage its ImageNoiseEstimator and save_image's 8-bit conversion (output.npz; run
`python tests/golden/gen_golden.py output` to write that file alone). The converged config-1
image at 256x256 and 16k samples (config1_256.npz) takes minutes: `... gen_golden.py config1`
writes it alone.
Inputs are this repo's seeded procedural scenes (xenon_b200/scenes.py), so the files are
reproducible: `python tests/golden/gen_golden.py`.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import ref  # noqa: E402
from xenon_b200 import abi, scenes  # noqa: E402

TRACE_SCENES = {
    "cornell": lambda: scenes.cornell(),
    "prims": lambda: scenes.prim_showcase(),
    "instanced": lambda: scenes.instanced_grid(grid=3, levels=(3, 3, 3, 3), with_prims=True),
    "icosphere": lambda: scenes.icosphere_scene(level=4),
    "room": lambda: scenes.guiding_room(level=3),
}

BSDF_MATERIALS = {
    "diffuse": abi.material(base_color=(0.7, 0.3, 0.5), roughness=1.0),
    "plastic": abi.material(base_color=(0.2, 0.6, 0.9), roughness=0.35),
    "conductor": abi.material(base_color=(0.95, 0.64, 0.54), metallic=1.0, roughness=0.3),
    "aniso_metal": abi.material(base_color=(0.8, 0.8, 0.82), metallic=1.0, roughness=0.25, anisotropy=0.6),
    "rough_glass": abi.material(base_color=(1.0, 1.0, 1.0), transmission=1.0, ior=1.5, roughness=0.2),
    "subsurface": abi.material(base_color=(0.9, 0.7, 0.6), subsurface=0.5, subsurface_color=(0.9, 0.3, 0.2)),
    "glass": abi.material(base_color=(1.0, 1.0, 1.0), transmission=1.0, ior=1.5, roughness=0.0),
    "mirror": abi.material(base_color=(0.9, 0.9, 0.9), metallic=1.0, roughness=0.01),
}


def rays_for(desc, n, seed):
    lo, hi = scenes.scene_bounds(desc)
    if desc.prims and not desc.meshes:
        lo, hi = np.array([-10, 0, -5], np.float32), np.array([10, 6, 5], np.float32)
    pad = (hi - lo) * 0.05 + 0.1
    r = scenes.random_rays((lo - pad, hi + pad), n, seed)
    cam = ref.camera(desc.eye, desc.target, desc.fov, desc.width / desc.height)
    rng = np.random.default_rng(seed + 1)
    st = rng.random((n, 2)).astype(np.float32)
    d = cam[3:6] + st[:, :1] * cam[6:9] + st[:, 1:] * cam[9:12] - cam[0:3]
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    r2 = abi.make_rays(np.tile(cam[0:3], (n, 1)), d)
    return np.concatenate([r, r2])


def main():
    out = {}
    # ── traversal, BVH, camera ──
    for name, build in TRACE_SCENES.items():
        desc = build()
        rs = ref.RefScene(desc)
        rays = rays_for(desc, 1024, 17)
        closest = rs.trace(rays, 0)
        anyhit = rs.trace(rays, 1)
        v = abi.view_arrays(rs.view())
        out[f"trace_{name}_rays"] = rays
        out[f"trace_{name}_closest"] = closest
        out[f"trace_{name}_any"] = np.isfinite(anyhit["t"])
        out[f"bvh_{name}_tlas"] = v["tlas_nodes"]
        out[f"bvh_{name}_tlas_inst"] = v["tlas_inst"]
        out[f"bvh_{name}_prim_nodes"] = v["prim_nodes"]
        out[f"bvh_{name}_prim_indices"] = v["prim_indices"]
        for i, m in enumerate(v["meshes"]):
            out[f"bvh_{name}_mesh{i}_nodes"] = m["nodes"]
            out[f"bvh_{name}_mesh{i}_prims"] = m["prims"]
            if m["nrm"] is not None:
                out[f"bvh_{name}_mesh{i}_normals"] = m["nrm"]
        out[f"camera_{name}"] = ref.camera(desc.eye, desc.target, desc.fov, desc.width / desc.height)
    np.savez_compressed(os.path.join(HERE, "trace_bvh.npz"), **out)

    # ── BSDF grids and samples ──
    out = {}
    rng = np.random.default_rng(5)
    n = 1024
    wo = rng.normal(size=(n, 3)); wo /= np.linalg.norm(wo, axis=1, keepdims=True)
    wi = rng.normal(size=(n, 3)); wi /= np.linalg.norm(wi, axis=1, keepdims=True)
    wo[: n // 2, 2] = np.abs(wo[: n // 2, 2])
    wo, wi = wo.astype(np.float32), wi.astype(np.float32)
    out["wo"], out["wi"] = wo, wi
    states = np.array([ref.seed_pcg(100 + i) for i in range(n)], np.uint64)
    out["states"] = states
    for name, m in BSDF_MATERIALS.items():
        f, p = ref.bsdf_eval(m, wo, wi)
        out[f"{name}_material"] = m
        out[f"{name}_f"], out[f"{name}_pdf"] = f, p
        swi, sf, sp, sfl, sst = ref.bsdf_sample(m, wo, states)
        out[f"{name}_s_wi"], out[f"{name}_s_f"], out[f"{name}_s_pdf"] = swi, sf, sp
        out[f"{name}_s_flags"], out[f"{name}_s_states"] = sfl, sst
        d = abi.MaterialDerived()
        ref.lib().xr_material_prepare(ref.ptr(m), __import__("ctypes").byref(d))
        out[f"{name}_derived"] = np.array([d.alpha, d.alpha_x, d.alpha_y, *d.f0, float(d.flags)], np.float32)
    out["seed_pcg"] = np.array([ref.seed_pcg(s) for s in (0, 1, 2, 12345, 2**40 + 7)], np.uint64)
    np.savez_compressed(os.path.join(HERE, "bsdf.npz"), **out)

    # ── renders (FP64 sums of samples 1..k, top-down rows) ──
    out = {}
    cases = {"cornell": (scenes.cornell(), 32, 32, 2), "icosphere": (scenes.icosphere_scene(level=4), 32, 18, 2),
             "prims": (scenes.prim_showcase(), 32, 24, 2),
             "instanced": (scenes.instanced_grid(grid=3, levels=(3, 3, 3, 3), with_prims=True), 32, 18, 2)}
    for name, (desc, w, h, spp) in cases.items():
        rr = ref.RefRenderer(w, h, desc.min_bounces, desc.max_bounces)
        s, _ = rr.render(ref.RefScene(desc), desc.eye, desc.target, desc.fov, 1, spp)
        out[f"{name}_sum"] = s
        out[f"{name}_spp"] = np.array(spp)
    # converged config-1 box (the reference's own render, 64x64, 4096 samples)
    desc = scenes.cornell()
    rr = ref.RefRenderer(64, 64, desc.min_bounces, desc.max_bounces)
    s, secs = rr.render(ref.RefScene(desc), desc.eye, desc.target, desc.fov, 1, 4096)
    out["cornell64_mean"] = (s / 4096).astype(np.float32)
    out["cornell64_spp"] = np.array(4096)
    np.savez_compressed(os.path.join(HERE, "render.npz"), **out)

    # ── loaders ──
    sc_path = os.path.join(HERE, "scenes", "loader_test.xenon")
    cwd = os.getcwd()
    os.chdir(os.path.join(HERE, "scenes"))
    try:
        import ctypes
        h = ctypes.c_void_p()
        cfg = np.zeros(3, np.int32)
        cam = np.zeros(12, np.float32)
        rc = ref.lib().xr_scene_load_xenon(b"loader_test.xenon", ctypes.byref(h), ref.ptr(cfg), ref.ptr(cam))
        assert rc == 0
        v = abi.SceneView()
        ref.lib().xr_scene_view(h, ctypes.byref(v))
        mats = np.frombuffer((ctypes.c_char * (v.num_materials * 84)).from_address(v.materials), np.float32).reshape(-1, 21).copy()
        prims = np.frombuffer((ctypes.c_char * (v.num_prims * 48)).from_address(v.prims), abi.PRIM_DTYPE).copy()
        suns = np.frombuffer((ctypes.c_char * (v.num_suns * 28)).from_address(v.suns), np.float32).reshape(-1, 7).copy()
        sky = np.array(list(v.sky.zenith) + list(v.sky.horizon) + list(v.sky.ground) + [v.sky.sharpness, v.sky.intensity], np.float32)
        arrays = abi.view_arrays(v)
        np.savez_compressed(os.path.join(HERE, "loader.npz"), config=cfg, camera=cam, materials=mats, prims=prims,
                            suns=suns, sky=sky, prim_nodes=arrays["prim_nodes"], tlas_nodes=arrays["tlas_nodes"])
    finally:
        os.chdir(cwd)
    print("golden vectors written to", HERE)


def output_stage():
    """The output stage: noise statistics and 8-bit values of seeded images, edge cases and the
    reference's converged 64x64 config-1 render (render.npz)."""
    rng = np.random.default_rng(11)
    yy, xx = np.mgrid[0:48, 0:64].astype(np.float32)
    smooth = np.stack([xx / 64, yy / 48, 0.5 + 0.0 * xx], -1)
    imgs = {
        "noisy_gradient": smooth * (1 + 0.2 * rng.normal(size=smooth.shape)),
        "hdr_edges": np.where((xx[..., None] // 8 + yy[..., None] // 8) % 2 == 0, 3.0, 0.2)
                     * (1 + 0.05 * rng.normal(size=smooth.shape)) - 0.01,
        "tiny_3x3": rng.random((3, 3, 3)),
        "no_interior_2x5": rng.random((2, 5, 3)),
        "black": np.zeros((9, 7, 3)),
        "cornell64": np.load(os.path.join(HERE, "render.npz"))["cornell64_mean"],
    }
    out = {}
    for name, img in imgs.items():
        img = np.ascontiguousarray(img, np.float32)
        f, c = ref.noise_stats(img)
        out[f"{name}_image"] = img
        out[f"{name}_stats"], out[f"{name}_counts"] = f, c
        out[f"{name}_rgb8"] = ref.image_rgb8(img)
    np.savez_compressed(os.path.join(HERE, "output.npz"), **out)
    print("output-stage vectors written to", HERE)


def config1_converged():
    """Config 1 at its own size, converged: the reference's render of the 256x256 Cornell box
    over samples 1..16384 (FP64 sums, strict build; about five minutes on eight cores), stored as
    the float32 mean image (top-down rows)."""
    desc = scenes.cornell()
    spp = 16384
    rr = ref.RefRenderer(desc.width, desc.height, desc.min_bounces, desc.max_bounces)
    s, secs = rr.render(ref.RefScene(desc), desc.eye, desc.target, desc.fov, 1, spp)
    np.savez_compressed(os.path.join(HERE, "config1_256.npz"), mean=(s / spp).astype(np.float32),
                        spp=np.array(spp), seconds=np.array(secs))
    print(f"config-1 16k-spp reference written ({secs:.0f} s)")


if __name__ == "__main__":
    if sys.argv[1:] == ["config1"]:
        config1_converged()
        sys.exit(0)
    if sys.argv[1:] != ["output"]:
        main()
        config1_converged()
    output_stage()
