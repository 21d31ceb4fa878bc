"""Seeded ray batches for the traversal benchmark and the traversal parity tests.

* incoherent rays: origins uniform in the scene's world bounds (the TLAS root box), directions
  uniform on the sphere;
* secondary rays: the rays the path tracer itself casts at bounce 2 and later. Camera rays
  (jittered over the scene's view, as raygen draws them, src/render/cpu_tiled.cpp:20-28) are
  traced, and every hit continues along a direction drawn by the device BSDF sampler for the
  hit's material (xb_bsdf_sample, the reference's bsdf_sample, src/material/bsdf.h:666-708) in
  the shading-normal frame, from an origin offset along the geometric normal
  (offset_ray_origin, src/math/ray.h:22-26); after `bounce` such steps the surviving rays are
  the batch.
"""
from __future__ import annotations

import numpy as np

from . import abi


def world_bounds(view: abi.SceneView) -> tuple:
    """The scene's world-space bounds: the TLAS root box of an uploaded-format view."""
    nodes = abi.view_arrays(view)["tlas_nodes"]
    if len(nodes) == 0:
        raise ValueError("world_bounds: the view has no TLAS")
    return nodes[0]["mn"].astype(np.float32), nodes[0]["mx"].astype(np.float32)


def incoherent_rays(view: abi.SceneView, n: int, seed: int) -> np.ndarray:
    """n rays with origins uniform in the world bounds and directions uniform on S^2."""
    lo, hi = (np.asarray(b, np.float64) for b in world_bounds(view))
    rng = np.random.default_rng(seed)
    org = lo + (hi - lo) * rng.random((n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return abi.make_rays(org.astype(np.float32), d.astype(np.float32))


def _frame(nrm: np.ndarray):
    """Orthonormal tangent frames around unit normals (Duff et al., "Building an Orthonormal
    Basis, Revisited", JCGT 2017), the construction the reference's ONB uses (src/math/ray.h:95-113)."""
    nx, ny, nz = nrm[:, 0], nrm[:, 1], nrm[:, 2]
    sign = np.where(nz >= 0, 1.0, -1.0)
    a = -1.0 / (sign + nz)
    b = nx * ny * a
    t = np.stack([1.0 + sign * nx * nx * a, sign * b, -sign * nx], 1)
    bt = np.stack([b, sign + ny * ny * a, -ny], 1)
    return t, bt


def camera_rays(cam: abi.Camera, width: int, height: int, n: int, seed: int) -> np.ndarray:
    """n camera rays through uniformly drawn pixel positions of a width x height view."""
    c = cam.to_array().astype(np.float64)
    eye, ll, hor, ver = c[0:3], c[3:6], c[6:9], c[9:12]
    rng = np.random.default_rng(seed)
    su = rng.random(n)[:, None]
    sv = rng.random(n)[:, None]
    d = ll + su * hor + sv * ver - eye
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return abi.make_rays(np.tile(eye, (n, 1)).astype(np.float32), d.astype(np.float32))


def secondary_rays(renderer, materials, cam: abi.Camera, width: int, height: int, n: int, seed: int,
                   bounce: int = 2, eps: float = 1e-4) -> np.ndarray:
    """n rays of bounce `bounce` (>= 1) of the path tracer on the renderer's uploaded scene.
    materials: the scene's xb_material arrays (float32[21] each), indexed by the hits' mat_id."""
    from . import bsdf_sample
    rng = np.random.default_rng(seed)
    out = []
    have = 0
    draw = 2 * n
    for _ in range(64):
        rays = camera_rays(cam, width, height, draw, int(rng.integers(1 << 30)))
        for _b in range(bounce):
            h = renderer.trace_rays(rays, abi.XB_TRACE_CLOSEST)
            ok = np.isfinite(h["t"]) & (h["mat_id"] >= 0)
            rays, h = rays[ok], h[ok]
            if len(rays) == 0:
                break
            nrm = h["normal"].astype(np.float64)
            nrm /= np.maximum(np.linalg.norm(nrm, axis=1, keepdims=True), 1e-30)
            t, bt = _frame(nrm)
            wo_w = -rays["dir"].astype(np.float64)
            wo = np.stack([(wo_w * t).sum(1), (wo_w * bt).sum(1), (wo_w * nrm).sum(1)], 1)
            wi = np.zeros_like(wo)
            valid = np.zeros(len(rays), bool)
            for m in np.unique(h["mat_id"]):
                sel = np.nonzero(h["mat_id"] == m)[0]
                states = rng.integers(1, 1 << 62, size=len(sel), dtype=np.uint64)
                w, _f, pdf, fl, _ = bsdf_sample(materials[int(m)], wo[sel].astype(np.float32), states)
                wi[sel] = w
                valid[sel] = ((fl & 1) != 0) & (pdf > 0)
            d = wi[:, 0:1] * t + wi[:, 1:2] * bt + wi[:, 2:3] * nrm
            d /= np.maximum(np.linalg.norm(d, axis=1, keepdims=True), 1e-30)
            gn = h["geo_normal"].astype(np.float64)
            side = np.where((d * gn).sum(1) > 0, 1.0, -1.0)[:, None]
            org = h["pos"].astype(np.float64) + gn * side * eps
            keep = valid & np.isfinite(d).all(1)
            rays = abi.make_rays(org[keep].astype(np.float32), d[keep].astype(np.float32), tmin=eps)
        out.append(rays)
        have += len(rays)
        if have >= n:
            break
        draw = int(min(8 * n, max(draw, 2 * (n - have) * draw / max(len(rays), 1))))
    allr = np.concatenate(out)[:n]
    if len(allr) < n:
        raise RuntimeError(f"secondary_rays: only {len(allr)} of {n} rays survived {bounce} bounces")
    return allr
