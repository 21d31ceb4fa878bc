"""Shared helpers for the parity tests (ray batches, ulp distances, hit comparison)."""
from __future__ import annotations

import numpy as np

from xenon_b200 import abi, scenes


def ulp_diff(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Distance in units of last place between float32 arrays (same-sign finite values)."""
    a = np.asarray(a, np.float32).view(np.int32).astype(np.int64)
    b = np.asarray(b, np.float32).view(np.int32).astype(np.int64)
    a = np.where(a < 0, np.int64(-0x80000000) - a, a)
    b = np.where(b < 0, np.int64(-0x80000000) - b, b)
    return np.abs(a - b)


def camera_rays(desc, n_side: int, seed: int = 0) -> np.ndarray:
    """Jittered primary rays of the scene camera through an n_side x n_side grid."""
    from oracle import ref
    cam = ref.camera(desc.eye, desc.target, desc.fov, desc.width / desc.height)
    eye, ll, hz, vt = cam[0:3], cam[3:6], cam[6:9], cam[9:12]
    rng = np.random.default_rng(seed)
    s = (np.arange(n_side)[:, None] + rng.random((n_side, n_side))) / n_side
    t = (np.arange(n_side)[None, :] + rng.random((n_side, n_side))) / n_side
    s, t = s.reshape(-1, 1).astype(np.float32), t.reshape(-1, 1).astype(np.float32)
    d = (ll + s * hz + t * vt - eye).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return abi.make_rays(np.tile(eye, (len(d), 1)), d.astype(np.float32))


def mixed_rays(desc, n: int, seed: int) -> np.ndarray:
    """Incoherent rays in the scene bounds plus camera rays."""
    lo, hi = scenes.scene_bounds(desc)
    if desc.prims and not desc.meshes:
        lo, hi = np.array([-10, 0, -5], np.float32), np.array([10, 6, 5], np.float32)
    pad = (hi - lo) * 0.05 + 0.1
    r1 = scenes.random_rays((lo - pad, hi + pad), n, seed)
    r2 = camera_rays(desc, int(np.sqrt(n)), seed)
    return np.concatenate([r1, r2])


def prim_instance_ids(desc) -> set:
    """Instance ids whose geometry is the analytic prim group."""
    if not desc.prims:
        return set()
    if not desc.instances:
        return {len(desc.meshes)}
    return {iid for (geom, _t, _s, _r, iid) in desc.instances if geom == abi.XB_GEOM_PRIMS}


def compare_hits(got: np.ndarray, want: np.ndarray, max_ulp: int = 4, prim_ids: set = frozenset()) -> dict:
    """Ids must match exactly; t, and the barycentrics u/v of triangle hits, within max_ulp.
    Analytic prims report UVs from atan2/acos (CUDA vs glibc), compared to 1e-5 absolute."""
    hit = np.isfinite(want["t"])
    out = {"n": len(want), "hits": int(hit.sum())}
    out["hit_mismatch"] = int((np.isfinite(got["t"]) != hit).sum())
    for k in ("prim_id", "instance_id", "mat_id"):
        out[k + "_mismatch"] = int((got[k] != want[k]).sum())
    both = hit & np.isfinite(got["t"])
    is_prim = np.isin(want["instance_id"], list(prim_ids)) if prim_ids else np.zeros(len(want), bool)
    tri = both & ~is_prim
    pr = both & is_prim
    out["t_ulp_max"] = int(ulp_diff(got["t"][both], want["t"][both]).max()) if both.any() else 0
    for k in ("u", "v"):
        out[k + "_ulp_max"] = int(ulp_diff(got[k][tri], want[k][tri]).max()) if tri.any() else 0
        out[k + "_prim_maxabs"] = float(np.abs(got[k][pr] - want[k][pr]).max()) if pr.any() else 0.0
    out["prim_hits"] = int(pr.sum())
    out["front_mismatch"] = int((got["front_face"][both] != want["front_face"][both]).sum())
    for k in ("normal", "geo_normal", "pos"):
        out[k + "_maxabs"] = float(np.abs(got[k][both] - want[k][both]).max()) if both.any() else 0.0
    return out


def deep_chain_scene(depth: int = 100, seed: int = 3):
    """A one-mesh scene whose BLAS is a chain of `depth` interior nodes, every node with the
    mesh's bounding box: interior node 2k has children 2k+1 (a one-triangle leaf) and 2k+2 (the
    next interior node; the last one's children are two leaves). Both children of every node are
    entered at the same t, so the traversal continues into the right child (the reference's
    order for equal entry distances, blas.cpp:242-262) and pushes the leaf: a ray through the box
    needs `depth` stack entries, more than the 64 the traversal holds when depth > 64.
    Returns (host scene, its view with the chain BLAS, rays through the box)."""
    import ctypes

    from xenon_b200 import HostScene
    rng = np.random.default_rng(seed)
    ntri = depth + 1
    base = rng.random((ntri, 3)).astype(np.float32)
    pos = np.repeat(base, 3, axis=0) + (rng.random((3 * ntri, 3)) * 0.05).astype(np.float32)
    desc = scenes.SceneDesc()
    desc.add_material("m", abi.material())
    desc.add_mesh(scenes.MeshDesc(positions=pos.astype(np.float32),
                                  indices=np.arange(3 * ntri, dtype=np.int32).reshape(ntri, 3)))
    hs = HostScene.from_desc(desc)
    v = hs.view()
    mn, mx = pos.min(0), pos.max(0)
    nodes = np.zeros(2 * depth + 1, abi.NODE_DTYPE)
    nodes["mn"], nodes["mx"] = mn, mx
    for k in range(depth):
        nodes[2 * k]["child"] = 2 * k + 1
        nodes[2 * k + 1]["child"], nodes[2 * k + 1]["count"] = k, 1
    nodes[2 * depth]["child"], nodes[2 * depth]["count"] = depth, 1
    prims = np.arange(ntri, dtype=np.uint32)
    mv = v.meshes[0]
    mv.blas_nodes = nodes.ctypes.data
    mv.num_blas_nodes = len(nodes)
    mv.blas_prims = prims.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))
    v._chain = (nodes, prims)          # the view points into these arrays
    n = 4096
    org = np.stack([np.full(n, mn[0] - 1.0), rng.uniform(mn[1], mx[1], n), rng.uniform(mn[2], mx[2], n)], 1)
    rays = abi.make_rays(org.astype(np.float32), np.tile(np.float32([1, 0, 0]), (n, 1)))
    return hs, v, rays
