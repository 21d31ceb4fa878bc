"""Multi-GPU rendering by sample index: one process per GPU, one exchange.

The scene is replicated on every GPU. Samples [first, first + count) of the sequence are split
into contiguous blocks, one per rank; a rank renders its block with xb_render_range, whose
sample k of pixel p is seeded exactly as on one GPU (seed_pcg(p + k * 0xdeadbeef)). The only
collective of a plain render is one sum of the per-rank FP64 accumulations (per pixel the sum of
the samples and the sum of their squares): with a renderer created with FP64 accumulation on an
NCCL group the sums go from xb_resolve_fp64_device straight into the all-reduce, on the device
(NVLink on B200); gloo groups (the CPU tests) take them through the host. The mean equals the
one-GPU render up to summation order, and the per-pixel variance of the whole render comes with it.

Guided rendering (share_guide): one network serves every rank. Rank `src` trains it on samples
1..train_spp (the renderer's online training), the parameters (abi.GUIDE_PARAMS floats) are
broadcast, and every rank then renders its block of samples train_spp + 1, ... with that network
and no further training, so the guided image is one estimator split by sample index.
"""
from __future__ import annotations

import numpy as np


def shard(first: int, count: int, rank: int, world: int) -> tuple[int, int]:
    """(first, count) of the contiguous block of samples owned by `rank`."""
    if world <= 0 or not 0 <= rank < world or count < 0:
        raise ValueError("bad shard request")
    q, rem = divmod(count, world)
    start = first + rank * q + min(rank, rem)
    return start, q + (1 if rank < rem else 0)


def _backend(group):
    import torch.distributed as dist
    return dist.get_backend(group) if dist.is_initialized() else "gloo"


def _local_moments(renderer, n: int, device: str):
    """This rank's per-pixel [sum, sum of squares] of its n samples as one float64 tensor
    (2, H, W, 3) on `device`: from the renderer's FP64 sums and Welford M2 when it has them
    (M2 + sum^2 / n = sum of squares), else from its FP32 mean (sum only, squares unknown: NaN)."""
    import torch
    shape = (2, renderer.height, renderer.width, 3)
    t = torch.zeros(shape, dtype=torch.float64, device=device)
    if n == 0:
        return t
    if getattr(renderer, "fp64", False):
        if device != "cpu" and hasattr(renderer, "resolve_fp64_device"):
            renderer.resolve_fp64_device(t[0].data_ptr(), t[1].data_ptr())
        else:
            s, m2 = renderer.resolve_fp64()
            t[0].copy_(torch.from_numpy(np.ascontiguousarray(s)))
            t[1].copy_(torch.from_numpy(np.ascontiguousarray(m2)))
        t[1] += t[0] * t[0] / n
    else:
        t[0].copy_(torch.from_numpy(renderer.resolve().astype(np.float64) * n))
        t[1].fill_(float("nan"))
    return t


def render_sharded(renderer, cam, first: int, count: int, rank: int, world: int, group=None,
                   dst: int | None = None, with_variance: bool = False):
    """Renders this rank's shard and sums the accumulations across ranks.

    `renderer` needs render_range(cam, first, count), resolve() and, for the FP64 path, an `fp64`
    attribute with resolve_fp64() / resolve_fp64_device() (xenon_b200.Renderer has them). Returns
    the mean image over all `count` samples on every rank (dst None: all-reduce) or on rank `dst`
    only (reduce; other ranks get None); with_variance: (mean, per-pixel sample variance), the
    variance NaN unless the renderer accumulates in FP64."""
    import torch.distributed as dist

    s0, n = shard(first, count, rank, world)
    if n > 0:
        renderer.render_range(cam, s0, n)
    device = "cuda" if _backend(group) == "nccl" else "cpu"
    t = _local_moments(renderer, n, device)
    if dst is None:
        dist.all_reduce(t, group=group)
    else:
        dist.reduce(t, dst=dst, group=group)
        if rank != dst:
            return None
    s1, s2 = t[0], t[1]
    mean = (s1 / count).cpu().numpy()
    if not with_variance:
        return mean
    var = ((s2 - s1 * s1 / count) / max(count - 1, 1)).cpu().numpy()
    return mean, var


def share_guide(renderer, cam, train_spp: int, rank: int, world: int, group=None, src: int = 0,
                **guiding) -> int:
    """One guiding network for every rank: rank `src` trains it on samples 1..train_spp (online
    training as in a single-GPU guided render, those samples left out of its image), then the
    parameters are broadcast and set on the other ranks, whose renderers guide with them and
    never train. Returns the first sample index for the image (train_spp + 1); render the image
    with render_sharded(renderer, cam, train_spp + 1, count, ...). `guiding`: other xb_guiding
    fields (steps_per_spp, batch, learning_rate, ...), the same on every rank."""
    import torch
    import torch.distributed as dist

    from .abi import GUIDE_PARAMS
    if train_spp < 1:
        raise ValueError("share_guide: train_spp >= 1")
    guiding = {k: v for k, v in guiding.items() if k not in ("train_spp", "keep_training_samples")}
    device = "cuda" if _backend(group) == "nccl" else "cpu"
    if rank == src:
        renderer.set_guiding(True, train_spp=train_spp, keep_training_samples=0, **guiding)
        renderer.render_range(cam, 1, train_spp)
        renderer.reset()
        p = torch.from_numpy(np.ascontiguousarray(renderer.guide_params(), np.float32)).to(device)
    else:
        renderer.set_guiding(True, train_spp=-1, **guiding)
        p = torch.zeros(GUIDE_PARAMS, dtype=torch.float32, device=device)
    dist.broadcast(p, src=src, group=group)
    if rank != src:
        renderer.set_guide_params(p.cpu().numpy())
    return train_spp + 1
