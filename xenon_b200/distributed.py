"""Multi-GPU rendering by sample index: one process per GPU, one exchange.

The scene is replicated on every GPU. Samples [first, first + count) of the sequence are split
into contiguous blocks, one per rank; a rank renders its block with xb_render_range, whose
sample k of pixel p is seeded exactly as on one GPU (seed_pcg(p + k * 0xdeadbeef)). The only
collective is a sum of the per-rank framebuffer sums (NCCL reduce / all-reduce over NVLink on
B200; gloo in the CPU tests). The result equals the one-GPU render up to summation order.
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


def render_sharded(renderer, cam, first: int, count: int, rank: int, world: int, group=None,
                   dst: int | None = None) -> np.ndarray | None:
    """Renders this rank's shard and sums the framebuffers across ranks.

    `renderer` needs render_range(cam, first, count) and resolve() (mean over its own samples),
    like xenon_b200.Renderer. Returns the mean image over all `count` samples on every rank
    (dst None: all-reduce) or on rank `dst` only (reduce; other ranks get None)."""
    import torch
    import torch.distributed as dist

    s0, n = shard(first, count, rank, world)
    if n > 0:
        renderer.render_range(cam, s0, n)
        local = renderer.resolve().astype(np.float64) * n
    else:
        local = None
    shape = (renderer.height, renderer.width, 3)
    backend = dist.get_backend(group) if dist.is_initialized() else "gloo"
    device = "cuda" if backend == "nccl" else "cpu"
    t = torch.zeros(shape, dtype=torch.float64, device=device)
    if local is not None:
        t.copy_(torch.from_numpy(local))
    if dst is None:
        dist.all_reduce(t, group=group)
    else:
        dist.reduce(t, dst=dst, group=group)
        if rank != dst:
            return None
    return (t / count).cpu().numpy()
