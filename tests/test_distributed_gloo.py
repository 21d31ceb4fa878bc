"""Multi-GPU host logic on CPU: world_size-2 gloo ranks split the samples with
xenon_b200.distributed and sum their framebuffers; the result must equal one process rendering
every sample. Each rank renders with the CPU oracle behind the same render_range/resolve
interface the GPU renderer has (no GPU here)."""
import os
import socket

import numpy as np
import pytest

from xenon_b200 import distributed


def test_shard_covers_every_sample_once():
    for count in (0, 1, 7, 64, 1000):
        for world in (1, 2, 3, 8):
            got = []
            for r in range(world):
                s, n = distributed.shard(5, count, r, world)
                got += list(range(s, s + n))
            assert got == list(range(5, 5 + count))
    with pytest.raises(ValueError):
        distributed.shard(1, 4, 2, 2)


class PortRenderer:
    """The CPU oracle with the GPU renderer's render_range / resolve interface."""

    def __init__(self, desc, w, h):
        from oracle import port
        from xenon_b200 import HostScene
        self.desc, self.width, self.height = desc, w, h
        self.ps = port.PortScene(HostScene.from_desc(desc).view())
        self.sum = np.zeros((h, w, 3))
        self.n = 0

    def render_range(self, cam, first, count):
        s, _ = self.ps.render(cam, self.width, self.height, self.desc.min_bounces, self.desc.max_bounces,
                              first, count, threads=2)
        self.sum += s
        self.n += count

    def resolve(self):
        return (self.sum / self.n).astype(np.float32)


def _rank_main(rank, world, port_no, out_dir):
    import torch.distributed as dist
    from xenon_b200 import camera, scenes
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port_no)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        desc = scenes.cornell()
        r = PortRenderer(desc, 16, 16)
        cam = camera(desc.eye, desc.target, desc.fov, 1.0)
        img = distributed.render_sharded(r, cam, 1, 6, rank, world)
        np.save(os.path.join(out_dir, f"rank{rank}.npy"), img)
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_two_gloo_ranks_equal_one_render(tmp_path):
    import torch.multiprocessing as mp
    from xenon_b200 import camera, scenes
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    desc = scenes.cornell()
    single = PortRenderer(desc, 16, 16)
    single.render_range(camera(desc.eye, desc.target, desc.fov, 1.0), 1, 6)
    want = single.sum / 6
    for r in range(world):
        got = np.load(tmp_path / f"rank{r}.npy")
        assert np.allclose(got, want, rtol=1e-6, atol=1e-7)
