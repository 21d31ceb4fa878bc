"""Multi-GPU host logic on CPU: world_size-2 gloo ranks split the samples with
xenon_b200.distributed and sum their framebuffers; the result must equal one process rendering
every sample. Each rank renders with the CPU oracle behind the same render_range/resolve
interface the GPU renderer has (no GPU here)."""
import os
import socket

import numpy as np
import pytest

from xenon_b200 import distributed
from xenon_b200.abi import GUIDE_PARAMS


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
    """The CPU oracle with the GPU renderer's render_range / resolve / resolve_fp64 interface (FP64
    sums and Welford M2 of the samples, as a renderer created with XB_FLAG_FP64_ACCUM keeps them),
    plus the guiding calls of share_guide: the oracle renders plain, and a network's parameters are
    a vector that "training" on samples first..first+count-1 sets to a function of those indices."""

    def __init__(self, desc, w, h, fp64=True):
        from oracle import port
        from xenon_b200 import HostScene
        self.desc, self.width, self.height = desc, w, h
        self.fp64 = fp64
        self.ps = port.PortScene(HostScene.from_desc(desc).view())
        self.reset()
        self.guiding = None
        self.params = None
        self.trained_on = []

    def reset(self):
        self.sum = np.zeros((self.height, self.width, 3))
        self.sq = np.zeros_like(self.sum)
        self.n = 0

    def render_range(self, cam, first, count):
        train_until = self.guiding["train_spp"] if self.guiding else 0
        for k in range(first, first + count):
            s, _ = self.ps.render(cam, self.width, self.height, self.desc.min_bounces, self.desc.max_bounces,
                                  k, 1, threads=2)
            if k <= train_until:                    # a training sample: trains, stays out of the image
                self.trained_on.append(k)
                continue
            self.sum += s
            self.sq += s * s
            self.n += 1
        if self.trained_on:
            self.params = np.float32(np.arange(GUIDE_PARAMS) % 97 + sum(self.trained_on))

    def resolve(self):
        return (self.sum / self.n).astype(np.float32)

    def resolve_fp64(self):
        return self.sum.copy(), self.sq - self.sum * self.sum / self.n

    def set_guiding(self, enabled=True, **kw):
        self.guiding = dict(kw) if enabled else None
        if self.params is None:
            self.params = np.zeros(GUIDE_PARAMS, np.float32)

    def guide_params(self):
        return self.params.copy()

    def set_guide_params(self, p):
        self.params = np.asarray(p, np.float32).copy()


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
        img, var = distributed.render_sharded(r, cam, 1, 6, rank, world, with_variance=True)
        np.save(os.path.join(out_dir, f"rank{rank}.npy"), img)
        np.save(os.path.join(out_dir, f"var{rank}.npy"), var)
        # guided: one network trained on rank 0 (samples 1..3), the image from samples 4..9
        g = PortRenderer(desc, 16, 16)
        first = distributed.share_guide(g, cam, 3, rank, world, steps_per_spp=8)
        gimg = distributed.render_sharded(g, cam, first, 6, rank, world, dst=0)
        np.save(os.path.join(out_dir, f"params{rank}.npy"), g.guide_params())
        np.save(os.path.join(out_dir, f"trained{rank}.npy"), np.array(g.trained_on, np.int64))
        np.save(os.path.join(out_dir, f"guided_cfg{rank}.npy"), np.array([g.guiding["train_spp"]]))
        if rank == 0:
            np.save(os.path.join(out_dir, "guided.npy"), gimg)
        else:
            assert gimg is None
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
    cam = camera(desc.eye, desc.target, desc.fov, 1.0)
    single = PortRenderer(desc, 16, 16)
    single.render_range(cam, 1, 6)
    want = single.sum / 6
    want_var = (single.sq - single.sum ** 2 / 6) / 5
    for r in range(world):
        got = np.load(tmp_path / f"rank{r}.npy")
        assert np.allclose(got, want, rtol=1e-12, atol=1e-12)     # FP64 sums: exact up to order
        assert np.allclose(np.load(tmp_path / f"var{r}.npy"), want_var, rtol=1e-9, atol=1e-12)
    # guided: every rank holds rank 0's network; only rank 0 trained, on samples 1..3; the image
    # is samples 4..9 of one render
    p0 = np.load(tmp_path / "params0.npy")
    assert np.array_equal(np.load(tmp_path / "params1.npy"), p0) and p0.any()
    assert list(np.load(tmp_path / "trained0.npy")) == [1, 2, 3]
    assert len(np.load(tmp_path / "trained1.npy")) == 0
    assert int(np.load(tmp_path / "guided_cfg1.npy")[0]) == -1    # rank 1 never trains
    single.reset()
    single.render_range(cam, 4, 6)
    assert np.allclose(np.load(tmp_path / "guided.npy"), single.sum / 6, rtol=1e-12, atol=1e-12)
