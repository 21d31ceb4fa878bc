"""The multi-GPU exchange on the device, with one NCCL rank (one GPU per run here): the FP64 sums
go from xb_resolve_fp64_device straight into ncclAllReduce, and share_guide trains and broadcasts
the network on the GPU. The sharded render must equal the plain one-process render of the same
samples; the N-rank split itself is tested on gloo ranks (test_distributed_gloo.py)."""
import socket

import numpy as np
import pytest

import xenon_b200 as xb
from xenon_b200 import distributed, scenes

pytestmark = pytest.mark.gpu
W, H = 64, 48


@pytest.fixture(scope="module")
def nccl_group():
    import torch
    import torch.distributed as dist
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            device_id=torch.device("cuda", 0))
    yield dist.group.WORLD
    dist.destroy_process_group()


def _scene():
    desc = scenes.cornell()
    return desc, xb.HostScene.from_desc(desc), xb.camera(desc.eye, desc.target, desc.fov, W / H)


def test_sharded_render_sums_fp64_on_the_device(nccl_group):
    desc, hs, cam = _scene()
    r = xb.Renderer(W, H, desc.max_bounces, desc.min_bounces, fp64=True)
    r.upload_scene(hs)
    mean, var = distributed.render_sharded(r, cam, 1, 16, 0, 1, group=nccl_group, with_variance=True)
    r.close()
    one = xb.Renderer(W, H, desc.max_bounces, desc.min_bounces, fp64=True)
    one.upload_scene(hs)
    one.render_range(cam, 1, 16)
    s, m2 = one.resolve_fp64()
    one.close()
    assert np.allclose(mean, s / 16, rtol=1e-12, atol=0)
    assert np.allclose(var, m2 / 15, rtol=1e-9, atol=1e-12)
    assert np.isfinite(var).all()


def test_shared_guide_on_the_device(nccl_group):
    desc, hs, cam = _scene()
    r = xb.Renderer(W, H, desc.max_bounces, desc.min_bounces, fp64=True)
    r.upload_scene(hs)
    first = distributed.share_guide(r, cam, 8, 0, 1, group=nccl_group, steps_per_spp=2, batch=1024, seed=5)
    assert first == 9 and r.guiding_stats()["adam_steps"] == 16
    params = r.guide_params()
    mean = distributed.render_sharded(r, cam, first, 8, 0, 1, group=nccl_group)
    assert np.isfinite(mean).all() and mean.mean() > 0
    # the network is the trained one and stays as it is (no training on the image's samples)
    assert np.array_equal(r.guide_params(), params)
    r.close()
