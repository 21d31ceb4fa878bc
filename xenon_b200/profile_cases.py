"""Small, fixed workloads for profiling single kernels (ncu) through the public API.

    python -m xenon_b200.profile_cases shadow_d0 [W H]      config-2 scene, camera rays and their
                                                            sun shadow rays only (max_bounces 1)
    python -m xenon_b200.profile_cases guide_small          config-4 room 320x180, depth 16,
                                                            guiding with 2 training samples
    python -m xenon_b200.profile_cases guided_room [W H]    config-4 room, guided bounces with an
                                                            untrained network (no training launches)
    python -m xenon_b200.profile_cases plain_room [W H]     the same renders with plain sampling
    python -m xenon_b200.profile_cases config2 [W H SPP]    config-2 scene, its tuning, SPP samples
                                                            (default 640x360, 2): prints the rays
    python -m xenon_b200.profile_cases config3 [SPP]        config-3 scene at full size, its tuning
    python -m xenon_b200.profile_cases config2_wave [SS]    config-2 scene at 1920x1080, one sample as
                                                            one wave (2,073,600 paths, one lane, direct
                                                            launches; under 1 GB of queues): every
                                                            kernel of a bounce at its full size; SS = 16
                                                            keeps 16 BLAS stack entries in shared memory
    python -m xenon_b200.profile_cases trace_uniform [N]    2^N (default 22) incoherent rays on the config-2
                                                            scene through xb_trace_rays_device, closest
                                                            then any hit

Each case prints one line and exits 0; it renders a handful of samples so a capture of one
launch ends quickly.
"""
from __future__ import annotations

import os
import sys


def _lib():
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import xenon_b200 as xb
    from xenon_b200 import autotune, scenes
    return xb, autotune, scenes


def shadow_d0(w: int = 1920, h: int = 1080) -> None:
    xb, autotune, scenes = _lib()
    desc = scenes.icosphere_scene(level=8, width=w, height=h)
    r = xb.Renderer(w, h, max_bounces=1, min_bounces=3)
    r.upload_scene(xb.HostScene.from_desc(desc))
    t = autotune.load_tuning("config2")
    if t:
        r.set_tuning(**t)
    r.render_frame(xb.camera(desc.eye, desc.target, desc.fov, w / h), 1)
    st = r.stats()
    print("shadow_d0", w, h, "ms", st.last_ms, "shadow rays", st.rays_shadow)


def guide_small() -> None:
    xb, _, scenes = _lib()
    w, h = 320, 180
    desc = scenes.guiding_room(level=6, width=w, height=h)
    r = xb.Renderer(w, h, max_bounces=16, min_bounces=3)
    r.upload_scene(xb.HostScene.from_desc(desc))
    r.set_guiding(True, train_spp=2, steps_per_spp=4, batch=16384)
    r.render_frame(xb.camera(desc.eye, desc.target, desc.fov, w / h), 6)
    print("guide_small ms", r.stats().last_ms, r.guiding_stats())


def guided_room(w: int = 320, h: int = 180, guided: bool = True) -> None:
    xb, _, scenes = _lib()
    desc = scenes.guiding_room(level=6, width=w, height=h)
    r = xb.Renderer(w, h, max_bounces=16, min_bounces=3, wave_paths=1 << 19)
    r.upload_scene(xb.HostScene.from_desc(desc))
    if guided:
        r.set_guiding(True, train_spp=-1)
    r.render_frame(xb.camera(desc.eye, desc.target, desc.fov, w / h), 8)
    print("guided_room" if guided else "plain_room", "ms", r.stats().last_ms)


def plain_room(w: int = 320, h: int = 180) -> None:
    guided_room(w, h, guided=False)


def config2(w: int = 640, h: int = 360, spp: int = 2) -> None:
    xb, autotune, scenes = _lib()
    desc = scenes.icosphere_scene(level=8, width=w, height=h)
    r = xb.Renderer(w, h, desc.max_bounces, desc.min_bounces)
    r.upload_scene(xb.HostScene.from_desc(desc))
    r.set_tuning(**autotune.load_tuning("config2"))
    r.render_frame(xb.camera(desc.eye, desc.target, desc.fov, w / h), spp)
    st = r.stats()
    print("config2", w, h, "spp", spp, "rays_closest", st.rays_closest, "rays_shadow", st.rays_shadow,
          "ms", st.last_ms)


def config3(spp: int = 8) -> None:
    xb, autotune, scenes = _lib()
    desc = scenes.instanced_grid()
    r = xb.Renderer(desc.width, desc.height, desc.max_bounces, desc.min_bounces)
    r.upload_scene(xb.HostScene.from_desc(desc))
    r.set_tuning(**autotune.load_tuning("config3"))
    r.render_frame(xb.camera(desc.eye, desc.target, desc.fov, desc.width / desc.height), spp)
    st = r.stats()
    print("config3 spp", spp, "rays_closest", st.rays_closest, "rays_shadow", st.rays_shadow, "ms", st.last_ms)


def config2_wave(shared_stack: int = 1) -> None:
    xb, autotune, scenes = _lib()
    desc = scenes.icosphere_scene(level=8)
    w, h = desc.width, desc.height
    r = xb.Renderer(w, h, desc.max_bounces, desc.min_bounces)
    r.upload_scene(xb.HostScene.from_desc(desc))
    r.set_tuning(**autotune.load_tuning("config2"))
    r.set_tuning(waves=1, wave_paths=w * h, graph=2, shared_stack=shared_stack)
    r.render_frame(xb.camera(desc.eye, desc.target, desc.fov, w / h), 1)
    st = r.stats()
    print("config2_wave rays_closest", st.rays_closest, "rays_shadow", st.rays_shadow, "ms", st.last_ms)


def trace_uniform(log2n: int = 22) -> None:
    xb, _, scenes = _lib()
    import torch
    from xenon_b200 import abi, raybatch
    desc = scenes.icosphere_scene(level=8)
    hs = xb.HostScene.from_desc(desc)
    r = xb.Renderer(64, 64)
    r.upload_scene(hs)
    rays = raybatch.incoherent_rays(hs.view(), 1 << log2n, seed=5)
    d_rays = torch.from_numpy(rays.view("u1").reshape(-1)).cuda()
    d_hits = torch.empty(len(rays) * abi.HIT_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    for mode in (abi.XB_TRACE_CLOSEST, abi.XB_TRACE_ANY):
        r.trace_rays_device(d_rays.data_ptr(), len(rays), d_hits.data_ptr(), mode)
    r.sync()
    print("trace_uniform rays", len(rays))


CASES = {"config2_wave": config2_wave, "trace_uniform": trace_uniform, "shadow_d0": shadow_d0, "guide_small": guide_small, "guided_room": guided_room,
         "plain_room": plain_room, "config2": config2, "config3": config3}

if __name__ == "__main__":
    if len(sys.argv) < 2 or sys.argv[1] not in CASES:
        print(__doc__)
        sys.exit(2)
    CASES[sys.argv[1]](*[int(a) for a in sys.argv[2:]])
