"""Autotuner for the wavefront launch parameters (xb_tuning).

For one scene and resolution it measures the device time per sample (CUDA events inside
xb_render) while varying one parameter at a time around the current best (coordinate descent,
two passes), and keeps the fastest setting:

  extend_persistent_from_depth   which bounces trace closest hits with persistent warps
  shadow_persistent              persistent warps or one ray per thread for shadow rays
  shadow_order                   nearer or farther child first for shadow (any-hit) rays
  overlap                        shadow rays of a bounce concurrent with the next bounce's closest hits
  waves                          waves in flight (stream lanes, 1-4)
  lane_stagger                   bounces a lane's first wave shades before the next lane's starts
  graph                          captured CUDA graphs of the bounce loop, or direct launches
  guided_form                    guided bounce as a bounce kernel + network pass, or one fused kernel
                                 (searched for guided workloads only)
  shade_occupancy                blocks per SM the shading kernels are compiled to fit (registers)
  shared_stack                   BLAS stack entries per thread kept in shared memory (1: none, 16)
  pixel_order                    camera rays in scanline order or in 8x4 pixel tiles per warp
  refill                         idle lanes that trigger a warp refill
  extend/shadow/shade_blocks_per_sm   blocks per SM in the grids (persistent kernels: at most
                                      those resident at once)
  wave_paths                     paths in flight per wave (queue capacity)

Results are stored as JSON under xenon_b200/tuning/<gpu>/<workload>.json and loaded by
load_tuning(); the renderer's image does not depend on any of these settings.
"""
from __future__ import annotations

import json
import os
import time

HERE = os.path.dirname(os.path.abspath(__file__))
TUNING_DIR = os.path.join(HERE, "tuning")

SPACE = {
    # no 0: a zero field keeps the current value (the xb_tuning convention)
    "extend_persistent_from_depth": [1, 2, 3, 64],
    "shadow_persistent": [1, 2],
    "shadow_order": [1, 2],
    "overlap": [1, 2],
    "waves": [1, 2, 3, 4],
    "lane_stagger": [1, 2, 3],
    "graph": [1, 2],
    "guided_form": [1, 2],
    "shade_occupancy": [4, 8, 12, 16],
    "shared_stack": [1, 16],
    "pixel_order": [1, 2],
    "refill": [2, 4, 8, 16, 24],
    "extend_blocks_per_sm": [2, 4, 8, 16, 64],
    "shadow_blocks_per_sm": [2, 4, 8, 16, 64],
    "shade_blocks_per_sm": [2, 4, 8, 16, 64],
    "wave_paths": [1 << 20, 1 << 21, 1 << 22],
}


def gpu_name() -> str:
    try:
        import torch
        return torch.cuda.get_device_name(0).replace(" ", "_")
    except Exception:
        return "unknown_gpu"


def tuning_path(workload: str, gpu: str | None = None) -> str:
    return os.path.join(TUNING_DIR, gpu or gpu_name(), f"{workload}.json")


def load_tuning(workload: str, gpu: str | None = None) -> dict | None:
    p = tuning_path(workload, gpu)
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)["tuning"]
    return None


def measure(renderer, cam, calls: int, spp_per_call: int, first: int) -> float:
    """Device ms per sample over `calls` xb_render calls of `spp_per_call` samples each (after
    one warm-up call); several waves per call, so waves in flight are measured as used."""
    renderer.render_range(cam, first, spp_per_call)
    ms = 0.0
    for k in range(calls):
        renderer.render_range(cam, first + (1 + k) * spp_per_call, spp_per_call)
        ms += renderer.stats().last_ms
    return ms / (calls * spp_per_call)


# Knobs that only guided bounces read: a plain workload leaves them as they are (any gain they
# showed there would be noise, and a plain tuning also serves guided views of the same scene).
GUIDED_ONLY = ("guided_form",)


def autotune(renderer, cam, workload: str, calls: int = 3, spp_per_call: int = 8, passes: int = 2,
             save: bool = True, log=print, guided: bool = False) -> dict:
    best = dict(renderer.tuning())
    seq = [1000]

    def run(t):
        renderer.set_tuning(**t)
        seq[0] += (calls + 1) * spp_per_call
        return measure(renderer, cam, calls, spp_per_call, seq[0])

    best_ms = run(best)
    log(f"start {best_ms:.3f} ms/spp {best}")
    for _ in range(passes):
        for key, values in SPACE.items():
            if key in GUIDED_ONLY and not guided:
                continue
            for v in values:
                if best.get(key) == v:
                    continue
                cand = dict(best)
                cand[key] = v
                ms = run(cand)
                if ms < best_ms * 0.995:
                    best, best_ms = cand, ms
                    log(f"  {key}={v}: {ms:.3f} ms/spp (new best)")
    renderer.set_tuning(**best)
    result = {"workload": workload, "gpu": gpu_name(), "ms_per_spp": best_ms, "tuning": best,
              "when": time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime())}
    if save:
        p = tuning_path(workload)
        os.makedirs(os.path.dirname(p), exist_ok=True)
        with open(p, "w") as f:
            json.dump(result, f, indent=1)
    return result


if __name__ == "__main__":
    import argparse
    import sys
    sys.path.insert(0, os.path.dirname(HERE))
    import xenon_b200 as xb
    from xenon_b200 import scenes
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="config2")
    ap.add_argument("--out", default=None, help="also write the result JSON here")
    ap.add_argument("--calls", type=int, default=3, help="xb_render calls per measurement")
    ap.add_argument("--spp-per-call", type=int, default=8, help="samples per xb_render call")
    ap.add_argument("--from-saved", action="store_true", help="start from the stored tuning")
    a = ap.parse_args()
    if a.workload == "config2":
        desc = scenes.icosphere_scene(level=8)
    elif a.workload == "config1":
        desc = scenes.cornell()
    elif a.workload in ("config4", "config4g"):
        desc = scenes.guiding_room()
    else:
        desc = scenes.instanced_grid()
    hs = xb.HostScene.from_desc(desc)
    r = xb.Renderer(desc.width, desc.height, desc.max_bounces, desc.min_bounces)
    r.upload_scene(hs)
    cam = xb.camera(desc.eye, desc.target, desc.fov, desc.width / desc.height)
    if a.from_saved and load_tuning(a.workload):
        r.set_tuning(**load_tuning(a.workload))
    if a.workload == "config4g":
        # guided rendering with a network trained on the first 64 samples, then held fixed
        r.set_guiding(True, train_spp=64, steps_per_spp=32, keep_training_samples=2)
        r.render_frame(cam, 64)
        r.set_guiding(True, train_spp=-1)
    res = autotune(r, cam, a.workload, calls=a.calls, spp_per_call=a.spp_per_call, guided=a.workload == "config4g")
    print(json.dumps(res))
    if a.out:
        with open(a.out, "w") as f:
            json.dump(res, f, indent=1)
