#!/usr/bin/env python3
"""Benchmark: Mrays/s of the plain GPU wavefront on config 2 (1 x B200 per rank).

Workload (config 2): icosphere level 8 (1,310,720 triangles) displaced by 4-octave value noise
of amplitude 0.15 r, GGX conductor roughness 0.3, 50x50 ground quad, sun 3.0 + gradient sky,
1920x1080, max depth 10, Russian roulette from bounce 3; synthetic, seed 1. One step = one
sample of every pixel (2,073,600 paths: camera rays, bounce rays and NEE shadow rays).

  value        rays traced (closest + shadow) / device time of the K timed steps (CUDA events on
               the renderer's stream), summed over ranks / max over ranks
  e2e          the same metric through the public C ABI with host buffers: xb_render +
               xb_resolve_async into pinned host memory every step (the framebuffer hand-off
               CudaRenderer does per sample; the read-back of sample k overlaps sample k+1), then
               xb_sync; host wall clock
  roofline     the closest-hit traversal kernel (extend): algorithmic bytes per launch ÷ its
               average launch time (CUDA events around each launch), against measured HBM GB/s
  cpu_baseline the reference's own CPU backend (render_frame_tiled, Release flags, all host
               threads) on a bounded sample of the same view; its Mrays/s uses the rays per path
               this GPU run measured (the reference counts no rays)

Studies at the end of the line (their full results with --detail-out): bvh_build (config 2's
BVH built on the host and on the device), config3 (throughput of config 3), incoherent (traversal alone on 2^22 incoherent and 2^22 bounce-2 rays, config 2 and 3),
views (config 5), sky_is (sky importance sampling at equal time) and guiding (config 4, equal-time
relMSE of guided vs plain: the second half of the metric).

Multi-GPU (torchrun): each rank renders its own sample indices (rank r renders samples
r*K+1 ...), so per-GPU work is fixed (weak scaling); the only exchange is one NCCL reduce of
the framebuffer after the timed region.

--impl reference times the reference's CPU implementation of this path on the host cores
(oracle/_ref: render_frame_tiled with its Release flags, every host thread, about one second of
samples per step on 1/64 of the view's pixels); its process loads no library of this package,
and its `config` is this arm's.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mrays/s; equal-time relMSE, guided vs plain GPU wavefront (1×B200)"


def workload(desc, level: int) -> str:
    """The workload's name with its actual sizes (config 2 at the defaults: level 8,
    1,310,722 triangles with the ground, 1920x1080, depth 10)."""
    return (f"config2: displaced icosphere L{level} ({desc.num_triangles:,} tris incl. ground) "
            f"{desc.width}x{desc.height}, depth {desc.max_bounces}")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--level", type=int, default=8, help="icosphere subdivision level (8 = config 2)")
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--spp-per-step", type=int, default=8,
                    help="samples per pixel rendered by one xb_render call (one step)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--thread-per-ray", action="store_true", help="one-ray-per-thread traversal kernels")
    ap.add_argument("--no-guiding-study", action="store_true", help="skip the config-4 guided vs plain study")
    ap.add_argument("--no-views-study", action="store_true", help="skip the config-5 many-views study")
    ap.add_argument("--no-config3", action="store_true", help="skip the config-3 throughput entry")
    ap.add_argument("--views-max-spp", type=int, default=64, help="config 5: cap on a view's spp (0: none)")
    ap.add_argument("--guide-seconds", type=float, default=6.0, help="equal device-time budget per method")
    ap.add_argument("--guide-ref-spp", type=int, default=16384, help="samples of the plain FP64 reference")
    ap.add_argument("--guide-train-spp", type=int, default=64, help="config 4: trained on the first 64 spp")
    ap.add_argument("--guide-steps-per-spp", type=int, default=32)
    ap.add_argument("--guide-fraction", type=float, default=0.0,
                    help="fixed probability of sampling the network (0: learned per vertex)")
    ap.add_argument("--guide-ratio-cap", type=float, default=0.0,
                    help="bound on a path's importance ratio (xb_guiding.ratio_cap; 0: the library's default)")
    ap.add_argument("--guide-first", type=int, default=0,
                    help="config 4: first sample index after the first train_spp samples (0: continuous)")
    ap.add_argument("--guide-blocks", default="0,1048576,2097152",
                    help="config 4: renders per method, each from its own block of sample indices "
                         "(--guide-first values, comma-separated; empty: --guide-first alone)")
    ap.add_argument("--guide-ref-cache", default="", help="config 4: load (or save) the FP64 reference here")
    ap.add_argument("--guide-width", type=int, default=1280)
    ap.add_argument("--no-incoherent", action="store_true", help="skip the incoherent-ray traversal bench")
    ap.add_argument("--no-sky-study", action="store_true", help="skip the sky importance sampling study")
    ap.add_argument("--no-build-study", action="store_true", help="skip the BVH build timing")
    ap.add_argument("--sky-seconds", type=float, default=2.0, help="sky study: device time per method")
    ap.add_argument("--incoherent-rays", type=int, default=1 << 22)
    ap.add_argument("--detail-out", default="", help="also write the studies' full results to this JSON file")
    ap.add_argument("--guide-height", type=int, default=720)
    return ap.parse_args()


def load_peaks() -> dict:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return {"hbm_gbs": d["hbm_gbs"], "bf16_tflops": d["bf16_tflops"], "source": "measured"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "source": "fallback"}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[5 + i].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def dist_setup(n_gpus: int):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return ws, rank, local


def allreduce_max(x: float, ws: int) -> float:
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def allreduce_sum(x: float, ws: int) -> float:
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t)
    return float(t.item())


def barrier(ws: int):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


class quiet_stdout:
    """Silences file descriptor 1 (the reference's C++ printf) so that stdout carries only the
    JSON line."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        self.null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self.null, 1)
        return self

    def __exit__(self, *a):
        sys.stdout.flush()
        os.dup2(self.saved, 1)
        os.close(self.saved)
        os.close(self.null)


def shared_config(desc, level: int) -> dict:
    """The workload, identical in the JSON lines of both arms (this one and --impl reference)."""
    return {"workload": workload(desc, level), "scene": "config 2 (synthetic, seed 1)",
            "width": desc.width, "height": desc.height, "min_bounces": desc.min_bounces,
            "max_bounces": desc.max_bounces, "triangles": desc.num_triangles,
            "l2": "GPU arm: 256 MiB written between timed steps (L2 flushed); CPU arm: not applicable"}


def cpu_reference_run(desc, steps: int, warmup: int, step_seconds: float) -> dict:
    """The reference's CPU backend (render_frame_tiled from oracle/_ref, Release flags, every
    host thread) on 1/64 of the view's pixels (the same camera): `warmup` untimed and `steps`
    timed calls, each of the samples per pixel that fill about `step_seconds` (at most 256), so
    that thread-pool start-up is a small part of each call. Loads no library of this package."""
    from oracle import ref
    L = ref.lib("fast")
    cores = int(L.xr_hardware_threads())
    w, h = desc.width // 8, desc.height // 8
    rs = ref.RefScene(desc, flavour="fast")
    rr = ref.RefRenderer(w, h, desc.min_bounces, desc.max_bounces, flavour="fast")
    _, t1 = rr.render(rs, desc.eye, desc.target, desc.fov, 1, 4)
    spp = int(max(1, min(256, step_seconds / max(t1 / 4, 1e-4))))
    first = 100
    for s in range(warmup):
        rr.render(rs, desc.eye, desc.target, desc.fov, first, spp)
        first += spp
    secs = 0.0
    for s in range(steps):
        _, t = rr.render(rs, desc.eye, desc.target, desc.fov, first, spp)
        first += spp
        secs += t
    msps = w * h * spp * steps / secs / 1e6
    return {"cores": cores, "msamples_per_s": msps, "seconds": secs, "spp_per_step": spp,
            "ms_per_step": secs * 1e3 / steps, "pixels": (w, h), "scene": rs,
            "sample": f"{w}x{h} px (1/64 of the pixels, same camera) x {spp} spp per call, "
                      f"render_frame_tiled with Release flags on {cores} threads"}


def rays_per_path_oracle(desc, rs) -> float:
    """Rays per path of this estimator (closest + shadow), counted by the CPU restatement
    (oracle/port.py) on the reference-built scene `rs` and the reference's camera: the
    reference counts no rays, so its Mrays/s is derived from this count."""
    from oracle import port, ref
    cam = ref.camera(desc.eye, desc.target, desc.fov, desc.width / desc.height)
    return port.rays_per_path(rs.view(), cam, desc.width, desc.height, desc.min_bounces, desc.max_bounces)


def cpu_reference_sample(desc, rays_per_path: float, budget_s: float) -> dict:
    """cpu_baseline of this arm: the reference CPU backend for about budget_s seconds; its
    Mrays/s uses the rays per path this GPU run measured."""
    from oracle import ref
    if not ref.available("fast"):
        return {"value": None, "unit": "Mrays/s", "cores": None, "kind": "reference",
                "sample": "oracle/_ref/libxnref_fast.so not built"}
    run = cpu_reference_run(desc, steps=3, warmup=0, step_seconds=budget_s / 3)
    return {"value": run["msamples_per_s"] * rays_per_path, "unit": "Mrays/s", "cores": run["cores"],
            "kind": "reference", "msamples_per_s": run["msamples_per_s"], "seconds": run["seconds"],
            "sample": run["sample"] + "; Mrays/s = Msamples/s x rays per path measured on the GPU "
                                      "for this config (derived: the reference counts no rays)"}


def run_reference(args):
    """--impl reference: the reference's own CPU implementation of the path, host threads."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    with quiet_stdout():
        line = reference_line(args)
    print(json.dumps(line))
    return 0


def reference_line(args) -> dict:
    from oracle import ref
    from xenon_b200 import scenes
    desc = scenes.icosphere_scene(level=args.level, width=args.width, height=args.height)
    if not ref.available("fast"):
        return {"impl": "reference", "unavailable": "oracle/_ref/libxnref_fast.so was not built"}
    # each step about 1 s of CPU work (less when many steps are asked for), whole run within minutes
    step_s = min(1.0, 150.0 / max(args.steps + args.warmup, 1))
    run = cpu_reference_run(desc, args.steps, args.warmup, step_s)
    rpp = rays_per_path_oracle(desc, run["scene"])
    msps = run["msamples_per_s"]
    value = msps * rpp
    unit = "Mrays/s"
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": unit, "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": run["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded procedural scene, seed 1)",
            "config": shared_config(desc, args.level),
            "cpu_baseline": {"value": value, "unit": unit, "cores": run["cores"], "kind": "reference",
                             "sample": run["sample"] + " per step"},
            "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "detail": {"msamples_per_s": msps, "rays_per_path": rpp,
                       "rays_per_path_source": "oracle/ restatement on the reference-built scene (derived: "
                                               "the reference counts no rays)",
                       "spp_per_step": run["spp_per_step"], "pixels": run["pixels"]}}
    return line


def guiding_study(args, device: int) -> dict:
    """Config 4: equal device-time relMSE of the guided and the plain wavefront against a plain
    FP64 reference of 16k samples. Both methods render in chunks of samples until their summed
    device time (CUDA events of each xb_render call) reaches the budget; the guided budget
    includes its online training on the first train_spp samples, of which the second half
    (rendered once half of the Adam steps are taken) is part of its image. Each method renders
    --guide-blocks times, the samples after training drawn from disjoint blocks of sample
    indices; the ratios are of the relMSE pooled over those renders (and per render)."""
    import xenon_b200 as xb
    from xenon_b200 import scenes
    W, H = args.guide_width, args.guide_height
    desc = scenes.guiding_room(width=W, height=H)
    hs = xb.HostScene.from_desc(desc)
    cam = xb.camera(desc.eye, desc.target, desc.fov, W / H)
    eps = 1e-2

    from xenon_b200 import autotune
    # each method with the launch settings the autotuner picked for it on this workload
    full = (W, H) == (1280, 720)
    tuned = autotune.load_tuning("config4") if full else None
    tuned_g = (autotune.load_tuning("config4g") or tuned) if full else None

    def renderer(fp64=False, guided=False):
        r = xb.Renderer(W, H, desc.max_bounces, desc.min_bounces, device=device, fp64=fp64)
        r.upload_scene(hs)
        t = tuned_g if guided else tuned
        if t:
            r.set_tuning(**t)
        return r

    t0 = time.perf_counter()
    ref_first = 1 << 24            # sample indices disjoint from the compared renders (1, 2, ...)
    if args.guide_ref_cache and os.path.exists(args.guide_ref_cache):
        z = np.load(args.guide_ref_cache)
        ref, ref_var, done, ref_ms = z["ref"], z["var"], int(z["spp"]), float(z["ms"])
    else:
        rr = renderer(fp64=True)
        ref_ms = 0.0
        done = 0
        while done < args.guide_ref_spp:
            n = min(256, args.guide_ref_spp - done)
            rr.render_range(cam, ref_first + done, n)
            ref_ms += rr.stats().last_ms
            done += n
        s64, m2 = rr.resolve_fp64()
        ref = s64 / done
        ref_var = m2 / max(done - 1, 1)
        rr.close()
        if args.guide_ref_cache:
            np.savez(args.guide_ref_cache, ref=ref, var=ref_var, spp=done, ms=ref_ms)
    denom = ref ** 2 + eps
    ref_err = float(np.mean(ref_var / done / denom))   # the reference's own expected relMSE

    def equal_time(guided: bool, first: int) -> dict:
        r = renderer(guided=guided)
        info = {}
        if guided:
            fixed = args.guide_fraction > 0
            r.set_guiding(True, train_spp=args.guide_train_spp, steps_per_spp=args.guide_steps_per_spp,
                          batch=16384, guide_fraction=args.guide_fraction if fixed else 0.7,
                          fixed_fraction=1 if fixed else 0, keep_training_samples=2,
                          ratio_cap=args.guide_ratio_cap)
        ms, rendered, chunk = 0.0, 0, 8
        ntrain = args.guide_train_spp
        while ms < args.guide_seconds * 1e3:
            # samples 1..train_spp (the guided render's training samples), then samples from
            # --guide-first on (default: train_spp + 1, one continuous sequence)
            if first and rendered >= ntrain:
                r.render_range(cam, first + rendered - ntrain, chunk)
            else:
                r.render_range(cam, 1 + rendered, chunk)
            ms += r.stats().last_ms
            rendered += chunk
            if guided and rendered == args.guide_train_spp:
                info["train_phase_ms"] = ms
        spp = r.spp                              # image samples (the first half of training excluded)
        img = r.resolve().astype(np.float64)
        if guided:
            info.update(r.guiding_stats())
            info["config"] = {k: v for k, v in r.guiding().items() if k in
                              ("train_spp", "steps_per_spp", "batch", "learning_rate", "guide_fraction",
                               "fixed_fraction", "keep_training_samples", "ratio_cap")}
        r.close()
        e = (img - ref) ** 2 / denom
        pix = e.mean(2).ravel()
        trimmed = np.sort(pix)[: int(len(pix) * 0.999)]
        worst = np.argsort(pix)[-5:][::-1]
        info["worst_pixels"] = [{"pixel": int(i), "relmse": float(pix[i]), "value": float(img.reshape(-1, 3)[i].mean()),
                                 "reference": float(ref.reshape(-1, 3)[i].mean())} for i in worst]
        info["pixels_relmse_over_1"] = int((pix > 1.0).sum())
        return {"spp": spp, "samples_rendered": rendered, "device_ms": ms, "relmse": float(pix.mean()),
                "relmse_minus_reference_noise": float(pix.mean()) - ref_err,
                "relmse_trimmed_0.1pct": float(trimmed.mean()), "image_mean": float(img.mean()), **info}

    # Several independent renders per method (disjoint blocks of sample indices after the
    # training samples): the room's caustics make single renders' relMSE a lottery of a few
    # bright samples, so the ratios are reported per block and pooled over the blocks.
    blocks = [int(b) for b in args.guide_blocks.split(",")] if args.guide_blocks else [args.guide_first]
    per_block = []
    for first in blocks:
        plain = equal_time(False, first)
        guided = equal_time(True, first)
        per_block.append({"first": first, "plain": plain, "guided": guided,
                          "ratio_raw": plain["relmse"] / max(guided["relmse"], 1e-30),
                          "ratio_trimmed": plain["relmse_trimmed_0.1pct"] / max(guided["relmse_trimmed_0.1pct"], 1e-30)})

    def pooled(key, method):
        return float(np.mean([b[method][key] for b in per_block]))
    pool = {k: {m: pooled(k, m) for m in ("plain", "guided")}
            for k in ("relmse", "relmse_minus_reference_noise", "relmse_trimmed_0.1pct")}
    return {"workload": "config4: closed room, light above a baffle, smooth glass geodesic sphere "
                        f"({desc.meshes[-1].indices.shape[0]:,} tris), {W}x{H}, depth 16",
            "tuning": {"plain": tuned or "defaults", "guided": tuned_g or "defaults"},
            "budget_device_s": args.guide_seconds, "reference": {"spp": done, "device_ms": ref_ms,
                                                               "image_mean": float(ref.mean()),
                                                               "expected_relmse": ref_err},
            "blocks": per_block,
            # the first block's renders (samples 1, 2, ...: the continuous sequence) as before
            "plain": per_block[0]["plain"], "guided": per_block[0]["guided"],
            "pooled": pool,
            "relmse_ratio_plain_over_guided": pool["relmse"]["plain"] / max(pool["relmse"]["guided"], 1e-30),
            "relmse_ratio_reference_noise_removed": pool["relmse_minus_reference_noise"]["plain"] /
                max(pool["relmse_minus_reference_noise"]["guided"], 1e-30),
            "relmse_ratio_trimmed": pool["relmse_trimmed_0.1pct"]["plain"] / max(pool["relmse_trimmed_0.1pct"]["guided"], 1e-30),
            "wall_s": time.perf_counter() - t0}


def sky_study(args, device: int) -> dict:
    """Sky importance sampling (XB_FLAG_SKY_IS) against the default estimator on config 2's view
    at 960x540: equal device time (--sky-seconds per method, CUDA events of each xb_render call),
    each image's relMSE against a plain FP64 render of 4096 samples at disjoint sample indices."""
    import xenon_b200 as xb
    from xenon_b200 import abi, autotune, scenes
    W, H = args.width // 2, args.height // 2
    desc = scenes.icosphere_scene(level=args.level, width=W, height=H)
    hs = xb.HostScene.from_desc(desc)
    cam = xb.camera(desc.eye, desc.target, desc.fov, W / H)
    tuned = autotune.load_tuning("config2")

    def renderer(flags=0, fp64=False):
        r = xb.Renderer(W, H, desc.max_bounces, desc.min_bounces, device=device, fp64=fp64, flags=flags)
        r.upload_scene(hs)
        if tuned:
            r.set_tuning(**tuned)
        return r

    rr = renderer(fp64=True)
    ref_spp = 4096
    for first in range(0, ref_spp, 512):
        rr.render_range(cam, (1 << 24) + first, 512)
    s64, _ = rr.resolve_fp64()
    ref = s64 / ref_spp
    rr.close()
    denom = ref ** 2 + 1e-2

    def equal_time(flags):
        r = renderer(flags)
        r.render_range(cam, 1 << 23, 8)          # warm-up (graphs, queues), not in the image
        r.reset()
        ms, n = 0.0, 0
        while ms < args.sky_seconds * 1e3:
            r.render_frame(cam, 8)
            ms += r.stats().last_ms
            n += 8
        img = r.resolve().astype(np.float64)
        r.close()
        e = np.sort(((img - ref) ** 2 / denom).mean(2).ravel())
        return {"spp": n, "device_ms": ms, "relmse": float(e.mean()),
                "relmse_trimmed": float(e[: int(len(e) * 0.999)].mean()), "image_mean": float(img.mean())}

    plain = equal_time(0)
    sky = equal_time(abi.XB_FLAG_SKY_IS)
    return {"workload": f"config2 view {W}x{H}, depth {desc.max_bounces}", "reference_spp": ref_spp,
            "plain": plain, "sky_is": sky, "ratio_raw": plain["relmse"] / max(sky["relmse"], 1e-30),
            "ratio_trimmed": plain["relmse_trimmed"] / max(sky["relmse_trimmed"], 1e-30),
            "mean_reference": float(ref.mean())}


def build_study(args) -> dict:
    """BVH build and refit of config 2's scene (1,310,722 triangles, binned SAH as the reference builds it):
    wall time of xb_scene_build (the BLAS, the TLAS and the flattened arrays; the mesh already
    added) with the recursive host build on one thread and on every host thread, and with the
    level-synchronous build on the device (XB_BUILD_DEVICE, host-to-device copy of the build items
    and the read-back of the nodes included); all three give the same node arrays (GPU tests).
    Median of three builds each, after one untimed device build."""
    import xenon_b200 as xb
    from xenon_b200 import abi, scenes
    desc = scenes.icosphere_scene(level=args.level)

    def timed(**kw):
        t = []
        for _ in range(3):
            s = xb.HostScene.from_desc(desc, build=False)
            t0 = time.perf_counter()
            s.build(**kw)
            t.append(time.perf_counter() - t0)
        return float(np.median(t))

    xb.HostScene.from_desc(desc, build_mode=abi.XB_BUILD_DEVICE)
    out = {"triangles": desc.num_triangles, "host_1_thread_s": timed(build_threads=1),
           "host_all_threads_s": timed(build_threads=0), "device_s": timed(build_mode=abi.XB_BUILD_DEVICE),
           "host_threads": os.cpu_count()}
    # refit of the displaced sphere's BLAS after its vertices moved (topology kept): on the device
    # (xb_refit_mesh: positions copied in, three refit passes, TLAS rebuilt) against the host refit
    # (xb_scene_refit_mesh) and a new upload; median of three after one untimed call each
    hs = xb.HostScene.from_desc(desc)
    m = int(np.argmax([len(mm.positions) for mm in desc.meshes]))
    pos = np.asarray(desc.meshes[m].positions, np.float32)
    moved = [(pos * np.float32(1.0 + 0.01 * k)).astype(np.float32) for k in range(1, 5)]
    r = xb.Renderer(64, 64)
    r.upload_scene(hs)

    def med(fn):
        fn(moved[0])
        t = []
        for p in moved[1:]:
            t0 = time.perf_counter()
            fn(p)
            t.append(time.perf_counter() - t0)
        return float(np.median(t))

    out["refit_vertices"] = int(len(pos))
    out["refit_device_s"] = med(lambda p: r.refit_mesh(m, p))

    def host_refit(p):
        hs.refit_mesh(m, p)
        r.upload_scene(hs)
    out["refit_host_and_upload_s"] = med(host_refit)
    r.close()
    return out


def config3_study(args, device: int) -> dict:
    """Config 3: TLAS over 16x16 instances of 4 seeded meshes (random materials), sky + 4 quad
    lights, 1920x1080, depth 12, with its autotuned launch settings; device Mrays/s and
    Msamples/s over a few steps of 4 samples, L2 flushed between steps. The config's 512 spp are
    this step repeated; its time per sample is what the steps measure."""
    import torch
    import xenon_b200 as xb
    from xenon_b200 import autotune, scenes
    desc = scenes.instanced_grid()
    hs = xb.HostScene.from_desc(desc)
    r = xb.Renderer(desc.width, desc.height, desc.max_bounces, desc.min_bounces, device=device)
    r.upload_scene(hs)
    tuned = autotune.load_tuning("config3")
    if tuned:
        r.set_tuning(**tuned)
    cam = xb.camera(desc.eye, desc.target, desc.fov, desc.width / desc.height)
    sps, steps = 8, 4
    for s in range(2):
        r.render_range(cam, 1 + s * sps, sps)
    r.reset()
    r.reset_stats()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    ms = 0.0
    for s in range(steps):
        flush.zero_()
        torch.cuda.synchronize()
        r.render_range(cam, 1 + (2 + s) * sps, sps)
        ms += r.stats().last_ms
    st = r.stats()
    r.close()
    return {"workload": "config3: 16x16 instances of 4 meshes (82k-328k tris), 1920x1080, depth 12, sky + 4 quads",
            "spp_per_step": sps, "steps": steps, "ms_per_spp": ms / (steps * sps),
            "mrays_per_s": (st.rays_closest + st.rays_shadow) / ms / 1e3,
            "msamples_per_s": st.paths / ms / 1e3, "tuning": tuned or "defaults",
            "l2": "flushed between steps"}


def views_study(args, device: int) -> dict:
    """Config 5: 32 seeded views of the config-3 instanced scene (side log-uniform 256-1024 px,
    spp from {16, 64, 256, 1024} capped at --views-max-spp, bounce limit 6-16) in one
    xb_render_views call with guiding on — one network, trained on the scene's own view
    (64 spp), serves every view — then per-view relMSE of those images against plain renders of
    the same views with 4x the samples. For context: the same views plain, batched and one by one."""
    import xenon_b200 as xb
    from xenon_b200 import scenes
    desc = scenes.instanced_grid()
    hs = xb.HostScene.from_desc(desc)
    specs = scenes.config5_views(desc, 32, seed=1, max_spp=args.views_max_spp)
    cams = [xb.camera(e, t, f, w / h) for (e, t, f, w, h, _, _) in specs]
    views = [(c, w, h, spp, mb) for c, (_, _, _, w, h, spp, mb) in zip(cams, specs)]
    paths = sum(w * h * spp for (_, w, h, spp, _) in views)
    maxb = max(mb for (*_, mb) in views)

    from xenon_b200 import autotune
    tuned = autotune.load_tuning("config3")

    def renderer(w=512, h=512):
        r = xb.Renderer(w, h, maxb, desc.min_bounces, device=device)
        r.upload_scene(hs)
        if tuned:
            r.set_tuning(**tuned)
        return r

    # plain: batched vs one by one, and the 4x reference
    r = renderer()
    r.render_views(views[:2])
    r.reset_stats()
    plain_imgs = r.render_views(views)
    plain_ms = r.stats().last_ms
    r.close()
    seq_ms = 0.0
    refs = []
    for (c, w, h, spp, mb) in views:
        rr = renderer(w, h)
        rr.set_bounces(desc.min_bounces, mb)
        rr.render_frame(c, 1)
        rr.reset()
        rr.render_frame(c, spp)
        seq_ms += rr.stats().last_ms
        # the reference: 4x the samples at indices no timed render uses
        rr.reset()
        rr.render_range(c, 1 << 24, 4 * spp)
        refs.append(rr.resolve())
        rr.close()
    # guided: one shared network, trained on the scene's own view
    g = renderer(desc.width, desc.height)
    g.set_guiding(True, train_spp=64, steps_per_spp=32)
    main_cam = xb.camera(desc.eye, desc.target, desc.fov, desc.width / desc.height)
    g.render_frame(main_cam, 64)
    train_ms = g.stats().last_ms
    g.reset_stats()
    guided_imgs = g.render_views(views)
    guided_ms = g.stats().last_ms
    # aggregate throughput at the configuration's own spp draws ({16, 64, 256, 1024}, no cap):
    # the same 32 views, plain and guided (the trained network), each in one xb_render_views call
    full = None
    if args.views_max_spp:
        fspecs = scenes.config5_views(desc, 32, seed=1, max_spp=0)
        fviews = [(c, w, h, spp, mb) for c, (_, _, _, w, h, spp, mb) in zip(cams, fspecs)]
        fpaths = sum(w * h * spp for (_, w, h, spp, _) in fviews)
        g.reset_stats()
        g.render_views(fviews)
        fg_ms = g.stats().last_ms
        rp = renderer()
        rp.reset_stats()
        rp.render_views(fviews)
        fp_ms = rp.stats().last_ms
        rp.close()
        full = {"paths": fpaths, "spp": [v[3] for v in fviews], "plain_batched_msamples_per_s": fpaths / fp_ms / 1e3,
                "guided_msamples_per_s": fpaths / fg_ms / 1e3, "plain_ms": fp_ms, "guided_ms": fg_ms}
    g.close()

    def relmse(img, ref):
        """Per-pixel relative squared error, channel mean: (raw mean, mean without the 0.1% largest
        pixels). Caustic paths (light through the glass instances) leave a few pixels per view
        thousands of times brighter than their mean in plain and guided renders alike; the raw
        mean follows those few pixels, the trimmed one the rest of the image."""
        img, ref = img.astype(np.float64), ref.astype(np.float64)
        e = np.sort(((img - ref) ** 2 / (ref ** 2 + 1e-2)).mean(axis=2).ravel())
        k = max(1, e.size // 1000)
        return float(e.mean()), float(e[:-k].mean())
    per_view = []
    for (c, w, h, spp, mb), gi, pi, rf in zip(views, guided_imgs, plain_imgs, refs):
        (g_raw, g_trim), (p_raw, p_trim) = relmse(gi, rf), relmse(pi, rf)
        per_view.append({"size": w, "spp": spp, "max_bounces": mb, "relmse_guided": g_raw, "relmse_plain": p_raw,
                         "relmse_guided_trimmed": g_trim, "relmse_plain_trimmed": p_trim})
    raw = [v["relmse_plain"] / max(v["relmse_guided"], 1e-30) for v in per_view]
    trim = [v["relmse_plain_trimmed"] / max(v["relmse_guided_trimmed"], 1e-30) for v in per_view]
    speed = plain_ms / guided_ms   # relMSE falls as 1/samples: equal time scales the ratio by it
    return {"workload": "config5: 32 views of config 3 (16x16 instances), side 256-1024 px log-uniform, "
                        f"spp from {{16,64,256,1024}} capped at {args.views_max_spp}, depth 6-16",
            "tuning": tuned or "defaults",
            "paths": paths, "guided_msamples_per_s": paths / guided_ms / 1e3, "guided_ms": guided_ms,
            "guide_training_ms": train_ms, "plain_batched_msamples_per_s": paths / plain_ms / 1e3,
            "plain_one_by_one_msamples_per_s": paths / seq_ms / 1e3,
            "relmse_ratio_plain_over_guided_median": float(np.median(raw)),
            "relmse_ratio_plain_over_guided_median_trimmed": float(np.median(trim)),
            "relmse_ratio_equal_time_median_trimmed": float(np.median(trim)) * speed,
            "full_spp": full,
            "relmse": "mean over pixels of (x - ref)^2 / (ref^2 + 0.01); trimmed: without the 0.1% largest pixels",
            "reference": "plain renders of the same views with 4x the samples", "per_view": per_view}


def _sig(x, digits: int = 4):
    """x rounded to `digits` significant digits (keeps the JSON line short)."""
    if not isinstance(x, float) or x == 0.0 or not np.isfinite(x):
        return x
    return float(f"{x:.{digits}g}")


def config3_summary(c):
    if not c or "error" in c:
        return c
    return {"workload": "config3", "mrays_per_s": _sig(c["mrays_per_s"]), "msamples_per_s": _sig(c["msamples_per_s"]),
            "ms_per_spp": _sig(c["ms_per_spp"])}


def incoherent_summary(inc):
    """Mrays/s per scene and batch in the JSON line (the full figures go to --detail-out)."""
    if not inc or "error" in inc:
        return inc
    out = {"rays": inc["rays_per_batch"]}
    for sc in ("config2", "config3"):
        out[sc] = {k: _sig(v["mrays_per_s"]) for k, v in inc[sc].items()}
    return out


def sky_summary(k):
    if not k or "error" in k:
        return k
    return {"ratio_raw": _sig(k["ratio_raw"]), "ratio_trimmed": _sig(k["ratio_trimmed"]),
            "spp_plain": k["plain"]["spp"], "spp_sky": k["sky_is"]["spp"]}


def views_summary(v):
    """The config-5 figures kept in the JSON line (the per-view list goes to --detail-out)."""
    if not v or "error" in v:
        return v
    keep = ("guided_msamples_per_s", "plain_batched_msamples_per_s", "plain_one_by_one_msamples_per_s",
            "relmse_ratio_plain_over_guided_median", "relmse_ratio_plain_over_guided_median_trimmed",
            "relmse_ratio_equal_time_median_trimmed")
    out = {"workload": "config5: 32 views of config 3", **{k: _sig(v[k]) for k in keep}}
    if v.get("full_spp"):
        out["full_spp_plain_msamples_per_s"] = _sig(v["full_spp"]["plain_batched_msamples_per_s"])
        out["full_spp_guided_msamples_per_s"] = _sig(v["full_spp"]["guided_msamples_per_s"])
    return out


def guiding_summary(g):
    """The config-4 figures kept in the JSON line: equal-time relMSE of plain and guided against
    the 16k-spp FP64 reference, their ratios, and what each method rendered in the budget."""
    if not g or "error" in g:
        return g
    p, q = g["plain"], g["guided"]
    out = {"workload": "config4 (" + g["workload"].split("(")[1].split(")")[0] + " sphere)",
           "budget_device_s": g["budget_device_s"], "reference_spp": g["reference"]["spp"],
           "ratio_raw": _sig(g["relmse_ratio_plain_over_guided"]),
           "ratio_reference_noise_removed": _sig(g["relmse_ratio_reference_noise_removed"]),
           "ratio_trimmed": _sig(g["relmse_ratio_trimmed"])}
    if "blocks" in g:
        out["renders_per_method"] = len(g["blocks"])
        out["ratio_raw_per_render"] = [_sig(b["ratio_raw"], 3) for b in g["blocks"]]
        out["ratio_trimmed_per_render"] = [_sig(b["ratio_trimmed"], 3) for b in g["blocks"]]
        out["relmse_plain"] = _sig(g["pooled"]["relmse"]["plain"])
        out["relmse_guided"] = _sig(g["pooled"]["relmse"]["guided"])
    out.update({"spp_plain": p["spp"], "spp_guided": q["spp"], "train_ms": _sig(q.get("train_phase_ms", 0.0)),
                "mean_plain": _sig(p["image_mean"], 6), "mean_guided": _sig(q["image_mean"], 6),
                "mean_reference": _sig(g["reference"]["image_mean"], 6)})
    return out


def incoherent_study(args, device: int) -> dict:
    """Traversal alone on incoherent rays: 2^22 rays with origins uniform in the scene's world
    bounds and directions uniform on the sphere, and 2^22 secondary rays harvested from bounce 2
    of the path tracer's own sampling (xenon_b200/raybatch.py), traced through
    xb_trace_rays_device (closest hit, then any hit) on config 2 and config 3, with each
    workload's tuning (which picks persistent warps or one ray per thread for each kind of query).
    Device Mrays/s from CUDA events around each launch on the launching stream; inputs and hit
    records (128 MiB + 256 MiB per batch) exceed the L2."""
    import torch
    import xenon_b200 as xb
    from xenon_b200 import abi, autotune, raybatch, scenes
    out = {}
    n = args.incoherent_rays
    for name, make in (("config2", lambda: scenes.icosphere_scene(level=args.level)),
                       ("config3", lambda: scenes.instanced_grid())):
        desc = make()
        hs = xb.HostScene.from_desc(desc)
        r = xb.Renderer(64, 64, desc.max_bounces, desc.min_bounces, device=device)
        r.upload_scene(hs)
        tuned = autotune.load_tuning(name)
        if tuned:   # persistent or one-ray-per-thread queries, as the workload's tuning picks
            r.set_tuning(**tuned)
        view = hs.view()
        cam = xb.camera(desc.eye, desc.target, desc.fov, desc.width / desc.height)
        batches = {"uniform": raybatch.incoherent_rays(view, n, seed=5),
                   "bounce2": raybatch.secondary_rays(r, desc.materials, cam, desc.width, desc.height, n,
                                                      seed=6, bounce=2)}
        res = {}
        # the launches and the events on one explicit stream (handle 0 would mean the renderer's own)
        stream = torch.cuda.Stream()
        for bname, rays in batches.items():
            d_rays = torch.from_numpy(rays.view(np.uint8).reshape(-1)).to("cuda")
            d_hits = torch.empty(len(rays) * abi.HIT_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
            for mode, mname in ((abi.XB_TRACE_CLOSEST, "closest"), (abi.XB_TRACE_ANY, "any")):
                def launch():
                    r.trace_rays_device(d_rays.data_ptr(), len(rays), d_hits.data_ptr(), mode, stream.cuda_stream)
                for _ in range(2):
                    launch()
                r.reset_profile()
                launch()
                torch.cuda.synchronize()
                pr = r.profile()
                if mode == abi.XB_TRACE_CLOSEST:
                    nodes, tris, tl, inst = pr.ext_blas_nodes, pr.ext_tris, pr.ext_tlas_nodes, pr.ext_instances
                else:
                    nodes, tris, tl, inst = pr.sh_blas_nodes, pr.sh_tris, pr.sh_tlas_nodes, pr.sh_instances
                bpr = (64 * nodes + 48 * tris + 32 * tl + 48 * inst) / len(rays) + 32 + 64
                ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
                reps = 5
                ms = 0.0
                for _ in range(reps):
                    torch.cuda.synchronize()
                    ev[0].record(stream)
                    launch()
                    ev[1].record(stream)
                    ev[1].synchronize()
                    ms += ev[0].elapsed_time(ev[1])
                ms /= reps
                hits = d_hits.cpu().numpy().view(abi.HIT_DTYPE)
                res[f"{bname}_{mname}"] = {"mrays_per_s": len(rays) / ms / 1e3, "ms": ms,
                                           "algorithmic_bytes_per_ray": bpr,
                                           "achieved_gbs": bpr * len(rays) / ms / 1e6,
                                           "hit_fraction": float(np.isfinite(hits["t"]).mean()),
                                           "blas_nodes_per_ray": nodes / len(rays), "tris_per_ray": tris / len(rays)}
            del d_rays, d_hits
        r.close()
        out[name] = res
    return {"rays_per_batch": n, "entry": "xb_trace_rays_device (64-byte xb_hit records)", **out}


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    ws, rank, local = dist_setup(args.gpus)
    import torch
    import xenon_b200 as xb
    from xenon_b200 import abi, scenes

    torch.cuda.set_device(local)
    desc = scenes.icosphere_scene(level=args.level, width=args.width, height=args.height)
    W, H = desc.width, desc.height
    hs = xb.HostScene.from_desc(desc)
    r = xb.Renderer(W, H, desc.max_bounces, desc.min_bounces, device=local,
                    flags=abi.XB_FLAG_THREAD_PER_RAY if args.thread_per_ray else 0)
    r.upload_scene(hs)
    cam = xb.camera(desc.eye, desc.target, desc.fov, W / H)
    npix = W * H
    from xenon_b200 import autotune
    tuned = autotune.load_tuning("config2") if (W, H, args.level) == (1920, 1080, 8) else None
    if tuned:
        r.set_tuning(**tuned)

    # traversal work per ray (untimed pass with counters), for the roofline's algorithmic bytes
    r.set_profiling(abi.XB_PROFILE_COUNT_TRAVERSAL)
    r.reset_stats()
    r.reset_profile()
    r.render_range(cam, 100000, 1)
    cst = r.stats()
    cpr = r.profile()
    n_ext = cst.rays_closest
    ext_bytes_per_ray = (64 * cpr.ext_blas_nodes + 48 * cpr.ext_tris + 32 * cpr.ext_tlas_nodes +
                         48 * cpr.ext_instances) / n_ext + 32 + 20
    n_sh = max(cst.rays_shadow, 1)
    work = {"blas_nodes_per_ray": cpr.ext_blas_nodes / n_ext, "tris_per_ray": cpr.ext_tris / n_ext,
            "tlas_nodes_per_ray": cpr.ext_tlas_nodes / n_ext, "instances_per_ray": cpr.ext_instances / n_ext,
            "shadow_blas_nodes_per_ray": cpr.sh_blas_nodes / n_sh, "shadow_tris_per_ray": cpr.sh_tris / n_sh}
    r.reset()

    # warm-up
    r.set_profiling(0)
    sps = args.spp_per_step
    base = rank * (args.steps + args.warmup + 8) * sps + 1
    for s in range(args.warmup):
        r.render_range(cam, base + s * sps, sps)
    r.reset()
    r.reset_stats()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    barrier(ws)
    torch.cuda.synchronize()
    dev_ms = 0.0
    with ClockSampler(local) as clk:
        for s in range(args.steps):
            flush.zero_()                      # L2 flush between timed steps (outside the events)
            torch.cuda.synchronize()
            r.render_range(cam, base + (args.warmup + s) * sps, sps)
            dev_ms += r.stats().last_ms
    torch.cuda.synchronize()
    barrier(ws)
    st = r.stats()
    rays = st.rays_closest + st.rays_shadow
    t_max = allreduce_max(dev_ms, ws)
    rays_all = allreduce_sum(float(rays), ws)
    value = rays_all / (t_max * 1e-3) / 1e6
    msamples = allreduce_sum(float(st.paths), ws) / (t_max * 1e-3) / 1e6
    rays_per_path = rays / st.paths

    # The timed steps replay captured bounce loops (CUDA graphs), inside which no event can time
    # one launch; the same steps again with stage timing (events around every launch, hence
    # direct launches) give each kernel's launch durations and counts.
    r.set_profiling(abi.XB_PROFILE_STAGE_TIMES)
    r.reset_profile()
    r.reset_stats()
    n_prof = max(3, min(args.steps, 20))
    prof_ms = 0.0
    for s in range(n_prof):
        flush.zero_()
        torch.cuda.synchronize()
        r.render_range(cam, base + (args.warmup + args.steps + s) * sps, sps)
        prof_ms += r.stats().last_ms
    prof = r.profile()
    pst = r.stats()
    launches_per_step = (prof.raygen_launches + prof.extend_launches + prof.shade_launches +
                         prof.shadow_launches + prof.accumulate_launches) / n_prof
    launches = launches_per_step * args.steps

    # Roofline of the extend kernel: its algorithmic bytes ÷ the time during which at least one
    # of its launches ran (the union of the launch intervals over all wave lanes, which cannot
    # exceed the step), from the same steps run again with stage timing.
    peaks = load_peaks()
    ext_bytes = ext_bytes_per_ray * pst.rays_closest
    ext_busy_ms = prof.extend_busy_ms
    achieved = ext_bytes / (ext_busy_ms * 1e-3) / 1e9
    step_avg = ext_bytes / n_prof / (t_max / args.steps * 1e-3) / 1e9
    traffic = None
    tp = os.path.join(ROOT, "profiles", "extend_kernel_config2.json")
    if os.path.exists(tp):
        with open(tp) as f:
            tj = json.load(f)
        if tj.get("dram_bytes_per_closest_ray"):
            traffic = tj["dram_bytes_per_closest_ray"] * pst.rays_closest / max(prof.extend_launches, 1)
    # the same kernel with one wave in flight (untimed pass): its launches then have the GPU to
    # themselves, while in the timed region the other lanes' kernels run beside them
    lanes = r.tuning()["waves"]
    one_lane = None
    if lanes > 1:
        r.set_tuning(waves=1)
        r.reset_profile()
        r.reset_stats()
        n1 = max(3, min(args.steps, 10))
        for s in range(n1):
            flush.zero_()
            torch.cuda.synchronize()
            r.render_range(cam, base + (args.warmup + args.steps + n_prof + s) * sps, sps)
        p1 = r.profile()
        a1 = ext_bytes_per_ray * r.stats().rays_closest / max(p1.extend_busy_ms * 1e-3, 1e-12) / 1e9
        one_lane = {"achieved": a1, "frac": a1 / peaks["hbm_gbs"], "extend_ms_per_launch":
                    p1.extend_ms / max(p1.extend_launches, 1)}
        r.set_tuning(waves=lanes)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": achieved / peaks["hbm_gbs"], "traffic": traffic,
                "peak_source": peaks["source"], "kernel": "extend_kernel (closest-hit traversal)",
                "algorithmic_bytes_per_ray": ext_bytes_per_ray,
                "algorithmic_bytes_per_launch": ext_bytes / max(prof.extend_launches, 1),
                "extend_busy_ms_per_step": ext_busy_ms / n_prof,
                "extend_launch_ms_per_step": prof.extend_ms / n_prof,
                "profiled_ms_per_step": prof_ms / n_prof, "ms_per_step": t_max / args.steps,
                "step_average_achieved": step_avg, "waves_in_flight": lanes,
                "timing": "algorithmic bytes / extend busy time: the union of the extend launches' intervals "
                          f"(CUDA events around each launch) over {n_prof} steps of the timed workload run again "
                          "with stage timing (the timed steps replay captured graphs, inside which no event "
                          "times one launch); extend_launch_ms_per_step sums the launches' own durations, "
                          "which overlap across wave lanes; step_average_achieved divides by the whole "
                          "timed step instead",
                "one_lane": one_lane, **work}

    # e2e through the public API with host buffers: render + resolve to pinned host memory
    host = torch.empty((H, W, 3), dtype=torch.float32, pin_memory=True)
    r.set_profiling(0)
    r.reset_stats()
    L = xb.lib()
    host2 = torch.empty((H, W, 3), dtype=torch.float32, pin_memory=True)
    outs = (host, host2)
    for s in range(2):                       # untimed warm-up of the same calls
        xb.native.check(L.xb_render(r.h, ctypes.byref(cam), sps), r.h)
        xb.native.check(L.xb_resolve_async(r.h, ctypes.c_void_p(outs[s % 2].data_ptr())), r.h)
    xb.native.check(L.xb_sync(r.h), r.h)
    r.reset()
    r.reset_stats()
    barrier(ws)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e2e_steps = max(3, min(args.steps, 20))
    for s in range(e2e_steps):
        xb.native.check(L.xb_render(r.h, ctypes.byref(cam), sps), r.h)
        # every step's mean image goes to the host; the copy of step k overlaps step k+1
        xb.native.check(L.xb_resolve_async(r.h, ctypes.c_void_p(outs[s % 2].data_ptr())), r.h)
    xb.native.check(L.xb_sync(r.h), r.h)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    e2e_s = allreduce_max(e2e_s, ws)
    st2 = r.stats()
    e2e_rays = allreduce_sum(float(st2.rays_closest + st2.rays_shadow), ws)
    e2e = {"value": e2e_rays / e2e_s / 1e6, "unit": "Mrays/s",
           "h2d_bytes_per_step": int(ctypes.sizeof(cam)),
           "d2h_bytes_per_step": int(W * H * 3 * 4), "steps": e2e_steps,
           "note": f"host wall clock over back-to-back steps of {sps} spp (no L2 flush between them, "
                   "unlike `value`); each step's mean image is read back by xb_resolve_async, "
                   "overlapping the next step, and xb_sync ends the timed region"}

    # the single exchange of the multi-GPU path: the per-pixel sums reduced to rank 0 on the
    # device (untimed; xenon_b200.distributed)
    if ws > 1:
        import torch.distributed as dist
        from xenon_b200 import distributed
        dist.reduce(distributed._local_moments(r, max(r.spp, 1), "cuda"), dst=0)

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        try:
            with quiet_stdout():
                cpu = cpu_reference_sample(desc, rays_per_path, args.cpu_seconds)
        except Exception as e:
            cpu = {"value": None, "unit": "Mrays/s", "cores": None, "kind": "reference",
                   "sample": f"failed: {e}"}

    config3 = None
    if rank == 0 and ws == 1 and not args.no_config3:
        try:
            config3 = config3_study(args, local)
        except Exception as e:
            config3 = {"error": f"{type(e).__name__}: {e}"}
    views = None
    if rank == 0 and ws == 1 and not args.no_views_study:
        try:
            views = views_study(args, local)
        except Exception as e:
            views = {"error": f"{type(e).__name__}: {e}"}
    incoherent = None
    if rank == 0 and ws == 1 and not args.no_incoherent:
        try:
            incoherent = incoherent_study(args, local)
        except Exception as e:
            incoherent = {"error": f"{type(e).__name__}: {e}"}
    build = None
    if rank == 0 and ws == 1 and not args.no_build_study:
        try:
            build = build_study(args)
        except Exception as e:
            build = {"error": f"{type(e).__name__}: {e}"}
    sky = None
    if rank == 0 and ws == 1 and not args.no_sky_study:
        try:
            sky = sky_study(args, local)
        except Exception as e:
            sky = {"error": f"{type(e).__name__}: {e}"}
    guiding = None
    if rank == 0 and ws == 1 and not args.no_guiding_study:
        try:
            guiding = guiding_study(args, local)
        except Exception as e:
            guiding = {"error": f"{type(e).__name__}: {e}"}

    if rank == 0:
        detail = {"spp_per_step": sps, "paths_per_step": npix * sps, "rays_per_path": rays_per_path,
                  "msamples_per_s": msamples, "parallelism": f"sample-sharded x{ws}" if ws > 1 else "1 GPU",
                  "tuning": r.tuning(), "tuning_source": "xenon_b200/tuning (autotuner)" if tuned else "defaults",
                  "stage_ms_per_step_profiled": {k: getattr(prof, k) / n_prof for k in
                                                 ("raygen_ms", "extend_ms", "shade_ms", "shadow_ms",
                                                  "accumulate_ms", "extend_busy_ms", "shade_busy_ms",
                                                  "shadow_busy_ms")}}
        studies = {"bvh_build": {k: _sig(v) for k, v in build.items()} if build and "error" not in build else build,
                   "config3": config3_summary(config3), "incoherent": incoherent_summary(incoherent),
                   "views": views_summary(views), "sky_is": sky_summary(sky), "guiding": guiding_summary(guiding)}
        if args.detail_out:
            with open(args.detail_out, "w") as f:
                json.dump({"detail": detail, "bvh_build": build, "config3": config3, "incoherent": incoherent, "views": views,
                           "sky_is": sky, "guiding": guiding}, f, indent=1)
        line = {"metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded procedural scene, seed 1)",
                "config": shared_config(desc, args.level), "detail": detail,
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches),
                "clocks": clk.summary(), **studies}
        print(json.dumps(line))
    r.close()
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
