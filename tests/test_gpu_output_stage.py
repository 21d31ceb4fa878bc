"""The output stage on the device (xb_output_stage: the reference's save_image pixels and its
ImageNoiseEstimator statistics, src/main.cpp:24-52, src/math/image.h:35-118) against the host
forms (xb_image_to_rgb8, xb_image_noise_stats), which are bit-identical to the reference's
(tests/test_output_stage.py), over the same rendered mean image."""
import numpy as np
import pytest

import xenon_b200 as xb
from xenon_b200 import scenes


@pytest.mark.gpu
@pytest.mark.parametrize("name,w,h,spp", [("cornell", 128, 128, 16), ("icosphere", 240, 135, 4),
                                          ("instanced", 200, 112, 2)])
def test_device_output_stage_matches_host(name, w, h, spp):
    desc = {"cornell": scenes.cornell, "icosphere": lambda: scenes.icosphere_scene(level=5),
            "instanced": lambda: scenes.instanced_grid(grid=3, levels=(3, 3, 3, 3))}[name]()
    r = xb.Renderer(w, h, desc.max_bounces, desc.min_bounces)
    r.upload_scene(xb.HostScene.from_desc(desc))
    r.render_frame(xb.camera(desc.eye, desc.target, desc.fov, w / h), spp)
    img = r.resolve()
    pix, st = r.output_stage()
    want_pix = xb.image_to_rgb8(img)
    want = xb.noise_stats(img)
    # 8-bit values: equal but where the gamma's powf rounds differently (CUDA vs the host's)
    diff = pix.astype(int) - want_pix.astype(int)
    assert np.abs(diff).max() <= 1 and np.mean(diff != 0) < 1e-3, np.mean(diff != 0)
    # exact: counts, thresholds, maximum and the order statistics
    for k in ("valid_pixel_count", "total_interior_pixel_count", "valid_pixel_ratio", "avg_luminance",
              "edge_threshold", "epsilon", "max_absolute", "median_absolute", "p95_absolute"):
        assert st[k] == want[k], (k, st[k], want[k])
    # FP64 sums reduced in another order: the float result within one ulp
    for k in ("mean_squared_score", "rms_score", "mean_absolute"):
        assert abs(st[k] - want[k]) <= 2 * np.spacing(np.float32(want[k])), (k, st[k], want[k])
    assert want["valid_pixel_count"] > 0
    # the device pixels make the same PNG file
    p8, _ = r.output_stage(rgb8=True, stats=False)
    assert np.array_equal(p8, pix)
