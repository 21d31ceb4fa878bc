"""Failure detection on the device without a fault: a bounded wait that runs out reports
XB_E_TIMEOUT through the host, and the context stays usable (a render afterwards is correct)."""
import numpy as np
import pytest

import xenon_b200 as xb
from xenon_b200 import abi, scenes

pytestmark = pytest.mark.gpu


def test_a_wait_that_runs_out_reports_and_leaves_the_context_usable():
    desc = scenes.cornell()
    cam = xb.camera(desc.eye, desc.target, desc.fov, 1.0)

    def render():
        r = xb.Renderer(32, 32, desc.max_bounces, desc.min_bounces)
        r.upload_scene(xb.HostScene.from_desc(desc))
        r.render_frame(cam, 2)
        img = r.resolve().copy()
        r.close()
        return img

    before = render()
    assert xb.lib().xb_selftest_wait(1) == abi.XB_OK
    assert xb.lib().xb_selftest_wait(0) == abi.XB_E_TIMEOUT
    assert "ran out" in xb.native.last_error()
    assert xb.lib().xb_selftest_wait(1) == abi.XB_OK
    assert np.array_equal(render(), before)
