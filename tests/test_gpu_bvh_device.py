"""XB_BUILD_DEVICE on a B200: node and order arrays equal the recursive build's (and so the
reference's), on small scenes and on the full config-2 mesh; build times printed."""
import time

import pytest

from xenon_b200 import HostScene, abi, scenes
from tests.test_bvh_levels import SCENES, _arrays, _signed_zero_mesh

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", list(SCENES) + ["signed_zeros", "config2"])
def test_device_build_equals_recursive_build(name):
    desc = {"signed_zeros": _signed_zero_mesh, "config2": scenes.icosphere_scene}.get(name, SCENES.get(name))()
    t0 = time.perf_counter()
    rec = _arrays(HostScene.from_desc(desc, build_threads=1))
    t1 = time.perf_counter()
    dev = _arrays(HostScene.from_desc(desc, build_mode=abi.XB_BUILD_DEVICE))
    t2 = time.perf_counter()
    print(name, "recursive %.3f s, device %.3f s" % (t1 - t0, t2 - t1))
    for k in rec:
        assert dev[k] == rec[k], k
