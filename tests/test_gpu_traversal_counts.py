"""The traversal work the roofline counts: per closest-hit ray, BLAS interior nodes popped (each
loads both 32-byte children), triangles tested, TLAS nodes popped and instances entered. The
GPU's counters (xb_get_profile, both query forms) must equal the restatement oracle's count of
the same traversal (the reference's visit order, src/geometry/blas.cpp:211-265,
src/geometry/tlas.cpp:172-245) on the same seeded rays, so the algorithmic bytes the bench
divides by time are the traversal's own."""
import numpy as np
import pytest

from oracle import port
from tests.helpers import mixed_rays
from xenon_b200 import HostScene, Renderer, abi, scenes

pytestmark = pytest.mark.gpu

SCENES = {
    "icosphere_L7": lambda: scenes.icosphere_scene(level=7),
    "instanced": lambda: scenes.instanced_grid(grid=4, levels=(4, 4, 5, 5)),
    "room": lambda: scenes.guiding_room(level=6),
}


@pytest.mark.parametrize("name", list(SCENES))
def test_gpu_traversal_counters_equal_the_oracle_count(name):
    desc = SCENES[name]()
    hs = HostScene.from_desc(desc)
    rays = mixed_rays(desc, 1 << 15, seed=17)
    hits_o, work = port.PortScene(hs.view()).trace(rays, abi.XB_TRACE_CLOSEST)
    assert work[0] > len(rays) and work[1] > 0
    for flags in (0, abi.XB_FLAG_THREAD_PER_RAY):   # persistent warps, one ray per thread
        r = Renderer(64, 64, flags=flags)
        r.upload_scene(hs)
        r.reset_profile()
        hits = r.trace_rays(rays, abi.XB_TRACE_CLOSEST)
        p = r.profile()
        r.close()
        got = [p.ext_blas_nodes, p.ext_tris, p.ext_tlas_nodes, p.ext_instances]
        assert got == [int(w) for w in work], (name, flags, got, list(work))
        assert np.array_equal(hits["prim_id"], hits_o["prim_id"])
