"""A brick pool far smaller than a frame's uploads: the LRU order wraps
within one page-request service (slots uploaded in this service are evicted
again), on both the host and the device paging paths.  Every frame's
residency and node words match the policy restatement, and every resident
slot holds its node's brick (one upload per slot survives a service)."""
import numpy as np
import pytest

import voxviz_b200 as vv
from oracle.paging_ref import PagingRef
from voxviz_b200 import scene
from tests import helpers

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("device_paging", [False, True])
def test_tiny_pool_wraps_and_matches_policy(device_paging):
    o = helpers.octree(seed=3, depth=5)
    f = vv.fmt_code("rgba8")
    pool_bricks = 12
    slots = scene.slot_grid(pool_bricks)
    ctx = vv.Context(0)
    r = vv.Renderer(ctx, o, fmt="rgba8", pool_bytes=pool_bricks * 1000 * vv.TEXEL_BYTES[f], preload_all=False,
                    device_paging=device_paging)
    sim = PagingRef(o.node_words(), slots)
    sim.init(False)
    wrapped = False
    for cam in scene.camera_path(11, o.heights(), 6, 128, 80):
        assert np.array_equal(ctx.download_nodes(), sim.words), f"node words diverged before frame {cam.frame}"
        r.draw(cam)
        r.update()
        up = sim.update(r.last_requests())
        wrapped |= len(up) > pool_bricks
        xyz, slot = r.residency()
        got = {tuple(int(v) for v in p): int(s) for p, s in zip(xyz, slot)}
        assert got == sim.residency(), f"residency differs after frame {cam.frame}"
        if len(slot):
            pool = ctx.download_bricks()
            assert np.array_equal(pool[slot], o.produce_bricks(xyz, f)), f"slot contents after frame {cam.frame}"
    assert wrapped, "no service uploaded more bricks than the pool holds"
    assert ctx.device_status() == 0
