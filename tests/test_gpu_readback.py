"""The asynchronous colour read-back of the renderer: the copy queued after
a draw lands the frame's colour (equal to the synchronous read-back), while
the page-request service and the next draws run; frames alternate between
two device colour buffers, so an earlier frame's copy is not overwritten."""
import numpy as np
import pytest

import voxviz_b200 as vv
from voxviz_b200 import scene
from tests import helpers

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def test_async_readback_matches_sync_readback():
    o = helpers.octree(seed=3, depth=6)
    ctx = vv.Context(0)
    r = vv.Renderer(ctx, o, fmt="rgba8", pool_bytes=700 * 4000, preload_all=False, device_paging=True)
    cams = scene.camera_path(5, o.heights(), 6, 200, 120)
    bufs = [torch.empty((120, 200, 4), dtype=torch.float32, pin_memory=True).numpy() for _ in range(3)]
    expected = []
    for k, cam in enumerate(cams):
        r.draw(cam)
        r.read_color_async(bufs[k % 3])
        r.update()
        expected.append(r.read_color())  # synchronous copy of the same frame (update leaves it)
        if k >= 2:
            r.wait_readback()
            # the three most recent frames are all intact in their host buffers
            for j in range(k - 2, k + 1):
                assert np.array_equal(bufs[j % 3], expected[j]), (k, j)
    r.wait_readback()
    assert ctx.device_status() == 0
