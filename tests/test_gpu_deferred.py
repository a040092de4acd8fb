"""Deferred uploads and the external page-request service.

A renderer that services its frame's requests through vv_renderer_service
with deferred uploads (stage, then enqueue, eagerly or from a captured CUDA
graph) ends every frame with the node words, brick pool and colour of a
renderer that runs the plain update() path, on a camera path that evicts."""
import numpy as np
import pytest

import voxviz_b200 as vv
from voxviz_b200 import scene
from tests import helpers

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _pair(pool_bricks=700, fmt="rgba8"):
    o = helpers.octree(seed=3, depth=6)
    pool_bytes = pool_bricks * 1000 * vv.TEXEL_BYTES[vv.fmt_code(fmt)]
    out = []
    for _ in range(2):
        ctx = vv.Context(0)
        r = vv.Renderer(ctx, o, fmt=fmt, pool_bytes=pool_bytes, preload_all=False, alpha_stop=0.99,
                        jitter_seed=7, device_paging=True)
        out.append((ctx, r))
    return o, out


def _same_state(a, b):
    (ca, ra), (cb, rb) = a, b
    assert np.array_equal(ca.download_nodes(), cb.download_nodes())
    xa, sa = ra.residency()
    xb, sb = rb.residency()
    assert np.array_equal(xa, xb) and np.array_equal(sa, sb)
    pa, pb = ca.download_bricks(), cb.download_bricks()
    for s in sa[:: max(1, len(sa) // 64)]:
        assert np.array_equal(pa[s], pb[s])


@pytest.mark.parametrize("graph", [False, True])
def test_deferred_service_matches_update(graph):
    o, (eager, deferred) = _pair()
    ce, re_ = eager
    cd, rd = deferred
    rd.set_deferred(True)
    cams = scene.camera_path(5, o.heights(), 12, 256, 160)
    g = None
    side = torch.cuda.Stream() if graph else None
    if graph:
        cd.set_stream(side.cuda_stream)
    evictions = 0
    for k, cam in enumerate(cams):
        re_.draw(cam)
        rd.draw(cam)
        if graph:
            side.synchronize()
        assert np.array_equal(re_.read_color(), rd.read_color()), f"colour differs at frame {k}"
        re_.update()
        fb = rd.frame_buffers()
        rd.service(fb["requests"], fb["request_count"], cam.width * cam.height)
        rd.stage_uploads()
        if graph:
            if g is None:
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g, stream=side):
                    rd.enqueue_uploads()
            g.replay()
            torch.cuda.synchronize()
        else:
            rd.enqueue_uploads()
            cd.synchronize()
        _same_state(eager, deferred)
        evictions = re_.stats()["evictions_total"]
    assert evictions > 0, "the pool was never full: eviction was not exercised"
    assert ce.device_status() == 0 and cd.device_status() == 0
    if graph:
        cd.set_stream(0)


def test_service_without_device_paging_is_a_state_error():
    o = helpers.octree(seed=3, depth=5)
    ctx = vv.Context(0)
    r = vv.Renderer(ctx, o, fmt="rgba8", preload_all=True, device_paging=False)
    cam = scene.seeded_view(3, o.heights(), 64, 64)
    r.draw(cam)
    fb = r.frame_buffers()
    with pytest.raises(vv.VVError):
        r.service(fb["requests"], fb["request_count"], 64 * 64)
    with pytest.raises(vv.VVError):
        r.set_deferred(True)
    with pytest.raises(vv.VVError):
        r.stage_uploads()
