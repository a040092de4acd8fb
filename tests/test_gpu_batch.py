"""The batched persistent launch (vv_render_batch): many views of several
octrees in one launch give, pixel for pixel, the colour and node-usage
lists of per-view vv_render calls, for every compiled tile shape and
steps-per-trip variant; the page-request passes run afterwards on the
batch's usage lists give the same request lists."""
import numpy as np
import pytest

import voxviz_b200 as vv
from tests import helpers

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

SIZES = [(256, 192), (100, 60), (333, 97), (64, 64), (40, 200), (512, 128)]


@pytest.fixture(scope="module")
def scenes():
    a = helpers.Scene(seed=1, depth=5, fmt="rgba8")
    b = helpers.Scene(seed=3, depth=4, fmt="rgba8")
    return [(a, helpers.GpuScene(a)), (b, helpers.GpuScene(b))]


def _views(scenes):
    out = []
    for i, (w, h) in enumerate(SIZES):
        sc, g = scenes[i % 2]
        u = sc.uniforms(sc.view(20 + i, w, h, frame=i))
        out.append((sc, g, u))
    return out


def _buffers(u):
    dev = torch.device("cuda", 0)
    return (torch.full((u.height, u.width, 4), -1.0, dtype=torch.float32, device=dev),
            torch.zeros((u.height, u.width, 12), dtype=torch.int32, device=dev))


def test_batch_matches_per_view_render_for_every_variant(scenes):
    views = _views(scenes)
    refs = [g.render(u, passes=vv.VV_PASS_RAYCAST) for _, g, u in views]
    bufs = [_buffers(u) for _, _, u in views]
    launch_ctx = scenes[0][1].ctx
    batch = vv.Batch(launch_ctx, [(g.ctx, 0, u, c.data_ptr(), us.data_ptr())
                                  for (_, g, u), (c, us) in zip(views, bufs)])
    for variant in vv.batch_variants():
        for c, us in bufs:
            c.fill_(-1.0)
            us.zero_()
        batch.render(variant)
        launch_ctx.synchronize()
        for (_, g, _), ref, (c, us) in zip(views, refs, bufs):
            assert g.ctx.device_status() == 0
            assert np.array_equal(c.cpu().numpy(), ref["color"]), variant
            assert np.array_equal(us.cpu().numpy().view(np.uint32), ref["usage"]), variant


def test_autotune_picks_a_variant_and_keeps_results(scenes):
    views = _views(scenes)
    refs = [g.render(u, passes=vv.VV_PASS_RAYCAST) for _, g, u in views]
    bufs = [_buffers(u) for _, _, u in views]
    launch_ctx = scenes[1][1].ctx
    batch = vv.Batch(launch_ctx, [(g.ctx, 0, u, c.data_ptr(), us.data_ptr())
                                  for (_, g, u), (c, us) in zip(views, bufs)])
    res = batch.autotune(reps=2)
    assert res["best"] in vv.batch_variants()
    assert len(res["ms"]) == len(vv.batch_variants()) and all(t > 0 for t in res["ms"].values())
    batch.render()
    launch_ctx.synchronize()
    for ref, (c, us) in zip(refs, bufs):
        assert np.array_equal(c.cpu().numpy(), ref["color"])


def test_requests_from_batched_usage_lists(scenes):
    views = _views(scenes)
    bufs = [_buffers(u) for _, _, u in views]
    launch_ctx = scenes[0][1].ctx
    batch = vv.Batch(launch_ctx, [(g.ctx, 0, u, c.data_ptr(), us.data_ptr())
                                  for (_, g, u), (c, us) in zip(views, bufs)])
    batch.render((16, 16, 2))
    launch_ctx.synchronize()
    for (sc, g, u), (c, us) in zip(views, bufs):
        ref = g.render(u, max_push=4)
        cap = u.width * u.height
        mask = torch.zeros((u.height, u.width), dtype=torch.int32, device="cuda")
        req = torch.zeros((cap, 4), dtype=torch.int32, device="cuda")
        cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
        g.ctx.render(u, 0, us.data_ptr(), mask.data_ptr(), req.data_ptr(), cnt.data_ptr(), cap, 4,
                     vv.VV_PASS_SELECT | vv.VV_PASS_COMPACT)
        g.ctx.synchronize()
        n = int(cnt.item())
        assert n == ref["count"]
        assert np.array_equal(req.cpu().numpy().view(np.uint32)[:n], ref["requests"])
        assert np.array_equal(mask.cpu().numpy().view(np.uint32), ref["mask"])


def test_batch_rejects_mixed_formats_and_unknown_variants(scenes):
    sc16 = helpers.Scene(seed=1, depth=4, fmt="fp16")
    g16 = helpers.GpuScene(sc16)
    sc, g = scenes[0]
    u8 = sc.uniforms(sc.view(3, 64, 64))
    u16 = sc16.uniforms(sc16.view(3, 64, 64))
    c1, us1 = _buffers(u8)
    c2, us2 = _buffers(u16)
    mixed = vv.Batch(g.ctx, [(g.ctx, 0, u8, c1.data_ptr(), us1.data_ptr()),
                             (g16.ctx, 0, u16, c2.data_ptr(), us2.data_ptr())])
    with pytest.raises(vv.VVError):
        mixed.render((16, 16, 1))
    one = vv.Batch(g.ctx, [(g.ctx, 0, u8, c1.data_ptr(), us1.data_ptr())])
    with pytest.raises(vv.VVError):
        one.render((24, 8, 1))
    one.render((8, 8, 4))
    g.ctx.synchronize()
    assert g.ctx.device_status() == 0
