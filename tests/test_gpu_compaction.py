"""Selection mask and histopyramid compaction on the GPU against the
oracle's literal walk of CompressNodeUsageList.frag, on ragged sizes."""
import numpy as np
import pytest

from oracle import gv_oracle as go
from tests import helpers

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def g():
    sc = helpers.Scene(seed=2, depth=5)
    return sc, helpers.GpuScene(sc)


@pytest.mark.parametrize("w,h", [(1, 1), (2, 3), (7, 4), (33, 17), (255, 1), (1, 130), (480, 270), (1920, 1080)])
def test_compaction_ragged_viewports(g, w, h):
    sc, gs = g
    u = sc.uniforms(sc.view(5, w, h))
    got = gs.render(u, max_push=8)
    ref = helpers.oracle_frame(u, sc.oracle_scene(), max_push=8)
    assert np.array_equal(got["usage"], ref["usage"])
    assert np.array_equal(got["mask"], ref["mask"])
    assert got["count"] == ref["count"]
    assert np.array_equal(got["requests"], ref["requests"])


@pytest.mark.parametrize("cap", [1, 37, 1000])
def test_request_cap_keeps_first_keys(g, cap):
    sc, gs = g
    u = sc.uniforms(sc.view(9, 320, 240))
    got = gs.render(u, max_push=12, cap=cap)
    ref = helpers.oracle_frame(u, sc.oracle_scene(), max_push=12, cap=cap)
    assert got["count"] == ref["count"] and got["count"] > cap
    assert np.array_equal(got["requests"], ref["requests"])


def test_request_set_covers_all_kept_items(g):
    sc, gs = g
    u = sc.uniforms(sc.view(13, 512, 512))
    got = gs.render(u, max_push=12)
    usage, mask = got["usage"], got["mask"]
    kept = set()
    for y, x in zip(*np.nonzero(mask)):
        bits = int(mask[y, x])
        items = [int(usage[y, x, i]) for i in range(12) if bits >> i & 1]
        kept.update(items[-4:] if len(items) > 4 else items)
    got_set = set(int(v) for v in got["requests"].reshape(-1) if v)
    assert got_set <= kept
    # with 12 pushes an entry keeps the last 4 pushed items of its pixel (FIFO overwrite)
    assert got_set == kept


@pytest.mark.parametrize("w,h,cap", [(64, 64, 0), (65, 65, 0), (127, 95, 0), (129, 1, 0), (2047, 3, 0), (97, 191, 0),
                                     (640, 480, 0), (1920, 1080, 5000), (1023, 767, 0), (4096, 2160, 0)])
def test_three_launch_compaction_equals_per_level(g, w, h, cap):
    """vv_ctx_set_compaction: the three-launch form (selection and the
    pyramid's lowest five levels per level-5 node, the levels above in one
    CTA, offsets down and compaction per node) gives the mask, count and
    requests of the per-level passes, on sizes whose levels fold rows and
    columns; the first sizes also against the oracle."""
    sc, gs = g
    u = sc.uniforms(sc.view(7, w, h))
    kw = {"max_push": 8}
    if cap:
        kw["cap"] = cap
    fused = gs.render(u, **kw)
    gs.ctx.set_compaction(per_level=True)
    try:
        per_level = gs.render(u, **kw)
    finally:
        gs.ctx.set_compaction(per_level=False)
    for k in ("mask", "requests"):
        assert np.array_equal(fused[k], per_level[k]), k
    assert fused["count"] == per_level["count"]
    assert fused["status"] == per_level["status"] == 0
    if w * h <= 128 * 128:
        ref = helpers.oracle_frame(u, sc.oracle_scene(), **kw)
        assert np.array_equal(fused["mask"], ref["mask"])
        assert fused["count"] == ref["count"]
        assert np.array_equal(fused["requests"], ref["requests"])
