"""The lighting path (GigaVoxels.frag with ComputeLighting): the GPU ray
cast with a gradient pool against the oracle's lit shader on the same
pools.  Lighting changes only colour, so the node-usage lists stay
bit-exact; colour within 1/255 (both sides run the same binary32
operations, pow(x, 100) restated as squarings)."""
import numpy as np
import pytest

import voxviz_b200 as vv
from oracle import gv_oracle as go
from tests import helpers

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lit_scene():
    sc = helpers.Scene(seed=1, depth=5, fmt="rgba8")
    g = helpers.GpuScene(sc)
    n = sc.xyz.shape[0]
    grads = {}
    for gf in ("fp32", "rgba8", "dxt1"):
        grads[gf] = np.zeros((sc.pool.shape[0], vv.BRICK_BYTES[vv.fmt_code(gf)]), dtype=np.uint8)
        grads[gf][:n] = sc.octree.produce_gradients(sc.xyz, gf)
    return sc, g, grads


@pytest.mark.parametrize("gfmt,unsigned", [("fp32", 0), ("rgba8", 1), ("dxt1", 1)])
def test_lit_view_matches_oracle(lit_scene, gfmt, unsigned):
    sc, g, grads = lit_scene
    n = sc.xyz.shape[0]
    g.ctx.create_gradpool(gfmt)
    g.ctx.upload_gradients(np.arange(n, dtype=np.uint32), grads[gfmt][:n])
    for seed in (3, 11):
        u = sc.uniforms(sc.view(seed, 256, 192))
        u.compute_lighting = 1
        u.gradients_unsigned = unsigned
        got = g.render(u)
        osc = go.Scene(sc.words, sc.pool, sc.slots, sc.fmt, sc.jitter, grads=grads[gfmt],
                       grad_fmt=vv.fmt_code(gfmt))
        ref = helpers.oracle_frame(u, osc)
        assert got["status"] == 0 and ref["status"] == 0
        assert np.array_equal(got["usage"], ref["usage"])
        err = np.abs(got["color"] - ref["color"])
        assert err.max() <= 1.0 / 255.0, err.max()
        assert np.array_equal(got["requests"], ref["requests"])
        # lighting does change the image
        u0 = sc.uniforms(sc.view(seed, 256, 192))
        unlit = g.render(u0)["color"]
        assert np.abs(unlit - got["color"]).max() > 0.05


def test_lighting_without_gradient_pool_is_refused():
    sc = helpers.Scene(seed=1, depth=4, fmt="rgba8")
    g = helpers.GpuScene(sc)
    u = sc.uniforms(sc.view(3, 64, 64))
    u.compute_lighting = 1
    with pytest.raises(vv.VVError):
        g.render(u)
