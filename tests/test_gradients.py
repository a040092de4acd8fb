"""Gradient bricks (the input of the lighting path) against the dense numpy
restatement of the reference's gradient cascade, bit for bit."""
import numpy as np

import voxviz_b200 as vv
from oracle import terrain_ref as tr
from voxviz_b200 import scene
from tests import helpers


def test_gradient_bricks_match_dense_restatement():
    o = helpers.octree(seed=2, depth=4)
    info = o.info
    leaf = o.mip_level(0)
    alpha = ((leaf >> 24).astype(np.float32) / np.float32(255.0)).astype(np.float32)
    levels = tr.gradient_pyramid(tr.leaf_gradients(alpha))
    _, _, _, xyz = scene.resident_scene(o, "rgba8")
    pick = xyz[:: max(1, len(xyz) // 40)]
    got = o.produce_gradients(pick, "fp32").view(np.float32).reshape(len(pick), 10, 10, 10, 4)
    for (x, y, z), g in zip(pick, got):
        ni = o.node_info(int(x), int(y), int(z))
        m = info.depth - ni.level
        ref = tr.gradient_brick(levels[m], ni.origin)
        assert np.array_equal(g[..., :3], ref), (x, y, z, ni.level)
        assert not np.any(g[..., 3])
    # the unsigned RGBA8 form: round((g + 1) / 2 * 255)
    got8 = o.produce_gradients(pick[:4], "rgba8").view(np.uint32).reshape(4, 10, 10, 10)
    ref8 = got[:4, ..., :3]
    q = np.floor(((ref8 + np.float32(1)) * np.float32(0.5)) * np.float32(255) + np.float32(0.5)).astype(np.uint32)
    packed = q[..., 0] | (q[..., 1] << 8) | (q[..., 2] << 16)
    assert np.array_equal(got8, packed)


def test_gradients_refuse_deep_trees():
    o = helpers.octree(seed=2, depth=7)
    import pytest
    with pytest.raises(vv.VVError):
        o.produce_gradients(np.zeros((1, 3), dtype=np.uint32), "fp32")
