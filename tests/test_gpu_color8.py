"""RGBA8 colour output (VV_PASS_COLOR_RGBA8): every pixel is the float
colour of the same frame as unorm8, round(clamp(c, 0, 1) * 255) with ties to
even, through vv_render and through a renderer created with color_rgba8."""
import numpy as np
import pytest

import voxviz_b200 as vv
from voxviz_b200 import scene
from tests import helpers

pytestmark = pytest.mark.gpu


def _unorm8(c):
    f = (np.clip(c.astype(np.float32), np.float32(0), np.float32(1)) * np.float32(255)).astype(np.float32)
    return np.rint(f).astype(np.uint8)


def test_render_rgba8_matches_float_colour():
    import torch
    sc = helpers.Scene(seed=1, depth=5)
    g = helpers.GpuScene(sc)
    W, H = 320, 200
    u = sc.uniforms(sc.view(3, W, H))
    dev = torch.device("cuda", 0)
    f32 = torch.zeros((H, W, 4), dtype=torch.float32, device=dev)
    c8 = torch.zeros((H, W), dtype=torch.int32, device=dev)
    g.ctx.render(u, f32.data_ptr(), passes=vv.VV_PASS_RAYCAST)
    g.ctx.render(u, c8.data_ptr(), passes=vv.VV_PASS_RAYCAST | vv.VV_PASS_COLOR_RGBA8)
    g.ctx.synchronize()
    assert g.ctx.device_status() == 0
    got = c8.cpu().numpy().view(np.uint8).reshape(H, W, 4)
    assert np.array_equal(got, _unorm8(f32.cpu().numpy()))
    assert (got[..., 3] == 255).any() and (got[..., 3] == 0).any()


def test_rgba8_renderer_matches_float_renderer():
    o = helpers.octree(seed=3, depth=6)
    W, H = 256, 160
    outs = []
    for rgba8 in (False, True):
        ctx = vv.Context(0)
        r = vv.Renderer(ctx, o, fmt="rgba8", pool_bytes=700 * 4000, preload_all=False, alpha_stop=0.99,
                        jitter_seed=7, device_paging=True, color_rgba8=rgba8)
        frames = []
        for cam in scene.camera_path(5, o.heights(), 6, W, H):
            r.draw(cam)
            colour = r.read_color()
            r.update()
            frames.append((colour, r.last_requests()))
        outs.append(frames)
    for (c32, q32), (c8, q8) in zip(*outs):
        assert c8.dtype == np.uint8 and np.array_equal(c8, _unorm8(c32))
        assert np.array_equal(q32, q8)
