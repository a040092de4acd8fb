"""GPU ray cast against the FP32 oracle on the same inputs: node-usage lists
(node indices, LOD choices, traversal order) bit-exact, colour within 1/255
(in practice identical: both sides run the same binary32 operations)."""
import numpy as np
import pytest

import voxviz_b200 as vv
from tests import helpers

pytestmark = pytest.mark.gpu

TOL = 1.0 / 255.0


@pytest.fixture(scope="module")
def cfg1():
    sc = helpers.Scene(seed=1, depth=5, collapse=True, fmt="rgba8")
    return sc, helpers.GpuScene(sc)


@pytest.mark.parametrize("view_seed,frame", [(3, 0), (5, 1), (11, 2), (17, 3)])
def test_config1_view_matches_oracle(cfg1, view_seed, frame):
    sc, g = cfg1
    u = sc.uniforms(sc.view(view_seed, 512, 512, frame=frame))
    got = g.render(u, max_push=4 * (frame % 3 + 1))
    ref = helpers.oracle_frame(u, sc.oracle_scene(), max_push=4 * (frame % 3 + 1))
    assert got["status"] == 0 and ref["status"] == 0
    assert np.array_equal(got["usage"], ref["usage"])
    err = np.abs(got["color"] - ref["color"])
    assert err.max() <= TOL, err.max()
    assert (err > 0).mean() < 1e-3
    assert np.array_equal(got["mask"], ref["mask"])
    assert got["count"] == ref["count"]
    assert np.array_equal(got["requests"], ref["requests"])


@pytest.mark.parametrize("alpha_stop", [0.995, 0.5])
def test_alpha_stop_parameter(cfg1, alpha_stop):
    sc, g = cfg1
    u = sc.uniforms(sc.view(7, 256, 192), alpha=alpha_stop)
    got = g.render(u)
    ref = helpers.oracle_frame(u, sc.oracle_scene())
    assert np.array_equal(got["usage"], ref["usage"])
    assert np.abs(got["color"] - ref["color"]).max() <= TOL


def test_full_tree_and_camera_inside():
    sc = helpers.Scene(seed=4, depth=4, collapse=False)
    g = helpers.GpuScene(sc)
    from voxviz_b200 import scene
    cams = scene.camera_path(2, sc.heights, 8, 200, 120)
    for cam in cams[::3]:
        u = sc.uniforms(cam)
        assert u.camera_inside == 1
        got = g.render(u)
        ref = helpers.oracle_frame(u, sc.oracle_scene())
        assert np.array_equal(got["usage"], ref["usage"])
        assert np.abs(got["color"] - ref["color"]).max() <= TOL
        assert np.array_equal(got["requests"], ref["requests"])


@pytest.mark.parametrize("fmt", ["fp16", "bf16", "fp32", "dxt5"])
def test_float_brick_formats_match_oracle(fmt):
    sc = helpers.Scene(seed=1, depth=5, fmt=fmt)
    g = helpers.GpuScene(sc)
    u = sc.uniforms(sc.view(3, 384, 256))
    got = g.render(u)
    ref = helpers.oracle_frame(u, sc.oracle_scene())
    assert np.array_equal(got["usage"], ref["usage"])
    assert np.abs(got["color"] - ref["color"]).max() <= TOL


@pytest.mark.parametrize("fmt,view", [("rgba8", 3), ("rgba8", 8), ("fp16", 5), ("bf16", 6), ("fp32", 7)])
def test_error_vs_fp64_oracle_within_bound_except_decision_flips(fmt, view):
    """Colour within 1/255 of the binary64 oracle on every pixel whose
    binary64 run takes the same decisions (descent, LOD, step counts, early
    termination) as the binary32 run; the pixels over 1/255 are all decision
    flips, and on the binary32 sample sequence the binary64 colour is within
    1/255 everywhere."""
    from oracle import gv_oracle as go
    sc = helpers.Scene(seed=1, depth=5, fmt=fmt)
    g = helpers.GpuScene(sc)
    u = sc.uniforms(sc.view(view, 512, 512))
    got = g.render(u, passes=vv.VV_PASS_RAYCAST)["color"].astype(np.float64)
    osc = sc.oracle_scene()
    flips, c64, _ = go.flip_pixels(u, osc)
    err = np.abs(got - c64).max(-1)
    assert err[~flips].max() <= TOL, err[~flips].max()
    assert not ((err > TOL) & ~flips).any()
    assert flips.mean() < 0.01, flips.mean()
    fixed = np.abs(got - go.fixed_path(u, osc)).max()
    assert fixed <= TOL, fixed
    rms = float(np.sqrt((np.abs(got - c64) ** 2).mean()))
    assert rms < TOL, rms


def test_miss_only_view_is_empty(cfg1):
    sc, g = cfg1
    look, up = vv.look_at([0.5, 0.5, 1.5], [0.5, 0.5, 3.0])  # looking away from the volume
    u = sc.uniforms(vv.make_camera([0.5, 0.5, 1.5], look, up, 64, 48))
    got = g.render(u)
    assert not got["color"].any() and not got["usage"].any()
    assert got["count"] == 0 and got["requests"].shape[0] == 0


@pytest.mark.parametrize("view,size,depth", [(3, (512, 512), 5), (8, (1920, 1080), 5), (6, (333, 177), 6),
                                             (2, (61, 37), 4)])
def test_brick_staging_ray_cast_equals_tiles(view, size, depth):
    """VV_RAYCAST_STAGED (each warp's shared brick slot copied to shared
    memory by cp.async.bulk) gives the same colour, usage lists, mask and
    requests as the tiled launch; non-RGBA8 pools refuse the mode."""
    sc = helpers.Scene(seed=1, depth=depth, fmt="rgba8")
    g = helpers.GpuScene(sc)
    u = sc.uniforms(sc.view(view, *size))
    a = g.render(u)
    g.ctx.set_raycast_mode("staged")
    try:
        b = g.render(u)
        b2 = g.render(u)
    finally:
        g.ctx.set_raycast_mode("tiles")
    for k in ("color", "usage", "mask", "requests"):
        assert np.array_equal(a[k], b[k]), k
        assert np.array_equal(a[k], b2[k]), k
    assert a["status"] == b["status"] == b2["status"] == 0
    h = helpers.GpuScene(helpers.Scene(seed=1, depth=4, fmt="fp16"))
    with pytest.raises(vv.VVError):
        h.ctx.set_raycast_mode("staged")


@pytest.mark.parametrize("fmt,view,size", [("rgba8", 3, (512, 512)), ("fp16", 5, (333, 177)),
                                           ("rgba8", 8, (1920, 1080)), ("fp32", 9, (61, 37)), ("dxt5", 4, (256, 256))])
def test_lane_refill_ray_cast_equals_tiles(fmt, view, size):
    """VV_RAYCAST_REFILL (persistent warps, finished lanes take new pixels)
    gives the same colour, usage lists, mask and requests as the tiled
    launch."""
    sc = helpers.Scene(seed=1, depth=5, fmt=fmt)
    g = helpers.GpuScene(sc)
    u = sc.uniforms(sc.view(view, *size))
    a = g.render(u)
    g.ctx.set_raycast_mode(True)
    try:
        b = g.render(u)
        b2 = g.render(u)  # the queue counter is reset per launch
    finally:
        g.ctx.set_raycast_mode(False)
    for k in ("color", "usage", "mask", "requests"):
        assert np.array_equal(a[k], b[k]), k
        assert np.array_equal(a[k], b2[k]), k
    assert a["status"] == b["status"] == 0
