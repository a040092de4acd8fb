"""Known-answer tests on one-node scenes, against analytic expectations
computed here in float64 from the geometry alone:

* a constant root node of colour c and alpha a: each ray enters the unit
  box (the front-face point of GigaVoxels.vert, then the jitter offset of
  GigaVoxels.frag:544-564), takes int(t / RayStepSize) + 1 constant samples
  to the box exit (ComputeMinRayBoxIntersection, :127-183) and composites
  them front to back (TraverseConstant, :233-285): after m samples
  dst.a = 1 - (1 - a)^m and dst.rgb = c (1 - (1 - a)^m) / a, m stopping once
  dst.a exceeds the termination threshold;
* a root brick whose texels hold a linear function of the texel index with
  alpha 1: the first brick sample (TraverseBrick, :327-391) is GL_LINEAR
  filtering of that function at the ray's entry, which reproduces it, and
  ends the ray.

The oracle is checked on the CPU; the kernels through the C ABI on the
GPU."""
import numpy as np
import pytest

import voxviz_b200 as vv
from voxviz_b200 import _native as N

W, H = 48, 36
RGB = (200, 120, 40)  # the constant node's colour; its alpha is a parameter


def _info(root_is_constant):
    i = N.OctreeInfo()
    i.depth = 0
    i.volume_dim = 8
    i.node_count = 8
    i.pool_dim[:] = [2, 2, 2]
    i.nonconst_count = 0 if root_is_constant else 1
    i.root_is_constant = 1 if root_is_constant else 0
    return i


def _camera(pos, target):
    look, up = vv.look_at(pos, target)
    return vv.make_camera(pos, look, up, W, H, near=0.01)


def _scene(constant, alpha=40):
    words = np.zeros((2, 2, 2, 2), dtype=np.uint32)
    pool = np.zeros((1, 4000), dtype=np.uint8)
    if constant:
        r, g, b = RGB
        words[0, 0, 0] = (0x40000000, r | (g << 8) | (b << 16) | (alpha << 24))
    else:
        words[0, 0, 0] = (0x80000000, (1 << 20) | (1 << 10) | 1)  # resident, brick at slot 0 + border
        i = np.arange(10)
        z, y, x = np.meshgrid(i, i, i, indexing="ij")
        tex = (20 * x) | ((20 * y) << 8) | ((20 * z) << 16) | (255 << 24)
        pool[0] = tex.astype("<u4").reshape(-1).view(np.uint8)
    jit = np.full(32 * 32, 255, dtype=np.uint8)
    jit[::3] = 128
    return words, pool, jit


def _rays(u, jit):
    """{(py, px): (start position after the jitter, direction)} of the rays
    that enter the box."""
    C = np.array(u.camera_position, dtype=np.float64)
    out = {}
    for py in range(H):
        for px in range(W):
            d = (np.array(u.near_origin, dtype=np.float64) + (px + 0.5) * np.array(u.near_dx, dtype=np.float64)
                 + (py + 0.5) * np.array(u.near_dy, dtype=np.float64))
            t0 = (0.0 - C) / d
            t1 = (1.0 - C) / d
            tn, tf = np.minimum(t0, t1), np.maximum(t0, t1)
            te, tx = tn.max(), tf.min()
            if not (te <= tx and te > 0):
                continue
            org = C + d * te
            dirv = (org - C) / np.linalg.norm(org - C)
            j = jit[(py % 32) * 32 + (px % 32)] / 255.0
            start = org + dirv * u.ray_step_size * j
            if not np.all((start > 0.0) & (start < 1.0)):
                continue
            out[(py, px)] = (start, dirv)
    return out


def _exit(start, dirv):
    t = 4.0
    for a in range(3):
        if dirv[a] > 0:
            t = min(t, (1.0 - start[a]) / dirv[a])
        elif dirv[a] < 0:
            t = min(t, (0.0 - start[a]) / dirv[a])
    return t


def _expect_constant(u, rays, alpha):
    a = alpha / 255.0
    c = np.array(RGB) / 255.0
    exp = {}
    for key, (start, dirv) in rays.items():
        q = _exit(start, dirv) / u.ray_step_size
        if abs(q - round(q)) < 1e-3:  # the binary32 count may round to either side
            continue
        n = int(q) + 1
        m, da = 0, 0.0
        while m < n and not da > u.alpha_stop:
            m += 1
            da = 1.0 - (1.0 - a) ** m
        exp[key] = np.concatenate([c * da / a, [da]])
    return exp


def _expect_brick(u, rays):
    return {key: np.array([20 * (0.5 + 8 * start[0]) / 255.0, 20 * (0.5 + 8 * start[1]) / 255.0,
                           20 * (0.5 + 8 * start[2]) / 255.0, 1.0]) for key, (start, _) in rays.items()}


CAMERAS = [((-0.9, 0.45, 0.55), (0.5, 0.5, 0.5)), ((1.7, 1.9, 1.4), (0.5, 0.4, 0.5)), ((0.4, -1.2, 0.3), (0.6, 0.5, 0.6))]


def _check(colour, rays, exp, tol):
    assert len(exp) > 100
    worst = max(float(np.abs(colour[py, px] - e).max()) for (py, px), e in exp.items())
    assert worst <= tol, worst
    # pixels whose ray misses the box stay (0, 0, 0, 0)
    missed = [(py, px) for py in range(H) for px in range(W) if (py, px) not in rays]
    assert missed and all(not colour[py, px].any() for py, px in missed)


# (constant root, its alpha): 40 never reaches the threshold inside the box,
# 120 ends every ray after a few samples
KINDS = [(True, 40), (True, 120), (False, 0)]


@pytest.mark.parametrize("constant,alpha", KINDS)
@pytest.mark.parametrize("cam_i", range(len(CAMERAS)))
def test_oracle_known_answers(constant, alpha, cam_i):
    from oracle import gv_oracle as go
    words, pool, jit = _scene(constant, alpha)
    u = vv.compute_uniforms(_info(constant), _camera(*CAMERAS[cam_i]), (1, 1, 1), 1.0, 0.99)
    rays = _rays(u, jit)
    exp = _expect_constant(u, rays, alpha) if constant else _expect_brick(u, rays)
    colour, _, st = go.raycast(u, go.Scene(words, pool, (1, 1, 1), vv.VV_FMT_RGBA8, jit))
    assert st == 0
    _check(colour, rays, exp, 2e-5)


@pytest.mark.gpu
@pytest.mark.parametrize("constant,alpha", KINDS)
@pytest.mark.parametrize("cam_i", range(len(CAMERAS)))
def test_kernel_known_answers(constant, alpha, cam_i):
    import torch
    words, pool, jit = _scene(constant, alpha)
    ctx = vv.Context(0)
    ctx.upload_nodes(words)
    ctx.create_brickpool((1, 1, 1), "rgba8")
    ctx.upload_bricks(np.zeros(1, dtype=np.uint32), pool)
    ctx.set_jitter(jit)
    u = vv.compute_uniforms(_info(constant), _camera(*CAMERAS[cam_i]), (1, 1, 1), 1.0, 0.99)
    dev = torch.device("cuda", 0)
    colour = torch.zeros((H, W, 4), dtype=torch.float32, device=dev)
    usage = torch.zeros((H, W, 12), dtype=torch.int32, device=dev)
    ctx.render(u, colour.data_ptr(), usage.data_ptr(), 0, 0, 0, 0, 4, vv.VV_PASS_RAYCAST)
    ctx.synchronize()
    assert ctx.device_status() == 0
    rays = _rays(u, jit)
    exp = _expect_constant(u, rays, alpha) if constant else _expect_brick(u, rays)
    _check(colour.cpu().numpy(), rays, exp, 2e-5)
