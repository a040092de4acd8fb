"""Adjoint of the ray cast (vv_render_forward_ckpt / vv_backward) and its
torch.autograd.Function.

* the checkpointing forward gives vv_render's colour bit for bit;
* dL/d(texel) matches the oracle's binary64 adjoint of the same binary32
  ray cast to 1e-3 relative (per texel, for texels above 1e-3 of the largest
  gradient; FP32 atomics are the only difference);
* the autograd gradient matches central finite differences (h = 1e-3) of
  the loss, reduced in float64 on the GPU, within the FP32 rounding of the
  perturbed forward (stated below);
* a few Adam steps through the Function reduce an L2 image loss.
"""
import numpy as np
import pytest

import voxviz_b200 as vv
from tests import helpers

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _pool_f32(sc):
    return np.ascontiguousarray(sc.pool).view(np.float32).reshape(sc.pool.shape[0], 1000, 4)


@pytest.fixture(scope="module")
def fp32_scene():
    sc = helpers.Scene(seed=1, depth=5, fmt="fp32")
    return sc, helpers.GpuScene(sc)


def _ckpt_color(g, u, per_ray=16):
    dev = torch.device("cuda", 0)
    H, W = u.height, u.width
    color = torch.zeros((H, W, 4), dtype=torch.float32, device=dev)
    ck = torch.empty(vv.Context.ckpt_bytes(W, H, per_ray), dtype=torch.uint8, device=dev)
    g.ctx.forward_ckpt(u, color.data_ptr(), ck.data_ptr(), per_ray)
    g.ctx.synchronize()
    return color, ck


@pytest.mark.parametrize("fmt", ["rgba8", "fp16", "fp32"])
def test_forward_ckpt_colour_is_render_colour(fmt):
    sc = helpers.Scene(seed=1, depth=5, fmt=fmt)
    g = helpers.GpuScene(sc)
    for seed in (3, 11):
        u = sc.uniforms(sc.view(seed, 256, 192))
        ref = g.render(u, passes=vv.VV_PASS_RAYCAST)["color"]
        for per_ray in (1, 4, 16):
            got, _ = _ckpt_color(g, u, per_ray)
            assert g.ctx.device_status() == 0
            assert np.array_equal(got.cpu().numpy(), ref)


@pytest.mark.parametrize("per_ray", [2, 16])
def test_backward_matches_fp64_oracle(fp32_scene, per_ray):
    from oracle import gv_oracle as go
    sc, g = fp32_scene
    u = sc.uniforms(sc.view(5, 96, 64))
    _, ck = _ckpt_color(g, u, per_ray)
    rng = np.random.default_rng(per_ray)
    dl = rng.standard_normal((u.height, u.width, 4)).astype(np.float32)
    dl_t = torch.from_numpy(dl).cuda()
    grad = torch.zeros(_pool_f32(sc).shape, dtype=torch.float32, device="cuda")
    g.ctx.backward(u, dl_t.data_ptr(), ck.data_ptr(), per_ray, grad.data_ptr())
    g.ctx.synchronize()
    assert g.ctx.device_status() == 0
    got = grad.cpu().numpy().astype(np.float64)
    ref = go.backward(u, sc.oracle_scene(), dl)
    scale = np.abs(ref).max()
    assert scale > 0
    assert np.array_equal(got != 0, ref != 0)
    big = np.abs(ref) > 1e-3 * scale
    rel = np.abs(got - ref)[big] / np.abs(ref)[big]
    assert rel.max() <= 1e-3, rel.max()
    assert np.abs(got - ref).max() <= 1e-5 * scale


def test_autograd_matches_finite_differences(fp32_scene):
    from voxviz_b200 import diff
    sc, g = fp32_scene
    ctx = vv.Context(0)
    ctx.upload_nodes(sc.words)
    ctx.set_jitter(sc.jitter)
    pool = torch.from_numpy(_pool_f32(sc).copy()).cuda().requires_grad_(True)
    us = [sc.uniforms(sc.view(s, 128, 96)) for s in (3, 5)]
    rng = np.random.default_rng(0)
    target = torch.from_numpy(rng.uniform(0, 1, (2, 96, 128, 4)).astype(np.float32)).cuda()

    def loss64(c):
        return ((c.double() - target.double()) ** 2).sum()

    c = diff.render(pool, ctx, sc.slots, us)
    loss64(c).backward()
    assert diff.check_status(ctx) == 0
    grad = pool.grad.detach().double()
    flat = grad.abs().flatten()
    idx = torch.topk(flat, 64).indices.cpu().numpy()
    h = 1e-3
    fd, an = [], []
    with torch.no_grad():
        base = pool.detach().clone()
        for i in idx:
            p1 = base.clone().flatten()
            p1[i] += h
            p2 = base.clone().flatten()
            p2[i] -= h
            l1 = loss64(diff.render(p1.view_as(base), ctx, sc.slots, us))
            l2 = loss64(diff.render(p2.view_as(base), ctx, sc.slots, us))
            fd.append(float((l1 - l2) / (2 * h)))
            an.append(float(grad.flatten()[i]))
    fd, an = np.array(fd), np.array(an)
    # FP32 rounding of the perturbed colours: |dc| <= 2^-24 per channel of
    # the affected pixels, so the FD itself carries ~1e-3 relative noise on
    # the largest gradients; a control-flow change (a ray crossing the
    # alpha stop) shows as a jump, which these texels do not cause.
    rel = np.abs(fd - an) / np.abs(an)
    assert np.median(rel) <= 1e-3, np.median(rel)
    assert (rel <= 1e-2).mean() >= 0.95, rel
    assert diff.check_status(ctx) == 0


def test_adam_fit_reduces_loss(fp32_scene):
    from voxviz_b200 import diff
    sc, _ = fp32_scene
    ctx = vv.Context(0)
    ctx.upload_nodes(sc.words)
    ctx.set_jitter(sc.jitter)
    clean = torch.from_numpy(_pool_f32(sc).copy()).cuda()
    gen = torch.Generator(device="cuda").manual_seed(5)
    noisy = clean + 0.05 * torch.randn(clean.shape, generator=gen, device="cuda")
    us = [sc.uniforms(sc.view(s, 128, 128)) for s in (3, 5, 7, 9)]
    with torch.no_grad():
        target = diff.render(noisy.contiguous(), ctx, sc.slots, us)
    pool = clean.clone().requires_grad_(True)
    opt = torch.optim.Adam([pool], lr=1e-2)
    losses = []
    for _ in range(12):
        opt.zero_grad()
        c = diff.render(pool, ctx, sc.slots, us)
        loss = ((c - target) ** 2).mean()
        loss.backward()
        opt.step()
        losses.append(float(loss.detach()))
    assert diff.check_status(ctx) == 0
    assert losses[-1] < 0.5 * losses[0], losses


def test_attach_rejects_misaligned_and_bad_shapes(fp32_scene):
    from voxviz_b200 import diff
    sc, _ = fp32_scene
    ctx = vv.Context(0)
    buf = torch.zeros(int(np.prod(sc.slots)) * 1000 * 4 + 1, dtype=torch.float32, device="cuda")
    with pytest.raises(vv.VVError):
        ctx.attach_bricks(buf.data_ptr() + 4, sc.slots, "fp32")
    with pytest.raises(ValueError):
        diff.attach_pool(ctx, buf, sc.slots)
