"""Adjoint of the ray cast (vv_render_forward_ckpt / vv_backward) and its
torch.autograd.Function.

* the checkpointing forward gives vv_render's colour bit for bit;
* dL/d(texel) matches the oracle's binary64 adjoint of the same binary32
  ray cast to 1e-3 relative (per texel, for texels above 1e-3 of the largest
  gradient; FP32 atomics are the only difference);
* binary64 accumulation (VV_GRAD_F64) and the sparse gradient (rows per
  touched slot) give the dense gradient;
* with binary64 accumulation the gradient matches central differences
  (h = 1e-3) of the binary64 functional along the fixed control flow within
  1e-3 relative on random texels;
* the autograd gradient matches central differences of the binary32 GPU
  forward within 1e-3 relative plus that forward's rounding, probes that
  change the control flow set aside;
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


def _backward_variants(g, u, ck, per_ray, dl_t, n_slots):
    """The adjoint of one view several ways: dense float, dense binary64,
    and sparse rows (slot map) in float and in binary64, in float with cell
    warp sums, with the atomics spread over copies of the rows, and with
    both; the sparse ones are scattered back to slots.  Returns {name:
    (slots, 1000, 4) float64} and the rows each sparse call claimed."""
    dev = torch.device("cuda", 0)
    out, rows = {}, {}
    dense = torch.zeros((n_slots, 1000, 4), dtype=torch.float32, device=dev)
    g.ctx.backward(u, dl_t.data_ptr(), ck.data_ptr(), per_ray, dense.data_ptr())
    out["dense_f32"] = dense.double()
    d64 = torch.zeros((n_slots, 1000, 4), dtype=torch.float64, device=dev)
    g.ctx.backward_ex(u, dl_t.data_ptr(), ck.data_ptr(), per_ray, d64.data_ptr(), f64=True)
    out["dense_f64"] = d64
    forms = {"rows_f32": {}, "rows_f64": {"f64": True}, "rows_f32_warp_sum": {"warp_sum": True},
             "rows_f32_spread": {"spread": True}, "rows_f32_spread_warp_sum": {"spread": True, "warp_sum": True}}
    for name, kw in forms.items():
        cap = n_slots
        rowbuf = torch.zeros((cap, 1000, 4), dtype=torch.float64 if kw.get("f64") else torch.float32, device=dev)
        smap = torch.full((n_slots,), -1, dtype=torch.int32, device=dev)
        used = torch.zeros(1, dtype=torch.int32, device=dev)
        g.ctx.backward_ex(u, dl_t.data_ptr(), ck.data_ptr(), per_ray, rowbuf.data_ptr(),
                          slot_map=smap.data_ptr(), rows_used=used.data_ptr(), rows_cap=cap, **kw)
        torch.cuda.synchronize()
        n = int(used.item())
        m = smap.cpu().numpy()
        assert set(np.unique(m[m >= 0])) == set(range(n))       # rows 0..n-1, one slot each
        full = torch.zeros((n_slots, 1000, 4), dtype=torch.float64, device=dev)
        sl = torch.from_numpy(np.nonzero(m >= 0)[0]).to(dev)
        full[sl] = rowbuf[smap[sl].long()].double()
        out[name] = full
        rows[name] = n
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in out.items()}, rows


def test_backward_binary64_and_sparse_rows(fp32_scene):
    """vv_backward_ex: binary64 accumulation and the sparse gradient (rows
    claimed by touched slots) give the dense gradient; the binary64 one
    matches the oracle's binary64 adjoint within 1e-3 relative on every
    texel, apart from the binary32 rounding of its per-sample terms
    (bounded by 1e-5 times the texel's sum of term magnitudes, which the
    oracle returns: a texel whose terms cancel to a tiny sum keeps the
    absolute error of its large terms)."""
    from oracle import gv_oracle as go
    sc, g = fp32_scene
    n_slots = int(np.prod(sc.slots))
    for seed, (w, h) in ((5, (96, 64)), (8, (160, 120))):
        u = sc.uniforms(sc.view(seed, w, h))
        _, ck = _ckpt_color(g, u, 16)
        rng = np.random.default_rng(seed)
        dl = rng.standard_normal((h, w, 4)).astype(np.float32)
        dl_t = torch.from_numpy(dl).cuda()
        got, rows = _backward_variants(g, u, ck, 16, dl_t, n_slots)
        assert g.ctx.device_status() == 0
        ref_abs = np.zeros((n_slots, 1000, 4), dtype=np.float64)
        ref = go.backward(u, sc.oracle_scene(), dl, grad_abs=ref_abs)
        scale = np.abs(ref).max()
        touched = np.abs(ref).reshape(n_slots, -1).max(axis=1) > 0
        for name, v in got.items():
            assert np.array_equal(v != 0, ref != 0), name
            assert np.abs(v - ref).max() <= 1e-5 * scale, (name, np.abs(v - ref).max() / scale)
        for name, n in rows.items():
            assert n >= int(touched.sum()) and n <= n_slots
        # binary64 accumulation: every texel, however small its gradient
        nz = ref != 0
        err = np.abs(got["dense_f64"] - ref)[nz]
        assert (err <= 1e-3 * np.abs(ref)[nz] + 1e-5 * ref_abs[nz]).all()
        cond = ref_abs[nz] / np.abs(ref)[nz]
        # where the terms do not cancel (magnitude within 10x of the sum) the
        # plain relative error is far below 1e-3
        assert (err / np.abs(ref)[nz])[cond <= 10].max() <= 1e-4


def test_spread_copies_stay_zero_between_calls(fp32_scene):
    """VV_GRAD_SPREAD: the context's extra copies of the rows are added
    into the caller's rows and left zero, so repeated calls - with other row
    capacities, after an overflow, and after a call without spreading - give
    the same gradient as plain atomics; it needs a slot map and binary32
    rows."""
    sc, g = fp32_scene
    u = sc.uniforms(sc.view(8, 160, 120))
    _, ck = _ckpt_color(g, u, 16)
    rng = np.random.default_rng(3)
    dl_t = torch.from_numpy(rng.standard_normal((120, 160, 4)).astype(np.float32)).cuda()
    n_slots = int(np.prod(sc.slots))
    dev = torch.device("cuda", 0)

    def run(cap, **kw):
        rowbuf = torch.zeros((cap, 1000, 4), dtype=torch.float32, device=dev)
        smap = torch.full((n_slots,), -1, dtype=torch.int32, device=dev)
        used = torch.zeros(1, dtype=torch.int32, device=dev)
        g.ctx.backward_ex(u, dl_t.data_ptr(), ck.data_ptr(), 16, rowbuf.data_ptr(), slot_map=smap.data_ptr(),
                          rows_used=used.data_ptr(), rows_cap=cap, **kw)
        torch.cuda.synchronize()
        m = smap.cpu().numpy()
        full = np.zeros((n_slots, 1000, 4), dtype=np.float64)
        sl = np.nonzero(m >= 0)[0]
        full[sl] = rowbuf.cpu().numpy()[m[sl]]
        return full

    ref = run(n_slots)
    scale = np.abs(ref).max()
    touched = int((np.abs(ref).reshape(n_slots, -1).max(axis=1) > 0).sum())
    for cap in (n_slots, touched + 3, n_slots // 2 + touched, touched):
        got = run(cap, spread=True)
        assert g.ctx.device_status() == 0
        assert np.array_equal(got != 0, ref != 0)
        assert np.abs(got - ref).max() <= 1e-5 * scale
    # an overflowing call drops contributions but leaves the copies clean
    run(2, spread=True)
    from voxviz_b200 import _native as N
    assert g.ctx.device_status(clear=True) == N.VV_ERR_OOM
    got = run(n_slots, spread=True, warp_sum=True)
    assert g.ctx.device_status() == 0
    assert np.abs(got - ref).max() <= 1e-5 * scale
    with pytest.raises(vv.VVError):
        run(n_slots, spread=True, f64=True)
    with pytest.raises(vv.VVError):
        run(n_slots, keep=True)


def test_spread_dense_rows_and_kept_sums(fp32_scene):
    """VV_GRAD_SPREAD on dense rows (one row per pool slot), and
    VV_GRAD_SPREAD_KEEP: two views whose copies are reduced once give the
    sum of the two views' plain gradients."""
    sc, g = fp32_scene
    n_slots = int(np.prod(sc.slots))
    dev = torch.device("cuda", 0)
    views = []
    for seed, (w, h) in ((5, (96, 64)), (8, (160, 120))):
        u = sc.uniforms(sc.view(seed, w, h))
        _, ck = _ckpt_color(g, u, 16)
        rng = np.random.default_rng(seed)
        views.append((u, ck, torch.from_numpy(rng.standard_normal((h, w, 4)).astype(np.float32)).cuda()))
    ref = torch.zeros((n_slots, 1000, 4), dtype=torch.float32, device=dev)
    for u, ck, dl in views:
        g.ctx.backward(u, dl.data_ptr(), ck.data_ptr(), 16, ref.data_ptr())
    one = torch.zeros_like(ref)
    u, ck, dl = views[0]
    g.ctx.backward_ex(u, dl.data_ptr(), ck.data_ptr(), 16, one.data_ptr(), spread=True)
    two = torch.zeros_like(ref)
    for k, (u, ck, dl) in enumerate(views):
        g.ctx.backward_ex(u, dl.data_ptr(), ck.data_ptr(), 16, two.data_ptr(), spread=True, keep=k == 0)
    torch.cuda.synchronize()
    assert g.ctx.device_status() == 0
    ref_one = torch.zeros_like(ref)
    u0, ck0, dl0 = views[0]
    g.ctx.backward(u0, dl0.data_ptr(), ck0.data_ptr(), 16, ref_one.data_ptr())
    r1, o1, r2, o2 = (x.cpu().numpy().astype(np.float64) for x in (ref_one, one, ref, two))
    for r, o in ((r1, o1), (r2, o2)):
        scale = np.abs(r).max()
        assert scale > 0
        assert np.array_equal(r != 0, o != 0)
        assert np.abs(o - r).max() <= 1e-5 * scale


def test_sparse_rows_report_overflow(fp32_scene):
    """Fewer rows than touched slots: VV_ERR_OOM in the device status."""
    sc, g = fp32_scene
    u = sc.uniforms(sc.view(5, 96, 64))
    _, ck = _ckpt_color(g, u, 16)
    dl_t = torch.ones((64, 96, 4), dtype=torch.float32, device="cuda")
    n_slots = int(np.prod(sc.slots))
    rowbuf = torch.zeros((2, 1000, 4), dtype=torch.float32, device="cuda")
    smap = torch.full((n_slots,), -1, dtype=torch.int32, device="cuda")
    used = torch.zeros(1, dtype=torch.int32, device="cuda")
    g.ctx.backward_ex(u, dl_t.data_ptr(), ck.data_ptr(), 16, rowbuf.data_ptr(), slot_map=smap.data_ptr(),
                      rows_used=used.data_ptr(), rows_cap=2)
    g.ctx.synchronize()
    from voxviz_b200 import _native as N
    assert g.ctx.device_status(clear=True) == N.VV_ERR_OOM
    assert int((smap >= 0).sum()) == 2


def test_gradient_matches_central_differences_of_binary64_functional(fp32_scene):
    """The adjoint against central differences (h = 1e-3): dL/d(texel) of
    F = sum over pixels of dL/dc * c (dL/dc held at the forward's value, so
    its texel gradient is exactly what the adjoint returns) with c composited
    in binary64 along the binary32 sample sequence (the control flow the
    adjoint holds fixed), at 96 random texels with a non-zero gradient, not
    only the largest.  The GPU reduces its per-sample contributions in
    binary64 (VV_GRAD_F64).  Every texel within 1e-3 relative plus the
    binary32 rounding of its per-sample terms (1e-5 times the magnitude of
    the terms, from the oracle's adjoint)."""
    from oracle import gv_oracle as go
    sc, g = fp32_scene
    n_slots = int(np.prod(sc.slots))
    us = [sc.uniforms(sc.view(s, 128, 96)) for s in (3, 5)]
    rng = np.random.default_rng(0)
    targets = rng.uniform(0, 1, (2, 96, 128, 4))
    grad = torch.zeros((n_slots, 1000, 4), dtype=torch.float64, device="cuda")
    dls = []
    for u, t in zip(us, targets):
        c, ck = _ckpt_color(g, u, 16)
        dl = (2.0 * (c.double().cpu().numpy() - t)).astype(np.float32)
        dls.append(dl)
        g.ctx.backward_ex(u, torch.from_numpy(dl).cuda().data_ptr(), ck.data_ptr(), 16, grad.data_ptr(), f64=True)
    g.ctx.synchronize()
    assert g.ctx.device_status() == 0
    an_all = grad.cpu().numpy()
    mag = np.zeros((n_slots, 1000, 4), dtype=np.float64)
    ref = np.zeros((n_slots, 1000, 4), dtype=np.float64)
    for u, dl in zip(us, dls):
        go.backward(u, sc.oracle_scene(), dl, grad=ref, grad_abs=mag)
    nz = np.argwhere(an_all != 0)
    pick = nz[rng.choice(len(nz), size=96, replace=False)]
    traj = sc.oracle_scene()
    vals_pool = np.array(sc.pool, copy=True)
    flat = vals_pool.view(np.float32).reshape(-1)
    vals = sc.oracle_scene(pool=vals_pool)
    h = np.float32(1e-3)
    rel, ok = [], []
    for s_, t_, ch in pick:
        i = (int(s_) * 1000 + int(t_)) * 4 + int(ch)
        old = flat[i]
        flat[i] = old + h
        up = float(flat[i])
        f1 = sum(float((dl.astype(np.float64) * go.fixed_path(u, traj, vals)).sum()) for u, dl in zip(us, dls))
        flat[i] = old - h
        dn = float(flat[i])
        f2 = sum(float((dl.astype(np.float64) * go.fixed_path(u, traj, vals)).sum()) for u, dl in zip(us, dls))
        flat[i] = old
        fd = (f1 - f2) / (up - dn)
        an = float(an_all[s_, t_, ch])
        rel.append(abs(fd - an) / abs(fd))
        ok.append(abs(fd - an) <= 1e-3 * abs(fd) + 1e-5 * float(mag[s_, t_, ch]))
    rel = np.array(rel)
    assert all(ok), (rel.max(), np.median(rel))
    assert np.median(rel) <= 1e-5, np.median(rel)


def test_autograd_gradient_within_fp32_forward_resolution(fp32_scene):
    """The autograd gradient against central differences (h = 1e-3) of the
    binary32 GPU forward with the loss reduced in binary64 on the GPU.  A
    probe whose +-h renders change the control flow (a ray's composited
    sample count moves: the alpha stop crossed) has no derivative there and
    is set aside (counted); on the others the difference is within 1e-3
    relative plus the forward's binary32 rounding: a colour composited from
    n samples carries at most (3n+1) u |c| (three roundings per sample, u =
    2^-24), in each of the two renders: |dL/dc| * 2 (3n+1) u |c| per changed
    pixel, summed, over 2h."""
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
    dlc = (2.0 * (c.detach().double() - target.double())).abs()

    def samples(p):
        # composited sample count per pixel of every view (the checkpoint header)
        diff.attach_pool(ctx, p, sc.slots)
        out = []
        for u in us:
            col = torch.empty((96, 128, 4), dtype=torch.float32, device="cuda")
            ck = torch.empty(vv.Context.ckpt_bytes(128, 96, 4), dtype=torch.uint8, device="cuda")
            ctx.forward_ckpt(u, col.data_ptr(), ck.data_ptr(), 4)
            hdr = ck[: 96 * 128 * 8].view(torch.int32).view(96, 128, 2)[..., 1].clone()
            out.append((col, hdr))
        return out

    flat = grad.abs().flatten()
    nz = torch.nonzero(flat).flatten().cpu().numpy()
    idx = rng.choice(nz, size=64, replace=False)
    h = 1e-3
    base = pool.detach().clone()
    n_flip, checked = 0, 0
    with torch.no_grad():
        r0 = samples(base)
        for i in idx:
            p1 = base.clone().flatten()
            p1[i] += h
            p2 = base.clone().flatten()
            p2[i] -= h
            r1, r2 = samples(p1.view_as(base)), samples(p2.view_as(base))
            if any(not torch.equal(a[1], b[1]) or not torch.equal(a[1], c_[1]) for a, b, c_ in zip(r0, r1, r2)):
                n_flip += 1
                continue
            c1 = torch.stack([a[0] for a in r1])
            c2 = torch.stack([a[0] for a in r2])
            fd = float((loss64(c1) - loss64(c2)) / (2 * h))
            an = float(grad.flatten()[i])
            # binary32 rounding of the two renders, on the pixels that changed
            changed = (c1 != c2)
            n = torch.stack([a[1] for a in r0]).double().unsqueeze(-1)
            rnd = 2.0 * (3.0 * n + 1.0) * torch.abs(torch.stack([c1, c2])).max(0).values.double() * 2.0 ** -24
            floor = float((dlc * rnd)[changed].sum()) / (2 * h)
            assert abs(fd - an) <= 1e-3 * abs(an) + floor, (i, fd, an, floor)
            checked += 1
    assert checked >= 48, (checked, n_flip)
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
