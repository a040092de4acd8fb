"""The allocation-free compaction entry point (vv_compact_requests_noalloc).

Callers that must not call cudaMalloc - allocator callbacks, real-time render
threads, frameworks that own all device memory - use this entry point; its
histopyramid lives in a fixed file-scope device array.  Here it is called
through the C ABI and compared with vv_render's selection + compaction passes
on the same node-usage lists, twice in a row (the array keeps the previous
call's contents, which must not leak into the next result).  This file is
collected last so that a failure here comes after every other test has run.
"""
import ctypes as C

import numpy as np
import pytest

import voxviz_b200 as vv
from voxviz_b200 import _native as N
from tests import helpers

pytestmark = pytest.mark.gpu


def _usage_for(g, u):
    import torch
    dev = torch.device("cuda", 0)
    usage = torch.zeros((u.height, u.width, 12), dtype=torch.int32, device=dev)
    g.ctx.render(u, usage=usage.data_ptr(), passes=vv.VV_PASS_RAYCAST)
    return usage


def _existing(g, u, usage, cap, max_push):
    import torch
    dev = usage.device
    mask = torch.zeros((u.height, u.width), dtype=torch.int32, device=dev)
    req = torch.zeros((max(cap, 1), 4), dtype=torch.int32, device=dev)
    cnt = torch.zeros(1, dtype=torch.int32, device=dev)
    g.ctx.render(u, usage=usage.data_ptr(), mask=mask.data_ptr(), requests=req.data_ptr(),
                 request_count=cnt.data_ptr(), request_cap=cap, compress_max_push=max_push,
                 passes=vv.VV_PASS_SELECT | vv.VV_PASS_COMPACT)
    g.ctx.synchronize()
    return mask, req, cnt


def _noalloc(u, usage, cap, max_push):
    import torch
    dev = usage.device
    mask = torch.full((u.height, u.width), -1, dtype=torch.int32, device=dev)
    req = torch.full((max(cap, 1), 4), -1, dtype=torch.int32, device=dev)
    cnt = torch.full((1,), -1, dtype=torch.int32, device=dev)
    rc = vv.lib().vv_compact_requests_noalloc(C.c_void_p(usage.data_ptr()), C.c_void_p(mask.data_ptr()), u.width,
                                              u.height, C.c_void_p(req.data_ptr()), C.c_void_p(cnt.data_ptr()), cap,
                                              max_push, C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == N.VV_OK, vv.lib().vv_last_error(None)
    torch.cuda.synchronize()
    return mask, req, cnt


def _same(a, b, cap):
    (ma, ra, ca), (mb, rb, cb) = a, b
    assert np.array_equal(ma.cpu().numpy(), mb.cpu().numpy())
    n = int(ca.item())
    assert n == int(cb.item())
    k = min(n, cap)
    assert np.array_equal(ra[:k].cpu().numpy(), rb[:k].cpu().numpy())
    return n


def test_noalloc_compaction_matches_render_passes_twice_in_a_row():
    sc = helpers.Scene(seed=2, depth=5)
    g = helpers.GpuScene(sc)
    # first call: a 1920x1080 frame, no cap
    u1 = sc.uniforms(sc.view(5, 1920, 1080, frame=1))
    usage1 = _usage_for(g, u1)
    n1 = _same(_existing(g, u1, usage1, 1920 * 1080, 8), _noalloc(u1, usage1, 1920 * 1080, 8), 1920 * 1080)
    assert n1 > 1000
    # second call: another view and an odd size with a small cap; the array
    # still holds the first call's pyramid
    u2 = sc.uniforms(sc.view(9, 333, 177, frame=2))
    usage2 = _usage_for(g, u2)
    n2 = _same(_existing(g, u2, usage2, 50, 12), _noalloc(u2, usage2, 50, 12), 50)
    assert n2 > 50


@pytest.mark.parametrize("w,h", [(1, 1), (1, 9), (9, 1), (2, 3), (5, 5), (64, 2)])
def test_noalloc_compaction_on_degenerate_frames(w, h):
    # one-level pyramids (1x1: no level 1, the count read from the mask),
    # and frames where only one dimension halves
    sc = helpers.Scene(seed=2, depth=5)
    g = helpers.GpuScene(sc)
    u = sc.uniforms(sc.view(5, w, h, frame=3))
    usage = _usage_for(g, u)
    cap = w * h
    _same(_existing(g, u, usage, cap, 8), _noalloc(u, usage, cap, 8), cap)


def test_noalloc_without_requests_or_count():
    import torch
    sc = helpers.Scene(seed=2, depth=5)
    g = helpers.GpuScene(sc)
    u = sc.uniforms(sc.view(7, 200, 120, frame=1))
    usage = _usage_for(g, u)
    m_ref, r_ref, c_ref = _existing(g, u, usage, 200 * 120, 4)
    # cap 0: mask and count only, no request written
    m0, r0, c0 = _noalloc(u, usage, 0, 4)
    assert np.array_equal(m0.cpu().numpy(), m_ref.cpu().numpy())
    assert int(c0.item()) == int(c_ref.item())
    assert bool((r0 == -1).all())
    # no count pointer: mask and requests only
    dev = usage.device
    mask = torch.full((u.height, u.width), -1, dtype=torch.int32, device=dev)
    req = torch.full((200 * 120, 4), -1, dtype=torch.int32, device=dev)
    rc = vv.lib().vv_compact_requests_noalloc(C.c_void_p(usage.data_ptr()), C.c_void_p(mask.data_ptr()), u.width,
                                              u.height, C.c_void_p(req.data_ptr()), None, 200 * 120, 4,
                                              C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == N.VV_OK, vv.lib().vv_last_error(None)
    torch.cuda.synchronize()
    n = int(c_ref.item())
    assert np.array_equal(mask.cpu().numpy(), m_ref.cpu().numpy())
    assert np.array_equal(req[:n].cpu().numpy(), r_ref[:n].cpu().numpy())
    assert bool((req[n:] == -1).all())


def test_noalloc_rejects_frames_beyond_its_array():
    import torch
    t = torch.zeros(16, dtype=torch.int32, device="cuda")
    p = C.c_void_p(t.data_ptr())
    rc = vv.lib().vv_compact_requests_noalloc(p, p, 4096, 1024, p, p, 1, 4, None)
    assert rc == N.VV_ERR_ARG
    assert b"VV_NOALLOC_MAX_PIXELS" in vv.lib().vv_last_error(None)
