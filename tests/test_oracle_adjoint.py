"""The oracle's binary64 adjoint against central finite differences of its
binary64 forward (h = 1e-3) on the largest texel gradients of a small view.
This pins the reference gradient the GPU adjoint is compared with."""
import numpy as np

from tests import helpers


def test_oracle_backward_matches_central_differences():
    from oracle import gv_oracle as go
    sc = helpers.Scene(seed=1, depth=5, fmt="fp32")
    u = sc.uniforms(sc.view(3, 48, 32))
    pool = np.ascontiguousarray(sc.pool).view(np.float32).reshape(sc.pool.shape[0], 1000, 4).copy()
    os_ = sc.oracle_scene(pool=pool)
    rng = np.random.default_rng(0)
    w = rng.standard_normal((u.height, u.width, 4)).astype(np.float32)
    g = go.backward(u, os_, w)
    assert np.count_nonzero(g) > 0
    h = 1e-3
    for i in np.argsort(-np.abs(g).ravel())[:8]:
        s, t, ch = np.unravel_index(i, g.shape)
        p1 = pool.copy()
        p1[s, t, ch] += h
        p2 = pool.copy()
        p2[s, t, ch] -= h
        c1, _, _ = go.raycast(u, sc.oracle_scene(pool=p1), 64, want_usage=False)
        c2, _, _ = go.raycast(u, sc.oracle_scene(pool=p2), 64, want_usage=False)
        fd = float(((c1 - c2) * w.astype(np.float64)).sum() / (2 * h))
        assert abs(fd - g[s, t, ch]) <= 1e-3 * abs(fd), (s, t, ch, fd, g[s, t, ch])


def test_oracle_backward_is_linear_in_dl_dcolor():
    from oracle import gv_oracle as go
    sc = helpers.Scene(seed=1, depth=5, fmt="fp32")
    u = sc.uniforms(sc.view(5, 40, 24))
    os_ = sc.oracle_scene()
    rng = np.random.default_rng(1)
    a = rng.standard_normal((u.height, u.width, 4)).astype(np.float32)
    b = rng.standard_normal((u.height, u.width, 4)).astype(np.float32)
    ga, gb = go.backward(u, os_, a), go.backward(u, os_, b)
    gab = go.backward(u, os_, (a + b).astype(np.float32))
    scale = np.abs(gab).max()
    assert np.abs(gab - (ga + gb)).max() <= 1e-6 * scale
