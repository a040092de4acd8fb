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


def test_fixed_path_matches_fp32_cast_to_rounding():
    """The binary64 re-evaluation of the binary32 sample sequence differs from
    the binary32 colour only by binary32 rounding."""
    from oracle import gv_oracle as go
    sc = helpers.Scene(seed=1, depth=5, fmt="fp16")
    u = sc.uniforms(sc.view(7, 64, 48))
    os_ = sc.oracle_scene()
    c32, _, _ = go.raycast(u, os_, 32, want_usage=False)
    c64 = go.fixed_path(u, os_)
    assert np.abs(c64 - c32).max() <= 2e-5


def test_fixed_path_central_differences_match_backward():
    """Finite differences of the fixed-trajectory binary64 colour (a smooth
    function of the texels) against the binary64 adjoint: the tight check."""
    from oracle import gv_oracle as go
    sc = helpers.Scene(seed=1, depth=5, fmt="fp32")
    u = sc.uniforms(sc.view(11, 40, 32))
    pool = np.ascontiguousarray(sc.pool).view(np.float32).reshape(sc.pool.shape[0], 1000, 4).copy()
    traj = sc.oracle_scene(pool=pool.copy())
    vals_pool = pool.copy()
    vals = sc.oracle_scene(pool=vals_pool)
    rng = np.random.default_rng(2)
    w = rng.standard_normal((u.height, u.width, 4)).astype(np.float32)
    g = go.backward(u, traj, w)
    nz = np.argwhere(g != 0)
    pick = nz[rng.choice(len(nz), size=24, replace=False)]
    h = 1e-3
    for s, t, ch in pick:
        old = vals_pool[s, t, ch]
        vals_pool[s, t, ch] = old + h
        c1 = go.fixed_path(u, traj, vals)
        vals_pool[s, t, ch] = old - h
        c2 = go.fixed_path(u, traj, vals)
        vals_pool[s, t, ch] = old
        fd = float(((c1 - c2) * w.astype(np.float64)).sum() / (float(np.float32(old + h)) - float(np.float32(old - h))))
        assert abs(fd - g[s, t, ch]) <= 1e-4 * max(abs(g[s, t, ch]), 1e-3 * np.abs(g).max()), (fd, g[s, t, ch])
