"""The N>1 paths on CPU: two gloo ranks (127.0.0.1) split a camera path
and a view set without overlap, reduce a timing to the maximum over ranks,
and take a data-parallel fit step over split views whose summed ray-cast
gradient (the oracle's adjoint) and Adam update equal the single-process
ones."""
import os
import socket

import pytest
import torch
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    from voxviz_b200 import dist

    assert dist.init(backend="gloo", timeout_s=60)
    r, _, w = dist.env()
    first, count = dist.path_segment(r, w, 256)
    views = dist.views_of_rank(16, r, w)
    slowest = dist.max_over_ranks(10.0 + 5.0 * r)
    g = torch.full((4, 1000, 4), float(r + 1))
    dist.sum_gradients(g)
    dist.barrier()
    out.put((r, first, count, views, slowest, float(g[0, 0, 0]), float(g.sum())))
    dist.shutdown()


@pytest.mark.timeout(180)
def test_two_gloo_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=150) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    frames = []
    views = []
    for r, first, count, v, slowest, g0, gsum in res:
        frames += list(range(first, first + count))
        views += v
        assert slowest == 15.0            # max over ranks
        assert g0 == 3.0                  # 1 + 2
        assert gsum == 3.0 * 4 * 1000 * 4
    assert frames == list(range(256))     # the path is split, every frame once
    assert sorted(views) == list(range(16))


def _fit_rank(rank: int, world: int, port: int, out):
    """One data-parallel fit step as the fit workload takes it: this rank's
    views, its share of the mean L2 image loss over all views, the texel
    gradient of the ray cast (the oracle's binary64 adjoint of the binary32
    ray cast) summed over ranks, one Adam step on the brick pool."""
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    from voxviz_b200 import dist

    assert dist.init(backend="gloo", timeout_s=60)
    sc, us, target, pool = _fit_problem()
    mine = dist.views_of_rank(len(us), rank, world)
    grad = torch.from_numpy(_view_gradients(sc, us, target, mine))
    dist.sum_gradients(grad)
    p = torch.from_numpy(pool.copy()).requires_grad_(True)
    opt = torch.optim.Adam([p], lr=0.01)
    p.grad = grad.clone()
    opt.step()
    out.put((rank, grad.numpy(), p.detach().numpy()))
    dist.shutdown()


def _fit_problem():
    """A depth-4 terrain with FP32 bricks, 5 small seeded views and seeded
    target images."""
    import numpy as np

    from tests import helpers

    sc = helpers.Scene(seed=2, depth=4, fmt="fp32")
    us = [sc.uniforms(sc.view(20 + v, 40, 28)) for v in range(5)]
    rng = np.random.default_rng(9)
    target = rng.uniform(0, 1, (len(us), 28, 40, 4))
    pool = np.ascontiguousarray(sc.pool).view(np.float32).reshape(sc.pool.shape[0], 1000, 4).astype(np.float64)
    return sc, us, target, pool


def _view_gradients(sc, us, target, views):
    """dL/d(texel) (binary64) of L = sum over all views of |c - t|^2 / numel,
    restricted to the given views."""
    import numpy as np

    from oracle import gv_oracle as go

    osc = sc.oracle_scene()
    grad = np.zeros((sc.pool.shape[0], 1000, 4), dtype=np.float64)
    for v in views:
        c, _, _ = go.raycast(us[v], osc, 32, want_usage=False)
        dl = (2.0 * (c.astype(np.float64) - target[v]) / target.size).astype(np.float32)
        go.backward(us[v], osc, dl, grad=grad)
    return grad


@pytest.mark.timeout(300)
def test_data_parallel_fit_step_equals_single_process():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_fit_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=250) for _ in range(world)), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    sc, us, target, pool = _fit_problem()
    grad = torch.from_numpy(_view_gradients(sc, us, target, range(len(us))))
    assert float(grad.abs().max()) > 0
    p = torch.from_numpy(pool.copy()).requires_grad_(True)
    opt = torch.optim.Adam([p], lr=0.01)
    p.grad = grad.clone()
    opt.step()
    for _, g, after in res:
        # the same sums in another order: equal to binary64 rounding
        assert torch.allclose(torch.from_numpy(g), grad, rtol=1e-12, atol=1e-14 * float(grad.abs().max()))
        assert torch.allclose(torch.from_numpy(after), p.detach(), rtol=1e-12, atol=1e-15)
