"""The N>1 plumbing on CPU: two gloo ranks (127.0.0.1) split a camera path
and a view set without overlap, reduce a timing to the maximum over ranks,
and sum texel gradients the way data-parallel fitting does."""
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
    views, its share of the mean loss over all views, the texel gradient
    summed over ranks, one Adam step."""
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    from voxviz_b200 import dist

    assert dist.init(backend="gloo", timeout_s=60)
    views, param, target, proj = _fit_problem()
    mine = dist.views_of_rank(views, rank, world)
    p = param.clone().requires_grad_(True)
    opt = torch.optim.Adam([p], lr=0.1)
    c = torch.stack([proj[v] @ p for v in mine])
    loss = ((c - target[mine]) ** 2).sum() / target.numel()
    loss.backward()
    dist.sum_gradients(p.grad)
    grad = p.grad.clone()
    opt.step()
    out.put((rank, grad.numpy(), p.detach().numpy()))
    dist.shutdown()


def _fit_problem():
    g = torch.Generator().manual_seed(5)
    views = 5
    param = torch.rand(12, generator=g, dtype=torch.float64)
    proj = torch.rand(views, 7, 12, generator=g, dtype=torch.float64)
    target = torch.rand(views, 7, generator=g, dtype=torch.float64)
    return views, param, target, proj


@pytest.mark.timeout(180)
def test_data_parallel_fit_step_equals_single_process():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_fit_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=150) for _ in range(world)), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    views, param, target, proj = _fit_problem()
    p = param.clone().requires_grad_(True)
    opt = torch.optim.Adam([p], lr=0.1)
    c = torch.stack([proj[v] @ p for v in range(views)])
    ((c - target) ** 2).mean().backward()
    grad = p.grad.clone()
    opt.step()
    for _, g, after in res:
        assert torch.allclose(torch.from_numpy(g), grad, rtol=1e-12, atol=1e-15)
        assert torch.allclose(torch.from_numpy(after), p.detach(), rtol=1e-12, atol=1e-15)
