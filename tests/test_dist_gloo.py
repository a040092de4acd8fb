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
