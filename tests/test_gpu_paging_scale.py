"""The paged 8192^3 terrain at full scale (depth 10, 1920x1080, the 2 GiB
RGBA8 pool of 538,002 slots, the seeded 256-frame path) through the
renderer plugin path with device paging.

Every checked frame's full-frame node-usage lists, selection mask and
compacted page requests are bit-exact against the FP32 oracle run on the
pools downloaded before the draw, its colour is within 1/255 of the oracle's,
and after the page-request service the node words (all 40.2 M nodes) and the
brick residency equal the paging-policy restatement.  Between the checked
stretches, frames further along the path fill the pool until the LRU evicts,
with the node words and residency still checked after every service (the
requests fed to the restatement are the GPU's, which the checked frames show
equal to the oracle's).

The reference path: GigaVoxelsNoLighting.frag:490-751 (ray cast),
CompressNodeUsageList.frag:44-150 (compaction),
NodeUsageListProcessor::run (GigaVoxelsOctTree.cpp:430-657) and
BrickPool::update (GigaVoxelsBrickPool.cpp:561-682) (service).
"""
import numpy as np
import pytest

import voxviz_b200 as vv
from oracle import gv_oracle as go
from oracle.paging_ref import PagingRef
from voxviz_b200 import scene
from tests import helpers

pytestmark = pytest.mark.gpu

DEPTH, W, H, PATH_FRAMES = 10, 1920, 1080, 256
POOL_BYTES = 2 << 30


def _check_policy(r, ctx, sim, frame):
    words = ctx.download_nodes()
    assert np.array_equal(words, sim.words), f"node words differ from the policy after frame {frame}"
    xyz, slot = r.residency()
    got = {(int(p[0]), int(p[1]), int(p[2])): int(s) for p, s in zip(xyz, slot)}
    assert got == sim.residency(), f"residency differs from the policy after frame {frame}"
    assert np.array_equal(r.lru_order(), sim.lru_order()), f"LRU order differs from the policy after frame {frame}"
    return words


def _checked_frame(r, ctx, sim, cam, words, slots, jit):
    pool = ctx.download_bricks()
    r.draw(cam)
    u = r.last_uniforms()
    usage, mask = r.read_lists()
    ref = helpers.oracle_frame(u, go.Scene(words, pool, slots, vv.VV_FMT_RGBA8, jit),
                               max_push=4 * (cam.frame % 3 + 1))
    assert ref["status"] == 0
    assert np.array_equal(usage, ref["usage"]), f"usage lists differ at frame {cam.frame}"
    assert np.array_equal(mask, ref["mask"]), f"selection masks differ at frame {cam.frame}"
    col = r.read_color()
    assert np.abs(col - ref["color"]).max() <= 1 / 255, f"colour differs at frame {cam.frame}"
    del pool
    r.update()
    req = r.last_requests()
    assert np.array_equal(req, ref["requests"]), f"page requests differ at frame {cam.frame}"
    sim.update(ref["requests"])
    return int((usage != 0).sum()), int(req.shape[0])


def test_config2_frames_bitexact_at_full_scale():
    o = vv.Octree.terrain(seed=1, depth=DEPTH)
    assert o.info.depth == DEPTH
    cams = scene.camera_path(2026, o.heights(), PATH_FRAMES, W, H)
    ctx = vv.Context(0)
    r = vv.Renderer(ctx, o, fmt="rgba8", pool_bytes=POOL_BYTES, preload_all=False, alpha_stop=0.99, jitter_seed=7,
                    device_paging=True)
    slots = tuple(ctx.slots)
    assert slots[0] * slots[1] * slots[2] == 538002
    sim = PagingRef(o.node_words(), slots)
    sim.init(False)
    jit = vv.make_jitter(7)
    words = _check_policy(r, ctx, sim, -1)
    # four consecutive frames from the cold start, every output checked
    entries = requests = 0
    for f in range(4):
        e, q = _checked_frame(r, ctx, sim, cams[f], words, slots, jit)
        entries += e
        requests += q
        words = _check_policy(r, ctx, sim, f)
    assert entries > 1_000_000 and requests > 10_000
    # fill the pool along the path until the LRU evicts (service checked
    # against the policy after every frame)
    f = 4
    while r.stats()["evictions_total"] == 0 and f < 4 + 60 * 4:
        r.draw(cams[f % PATH_FRAMES])
        r.update()
        sim.update(r.last_requests())
        words = _check_policy(r, ctx, sim, f)
        f += 4
    assert r.stats()["evictions_total"] > 0, "the 2 GiB pool never filled: eviction was not exercised"
    # two consecutive frames with the pool full, every output checked
    for k in range(2):
        _checked_frame(r, ctx, sim, cams[(f + k) % PATH_FRAMES], words, slots, jit)
        words = _check_policy(r, ctx, sim, f + k)
    # the 10-bit pool coordinates reach the far corner of the pool
    _, slot = r.residency()
    assert int(slot.max()) == 538001
    assert ctx.device_status() == 0
    r.close()
    ctx.close()
