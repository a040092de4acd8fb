"""The renderer plugin path with paging: every frame's node-usage lists,
selection mask and compacted page requests are bit-exact against the oracle
run on the same device pools, and the deterministic LRU service leaves the
same residency and node words as the policy restatement."""
import numpy as np
import pytest

import voxviz_b200 as vv
from oracle import gv_oracle as go
from oracle.paging_ref import PagingRef
from voxviz_b200 import scene
from tests import helpers

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("fmt,device_paging", [("rgba8", False), ("fp16", False), ("rgba8", True),
                                               ("bf16", True), ("dxt5", True), ("dxt5", False)])
def test_paged_camera_path_matches_oracle_and_policy(fmt, device_paging):
    depth, W, H, frames = 6, 256, 160, 12
    o = helpers.octree(seed=3, depth=depth)
    f = vv.fmt_code(fmt)
    pool_bricks = 700
    pool_bytes = pool_bricks * vv.BRICK_BYTES[f]
    slots = scene.slot_grid(pool_bricks)
    ctx = vv.Context(0)
    r = vv.Renderer(ctx, o, fmt=fmt, pool_bytes=pool_bytes, preload_all=False, alpha_stop=0.99, jitter_seed=7,
                    device_paging=device_paging)
    sim = PagingRef(o.node_words(), slots)
    sim.init(False)
    jit = vv.make_jitter(7)
    cams = scene.camera_path(5, o.heights(), frames, W, H)
    evicted = 0
    for cam in cams:
        words = ctx.download_nodes()
        assert np.array_equal(words, sim.words), f"node words diverged before frame {cam.frame}"
        pool = ctx.download_bricks()
        r.draw(cam)
        u = r.last_uniforms()
        assert tuple(int(v) // 10 for v in u.brick_pool_dimension) == slots
        usage, mask = r.read_lists()
        ref = helpers.oracle_frame(u, go.Scene(words, pool, slots, f, jit), max_push=4 * (cam.frame % 3 + 1))
        assert np.array_equal(usage, ref["usage"]), f"usage lists differ at frame {cam.frame}"
        assert np.array_equal(mask, ref["mask"])
        col = r.read_color()
        assert np.abs(col - ref["color"]).max() <= 1 / 255
        r.update()
        req = r.last_requests()
        assert np.array_equal(req, ref["requests"]), f"page requests differ at frame {cam.frame}"
        sim.update(ref["requests"])
        xyz, slot = r.residency()
        got = {tuple(int(v) for v in p): int(s) for p, s in zip(xyz, slot)}
        assert got == sim.residency(), f"residency differs after frame {cam.frame}"
        assert np.array_equal(r.lru_order(), sim.lru_order()), f"LRU order differs after frame {cam.frame}"
        st = r.stats()
        evicted = st["evictions_total"]
    assert evicted > 0, "the pool was never full: the check did not exercise eviction"
    # resident slots hold exactly the produced bricks of their nodes
    pool = ctx.download_bricks()
    xyz, slot = r.residency()
    sel = np.arange(0, len(slot), max(1, len(slot) // 50))
    assert np.array_equal(pool[slot[sel]], o.produce_bricks(xyz[sel], f))
    assert ctx.device_status() == 0
