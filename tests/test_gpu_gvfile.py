"""A tree read from .gvx/.gvb files (the offline voxelizer's layout, edge
bricks with border 0) through the renderer plugin path: every frame's usage
lists, selection mask and page requests bit-exact against the oracle run on
the same device pools, the LRU service against the policy restatement with
the bricks' borders, host and device paging; and a terrain written to files
and read back renders bit-identically to the terrain itself."""
import numpy as np
import pytest

import voxviz_b200 as vv
from oracle import gv_oracle as go
from oracle import gvfile_ref as gr
from oracle.paging_ref import PagingRef
from voxviz_b200 import scene
from tests import gvx_fixtures as gf
from tests import helpers

pytestmark = pytest.mark.gpu

SEED, DEPTH = 3, 5


@pytest.fixture(scope="module")
def dataset(tmp_path_factory):
    d = tmp_path_factory.mktemp("voxelizer")
    gf.write_voxelizer_style(str(d), seed=SEED, depth=DEPTH)
    return str(d / "tree.gvx")


@pytest.mark.parametrize("fmt,device_paging", [("rgba8", False), ("rgba8", True), ("fp16", True)])
def test_file_tree_paged_path_matches_oracle_and_policy(dataset, fmt, device_paging):
    W, H, frames = 256, 160, 10
    ref = gr.load_gvx(dataset, constant_colors=True)
    o = vv.Octree.load_gvx(dataset, constant_colors=True)
    f = vv.fmt_code(fmt)
    pool_bricks = 500
    slots = scene.slot_grid(pool_bricks)
    ctx = vv.Context(0)
    r = vv.Renderer(ctx, o, fmt=fmt, pool_bytes=pool_bricks * 1000 * vv.TEXEL_BYTES[f], preload_all=False,
                    alpha_stop=0.99, jitter_seed=7, device_paging=device_paging)
    borders = {k: tuple(int(v) for v in b["border"]) for k, b in ref["bricks"].items()}
    sim = PagingRef(o.node_words(), slots, borders=borders)
    sim.init(False)
    jit = vv.make_jitter(7)
    heights = helpers.octree(seed=SEED, depth=DEPTH).heights()
    cams = scene.camera_path(5, heights, frames, W, H)
    offset_bricks = 0
    for cam in cams:
        words = ctx.download_nodes()
        assert np.array_equal(words, sim.words), f"node words diverged before frame {cam.frame}"
        pool = ctx.download_bricks()
        r.draw(cam)
        u = r.last_uniforms()
        usage, mask = r.read_lists()
        oref = helpers.oracle_frame(u, go.Scene(words, pool, slots, f, jit), max_push=4 * (cam.frame % 3 + 1))
        assert np.array_equal(usage, oref["usage"]), f"usage lists differ at frame {cam.frame}"
        assert np.array_equal(mask, oref["mask"])
        col = r.read_color()
        assert np.abs(col - oref["color"]).max() <= 1 / 255
        r.update()
        req = r.last_requests()
        assert np.array_equal(req, oref["requests"]), f"page requests differ at frame {cam.frame}"
        sim.update(oref["requests"])
        xyz, slot = r.residency()
        got = {tuple(int(v) for v in p): int(s) for p, s in zip(xyz, slot)}
        assert got == sim.residency(), f"residency differs after frame {cam.frame}"
        offset_bricks = max(offset_bricks, sum(1 for p in got if borders[p] != (1, 1, 1)))
    assert r.stats()["evictions_total"] > 0, "the pool was never full"
    assert offset_bricks > 0, "no brick with a border other than 1 was resident"
    pool = ctx.download_bricks()
    xyz, slot = r.residency()
    sel = np.arange(0, len(slot), max(1, len(slot) // 60))
    assert np.array_equal(pool[slot[sel]], o.produce_bricks(xyz[sel], f))
    assert ctx.device_status() == 0


@pytest.mark.parametrize("device_paging", [False, True])
def test_terrain_files_render_like_the_terrain(tmp_path, device_paging):
    W, H, frames = 320, 200, 6
    t = helpers.octree(seed=SEED, depth=DEPTH)
    t.save_gvx(tmp_path)
    o = vv.Octree.load_gvx(tmp_path / "tree.gvx", constant_colors=True)
    assert np.array_equal(o.node_words(), t.node_words())
    pool_bytes = 600 * 1000 * 4
    out = []
    for tree in (t, o):
        ctx = vv.Context(0)
        r = vv.Renderer(ctx, tree, fmt="rgba8", pool_bytes=pool_bytes, preload_all=False, alpha_stop=0.99,
                        jitter_seed=7, device_paging=device_paging)
        frames_out = []
        for cam in scene.camera_path(11, t.heights(), frames, W, H):
            r.draw(cam)
            col = r.read_color()
            r.update()
            frames_out.append((col, r.last_requests(), ctx.download_nodes()))
        assert ctx.device_status() == 0
        out.append(frames_out)
    for k, ((c0, q0, w0), (c1, q1, w1)) in enumerate(zip(*out)):
        assert np.array_equal(c0, c1), f"colour differs at frame {k}"
        assert np.array_equal(q0, q1), f"requests differ at frame {k}"
        assert np.array_equal(w0, w1), f"node words differ after frame {k}"
