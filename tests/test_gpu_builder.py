"""The terrain octree built on the GPU (vv_octree_build_terrain_gpu: the
fBm heightfield, the column-run 2x2x2 box-filter mip pyramid with
round-half-up, GigaVoxelsOctTree.cpp:809-960, and the node classification
with the border rule, Node::computeNodeType :1490-1609) is the host build,
bit for bit: heights, every mip level, node words, and the bricks produced
from its pyramid - at depths 3 to 10 (config 2's 8192^3 tree included)."""
import numpy as np
import pytest

import voxviz_b200 as vv
from oracle.paging_ref import PagingRef

pytestmark = pytest.mark.gpu


def _nonconst_sample(words, n, seed):
    ref = PagingRef(words, (1, 1, 1))
    w0 = words[..., 0].reshape(-1)
    cand = np.nonzero(ref.valid_flat & ((w0 & np.uint32(0x40000000)) == 0))[0]
    rng = np.random.default_rng(seed)
    pick = np.sort(rng.choice(cand, size=min(n, len(cand)), replace=False))
    dz, dy, dx, _ = words.shape
    return np.stack([pick % dx, (pick // dx) % dy, pick // (dx * dy)], axis=1).astype(np.uint32)


def _same_tree(host, gpu, depth, dense_mips, bricks=1500):
    hi, gi = host.info, gpu.info
    assert (hi.node_count, tuple(hi.pool_dim), hi.nonconst_count, hi.root_word0, hi.root_word1) == \
           (gi.node_count, tuple(gi.pool_dim), gi.nonconst_count, gi.root_word0, gi.root_word1)
    words = host.node_words()
    assert np.array_equal(words, gpu.node_words())
    assert np.array_equal(host.heights(), gpu.heights())
    if dense_mips:
        for m in range(depth + 1):
            assert np.array_equal(host.mip_level(m), gpu.mip_level(m)), f"mip level {m}"
    xyz = _nonconst_sample(words, bricks, depth)
    assert np.array_equal(host.produce_bricks(xyz, "rgba8"), gpu.produce_bricks(xyz, "rgba8"))


@pytest.mark.parametrize("depth,collapse,seed", [(3, True, 2), (4, False, 5), (5, True, 1), (6, True, 3),
                                                 (6, False, 4)])
def test_gpu_build_equals_host_build(depth, collapse, seed):
    host = vv.Octree.terrain(seed=seed, depth=depth, collapse=collapse)
    gpu = vv.Octree.terrain(seed=seed, depth=depth, collapse=collapse, device=0)
    _same_tree(host, gpu, depth, dense_mips=True)


@pytest.mark.parametrize("depth", [8, 10])
def test_gpu_build_large(depth):
    host = vv.Octree.terrain(seed=1, depth=depth)
    gpu = vv.Octree.terrain(seed=1, depth=depth, device=0)
    _same_tree(host, gpu, depth, dense_mips=False)


def test_gpu_build_renders_like_host_build():
    """A renderer over the GPU-built tree draws and pages exactly as over the
    host-built one (usage lists, colour, residency)."""
    from voxviz_b200 import scene
    trees = [vv.Octree.terrain(seed=3, depth=6), vv.Octree.terrain(seed=3, depth=6, device=0)]
    cams = scene.camera_path(5, trees[0].heights(), 6, 192, 128)
    outs = []
    for o in trees:
        ctx = vv.Context(0)
        r = vv.Renderer(ctx, o, fmt="rgba8", pool_bytes=700 * 4000, preload_all=False, alpha_stop=0.99,
                        jitter_seed=7, device_paging=True)
        frames = []
        for cam in cams:
            r.draw(cam)
            usage, _ = r.read_lists()
            frames.append((r.read_color(), usage))
            r.update()
        outs.append((frames, r.residency()))
        r.close()
        ctx.close()
    for (ca, ua), (cb, ub) in zip(outs[0][0], outs[1][0]):
        assert np.array_equal(ca, cb) and np.array_equal(ua, ub)
    assert np.array_equal(outs[0][1][0], outs[1][1][0]) and np.array_equal(outs[0][1][1], outs[1][1][1])
