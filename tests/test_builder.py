"""The terrain octree builder against a dense restatement of the reference
builder (GigaVoxelsOctTree.cpp GenerateMipMaps / computeNodeType /
copyMipMapToBrick / BuildOctTree, OctTreeNodePool::create3DTexture)."""
import numpy as np
import pytest

import voxviz_b200 as vv
from oracle import terrain_ref as tr


@pytest.mark.parametrize("depth", [1, 2, 3, 4])
@pytest.mark.parametrize("collapse", [True, False])
@pytest.mark.parametrize("seed", [1, 5])
def test_builder_matches_dense_reference(depth, collapse, seed):
    o = vv.Octree.terrain(seed=seed, depth=depth, collapse=collapse)
    assert np.array_equal(o.heights(), tr.heights(seed, depth))
    mips = tr.mip_pyramid(tr.leaf_volume(seed, depth))
    assert len(mips) == depth + 1
    for level in range(depth + 1):
        assert np.array_equal(o.mip_level(level), mips[level]), f"mip level {level}"
    ref = tr.build_tree(mips, collapse=collapse)
    info = o.info
    assert info.node_count == ref["node_count"]
    assert tuple(info.pool_dim) == ref["pool_dim"]
    words = o.node_words()
    assert np.array_equal(words, ref["words"])
    xyz, expect = [], []
    for (gx, gy, gz), (lvl, i, j, k) in ref["nodes"].items():
        if not ref["words"][gz, gy, gx, 0] & 0x40000000:
            xyz.append((gx, gy, gz))
            expect.append(tr.copy_mip_to_brick(mips[depth - lvl], 8 * i, 8 * j, 8 * k))
        ni = o.node_info(gx, gy, gz)
        assert ni.valid and ni.level == lvl and tuple(ni.origin) == (8 * i, 8 * j, 8 * k)
    assert len(xyz) == info.nonconst_count
    got = o.produce_bricks(np.array(xyz, dtype=np.uint32), "rgba8").view(np.uint32).reshape(-1, 10, 10, 10)
    assert np.array_equal(got, np.array(expect))


def test_brick_formats_hold_normalized_values():
    o = vv.Octree.terrain(seed=3, depth=2)
    words = o.node_words()
    nz = np.argwhere((words[..., 0] & 0x40000000) == 0)
    xyz = np.array([[x, y, z] for z, y, x in nz if o.node_info(int(x), int(y), int(z)).valid][:16], dtype=np.uint32)
    b8 = o.produce_bricks(xyz, "rgba8").reshape(-1, 1000, 4).astype(np.float64)
    ref = (b8 / 255.0).astype(np.float32)
    f32 = o.produce_bricks(xyz, "fp32").view(np.float32).reshape(-1, 1000, 4)
    assert np.array_equal(f32, ref)
    f16 = o.produce_bricks(xyz, "fp16").view(np.float16).reshape(-1, 1000, 4)
    assert np.array_equal(f16, ref.astype(np.float16))
    bf = o.produce_bricks(xyz, "bf16").view(np.uint16).reshape(-1, 1000, 4)
    bits = ref.view(np.uint32)
    rne = ((bits + 0x7FFF + ((bits >> 16) & 1)) >> 16).astype(np.uint16)
    assert np.array_equal(bf, rne)


def test_node_pool_fits_ten_bit_grid_at_depth_seven():
    o = vv.Octree.terrain(seed=2, depth=7)
    info = o.info
    assert all(d <= 1022 and d % 2 == 0 for d in info.pool_dim)
    assert info.node_count % 8 == 0
    # every child pointer lands on an even (block-aligned) grid position inside the pool
    w0 = o.node_words()[..., 0]
    c = np.stack([(w0 >> 20) & 1023, (w0 >> 10) & 1023, w0 & 1023], -1)
    has = np.any(c != 0, -1)
    assert np.all(c[has] % 2 == 0)
    assert np.all(c[has] < np.array(info.pool_dim))
