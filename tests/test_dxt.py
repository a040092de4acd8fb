"""S3TC brick pools (VV_FMT_DXT5 colour, VV_FMT_DXT1 gradients): the host
encoder of the library against the oracle's decoder, and that decoder
against a restatement of EXT_texture_compression_s3tc's decode in numpy
with the expansion and rounding the library fixes (voxviz_b200/csrc/dxt.h).
The reference uploads DXT5 colour and DXT1 gradient bricks
(GigaVoxelsRenderer.cpp:235-258, GigaVoxelsBrickPool.cpp:153-250)."""
import numpy as np
import pytest

import voxviz_b200 as vv
from oracle import gv_oracle as go
from voxviz_b200 import scene
from tests import helpers


def _expand(c0):
    r, g, b = c0 >> 11, (c0 >> 5) & 63, c0 & 31
    return np.stack([(r << 3) | (r >> 2), (g << 2) | (g >> 4), (b << 3) | (b >> 2)], axis=-1)


def _np_decode(blocks, fmt):
    """The spec's decode in numpy: blocks (bricks, bytes) -> (bricks, 1000) RGBA8."""
    n = blocks.shape[0]
    bs = 16 if fmt == vv.VV_FMT_DXT5 else 8
    b = blocks.reshape(n, 90, bs).astype(np.int64)
    t = np.arange(1000)
    x, y, z = t % 10, (t // 10) % 10, t // 100
    blk = z * 9 + (y // 4) * 3 + x // 4
    tex = (y % 4) * 4 + x % 4
    cb = b[:, :, bs - 8:]
    c0 = cb[..., 0] | (cb[..., 1] << 8)
    c1 = cb[..., 2] | (cb[..., 3] << 8)
    codes = cb[..., 4] | (cb[..., 5] << 8) | (cb[..., 6] << 16) | (cb[..., 7] << 24)
    e0, e1 = _expand(c0), _expand(c1)
    four = np.ones_like(c0, dtype=bool) if fmt == vv.VV_FMT_DXT5 else c0 > c1
    p2 = np.where(four[..., None], (2 * e0 + e1 + 1) // 3, (e0 + e1 + 1) // 2)
    p3 = np.where(four[..., None], (e0 + 2 * e1 + 1) // 3, 0)
    pal = np.stack([e0, e1, p2, p3], axis=2)  # (n, 90, 4, 3)
    k = (codes[:, blk] >> (2 * tex)) & 3  # (n, 1000)
    rgb = np.take_along_axis(pal[:, blk], k[..., None, None].repeat(3, axis=-1), axis=2)[:, :, 0, :]
    a = np.zeros((n, 1000), dtype=np.int64)
    if fmt == vv.VV_FMT_DXT5:
        ab = b[:, :, :8]
        a0, a1 = ab[..., 0], ab[..., 1]
        bits = sum(ab[..., 2 + i] << (8 * i) for i in range(6))
        ak = (bits[:, blk] >> (3 * tex)) & 7
        A0, A1 = a0[:, blk], a1[:, blk]
        eight = A0 > A1
        interp8 = ((8 - ak) * A0 + (ak - 1) * A1 + 3) // 7
        interp6 = ((6 - ak) * A0 + (ak - 1) * A1 + 2) // 5
        a = np.where(ak == 0, A0, np.where(ak == 1, A1, np.where(eight, interp8,
                     np.where(ak == 6, 0, np.where(ak == 7, 255, interp6)))))
    return (rgb[..., 0] | (rgb[..., 1] << 8) | (rgb[..., 2] << 16) | (a << 24)).astype(np.uint32)


@pytest.mark.parametrize("fmt", [vv.VV_FMT_DXT5, vv.VV_FMT_DXT1])
def test_oracle_decode_matches_the_spec_restatement(fmt):
    rng = np.random.default_rng(fmt)
    blocks = rng.integers(0, 256, size=(40, vv.BRICK_BYTES[fmt]), dtype=np.uint8)
    assert np.array_equal(go.dxt_decode(blocks, fmt), _np_decode(blocks, fmt))


def _ch(a, c):
    return ((a >> (8 * c)) & 255).astype(np.int64)


def test_dxt5_bricks_of_the_terrain():
    o = helpers.octree(seed=1, depth=5)
    _, pool8, _, xyz = scene.resident_scene(o, "rgba8")
    blocks = o.produce_bricks(xyz, "dxt5")
    assert blocks.shape == (len(xyz), 1440)
    dec = go.dxt_decode(blocks, vv.VV_FMT_DXT5)
    orig = pool8[:len(xyz)].view(np.uint32).reshape(len(xyz), 1000)
    # transparent black stays exactly transparent black (air is not lit up)
    assert (dec[orig == 0] == 0).all()
    # alpha: 8 levels between the block's extremes, error at most range / 14
    assert np.abs(_ch(dec, 3) - _ch(orig, 3)).max() <= 255 // 14 + 1
    # colour: the nearest of 4 levels per block (range fit), 565 endpoints
    assert np.abs(_ch(dec, 0) - _ch(orig, 0)).mean() < 4


def test_dxt5_known_block():
    """A block with alpha endpoints 255/0 and colour endpoints 565 (31,63,1)
    and 0, every texel code 0: every texel decodes to (255,255,8,255) (bit
    replication of 31, 63 and 1)."""
    blk = np.zeros((1, 1440), dtype=np.uint8)
    w = blk.view(np.uint32).reshape(90, 4)
    w[:, 0] = 255
    w[:, 2] = (31 << 11) | (63 << 5) | 1
    dec = go.dxt_decode(blk, vv.VV_FMT_DXT5)
    assert (dec == np.uint32(255 | (255 << 8) | (8 << 16) | (255 << 24))).all()


def test_dxt1_gradients_of_the_terrain():
    o = helpers.octree(seed=1, depth=4)
    _, _, _, xyz = scene.resident_scene(o, "rgba8")
    g8 = o.produce_gradients(xyz, "rgba8").view(np.uint32).reshape(len(xyz), 1000)
    g1 = o.produce_gradients(xyz, "dxt1")
    assert g1.shape == (len(xyz), 720)
    dec = go.dxt_decode(g1, vv.VV_FMT_DXT1)
    assert (_ch(dec, 3) == 0).all()
    assert np.abs(_ch(dec, 0) - _ch(g8, 0)).mean() < 12


def test_oracle_ray_cast_on_a_dxt5_pool():
    """The oracle renders the DXT5 pool (decoded texels, filtered as RGBA8);
    against the RGBA8 pool the image differs by the compression only."""
    sc8 = helpers.Scene(seed=1, depth=5, fmt="rgba8")
    sc5 = helpers.Scene(seed=1, depth=5, fmt="dxt5")
    u = sc8.uniforms(sc8.view(3, 128, 128))
    c8, _, st8 = go.raycast(u, sc8.oracle_scene(), 32)
    c5, _, st5 = go.raycast(u, sc5.oracle_scene(), 32)
    assert st8 == st5 == 0
    e = np.abs(c5 - c8)
    assert e.max() < 0.5 and float(np.sqrt((e ** 2).mean())) < 0.05
