"""Empty-cell masks of the brick pool.  The masks the library keeps (pool
creation, brick uploads, the renderer's GPU brick production, an explicit
rebuild after attaching caller memory) equal a numpy restatement of their
definition, and a draw that skips the empty cells gives the same colour,
usage lists and page requests, bit for bit, as a draw without masks."""
import numpy as np
import pytest

import voxviz_b200 as vv
from voxviz_b200 import scene
from tests import helpers

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def reference_masks(pool: np.ndarray, fmt) -> np.ndarray:
    """(slots, 32) uint32: bit (z*9+y)*9+x set when the 2x2x2 texel cell whose
    first texel is (x,y,z) is zero in every byte."""
    tb = vv.TEXEL_BYTES[vv.fmt_code(fmt)]
    t = np.asarray(pool, dtype=np.uint8).reshape(-1, 10, 10, 10, tb)  # slot, z, y, x, bytes
    zero = ~t.any(axis=-1)
    cell = np.ones((t.shape[0], 9, 9, 9), dtype=bool)
    for dz in (0, 1):
        for dy in (0, 1):
            for dx in (0, 1):
                cell &= zero[:, dz:dz + 9, dy:dy + 9, dx:dx + 9]
    bits = np.zeros((t.shape[0], 1024), dtype=np.uint64)
    bits[:, :729] = cell.reshape(-1, 729)
    words = (bits.reshape(-1, 32, 32) << np.arange(32, dtype=np.uint64)).sum(axis=-1)
    return words.astype(np.uint32)


def random_bricks(rng, n: int, fmt) -> np.ndarray:
    """Bricks with zero texels at densities from none to all, one brick with a
    single non-zero texel, and (FP16) one of negative zeros."""
    f = vv.fmt_code(fmt)
    tb = vv.TEXEL_BYTES[f]
    out = rng.integers(1, 256, size=(n, 1000, tb), dtype=np.uint8)
    for i in range(n):
        out[i][rng.random(1000) < [0.0, 0.5, 0.9, 0.97, 1.0][i % 5]] = 0
    out[n - 1] = 0
    out[n - 1, 555] = 7
    if f == vv.VV_FMT_FP16 and n > 2:
        out[n - 2] = 0
        out[n - 2, :, 1::2] = 0x80  # every half is -0.0: zero in value, not in bits
    return out.reshape(n, 1000 * tb)


@pytest.mark.parametrize("fmt", ["rgba8", "fp16", "fp32"])
def test_masks_follow_pool_creation_and_uploads(fmt):
    rng = np.random.default_rng(11)
    ctx = vv.Context(0)
    ctx.create_brickpool((3, 2, 2), fmt)
    assert np.array_equal(ctx.download_cell_masks(), reference_masks(ctx.download_bricks(), fmt))
    for slot_ids in (np.array([0, 2, 5, 7, 11], dtype=np.uint32), np.array([5, 1, 11, 3], dtype=np.uint32)):
        ctx.upload_bricks(slot_ids, random_bricks(rng, slot_ids.size, fmt))
        assert np.array_equal(ctx.download_cell_masks(), reference_masks(ctx.download_bricks(), fmt))
    assert ctx.device_status() == 0


def test_masks_follow_gpu_brick_production():
    o = helpers.octree(seed=3, depth=6)
    ctx = vv.Context(0)
    r = vv.Renderer(ctx, o, fmt="rgba8", pool_bytes=700 * 4000, preload_all=False, device_paging=True)
    for cam in scene.camera_path(5, o.heights(), 5, 200, 120):
        r.draw(cam)
        r.update()
    masks = ctx.download_cell_masks()
    assert np.array_equal(masks, reference_masks(ctx.download_bricks(), "rgba8"))
    assert masks[:, :23].any(), "no empty cell in the produced bricks: nothing exercised"
    assert ctx.device_status() == 0


@pytest.mark.parametrize("fmt", ["rgba8", "fp32"])
def test_draw_with_masks_equals_draw_without(fmt):
    sc = helpers.Scene(seed=3, depth=5, fmt=fmt)
    masked = helpers.GpuScene(sc)
    plain = helpers.GpuScene(sc, vv.Context(0))
    # the same texels in caller memory: masks invalid until rebuilt
    _, nbytes = masked.ctx.brickpool_ptr()
    texels = torch.as_tensor(masked.ctx.download_bricks().reshape(-1), device="cuda").clone()
    assert texels.numel() == nbytes
    plain.ctx.attach_bricks(texels.data_ptr(), sc.slots, fmt)
    with pytest.raises(vv.VVError):
        plain.ctx.download_cell_masks()
    masks = masked.ctx.download_cell_masks()
    assert masks[:, :23].any()
    for k in range(3):
        u = sc.uniforms(sc.view(20 + k, 160, 96, frame=k))
        a, b = masked.render(u), plain.render(u)
        for key in ("color", "usage", "mask", "requests"):
            assert np.array_equal(a[key], b[key]), (k, key)
        assert a["status"] == 0 and b["status"] == 0
    plain.ctx.update_cell_masks()
    assert np.array_equal(plain.ctx.download_cell_masks(), masks)
