"""A paged scene of four terrain tiles on the GPU: the scene's colour is
each drawn tile's colour blended over the previous ones in render order
(GL_SRC_ALPHA, GL_ONE_MINUS_SRC_ALPHA) exactly, and a tile renders exactly
as a stand-alone renderer of its tree given the camera mapped into the
tile's box."""
import math

import numpy as np
import pytest

import voxviz_b200 as vv
from oracle import scene_ref as sr

pytestmark = pytest.mark.gpu

SIZE = 10.0
DEPTH = 3


@pytest.fixture(scope="module")
def tiles(tmp_path_factory):
    d = tmp_path_factory.mktemp("scene")
    out = []
    for k, (i, j) in enumerate([(0, 0), (1, 0), (0, 1), (1, 1)]):
        sub = d / f"grid_{i}_{j}_0"
        sub.mkdir()
        vv.Octree.terrain(seed=k + 1, depth=DEPTH).save_gvx(sub)
        p = sub / "tree.gvx"
        text = p.read_text()
        n = 8 << DEPTH
        head, rest = text.split(">", 1)
        for a, v in (("X", SIZE * i), ("Y", SIZE * j), ("Z", 0.0)):
            head = head.replace(f' {a}="0"', f' {a}="{v}"', 1)
        for a in ("DeltaX", "DeltaY", "DeltaZ"):
            head = head.replace(f'{a}="{1.0 / n:.9g}"', f'{a}="{SIZE / n}"', 1)
        p.write_text(head + ">" + rest)
        out.append({"center": (SIZE * i + SIZE / 2, SIZE * j + SIZE / 2, SIZE / 2),
                    "radius": SIZE / 2 * math.sqrt(3.0), "size_meters": (SIZE,) * 3,
                    "tree_file": f"grid_{i}_{j}_0/tree.gvx", "box": (SIZE * i, SIZE * j, 0.0)})
    vv.write_gvp(d / "root.gvp", out)
    return str(d / "root.gvp"), out


def _path(frames, W=256, H=160):
    cams = []
    for f in range(frames):
        a = 2.0 * math.pi * f / frames
        pos = (SIZE + 17.0 * math.cos(a), SIZE + 17.0 * math.sin(a), 9.0 + 3.0 * math.sin(2 * a))
        look, up = vv.look_at(pos, (SIZE, SIZE, 2.0))
        cams.append(vv.make_camera(pos, look, up, W, H, frame=f, near=0.05))
    return cams


def _tile_camera(cam, box_min):
    c = vv.make_camera(list(cam.position), list(cam.look), list(cam.up), cam.width, cam.height, frame=cam.frame,
                       fov_y_deg=cam.fov_y_deg, near=cam.near_dist)
    lo = np.array(box_min, dtype=np.float32)
    hi = lo + np.float32(SIZE)
    centre = ((lo + hi) * np.float32(0.5)).astype(np.float32)
    scale = (hi - lo).astype(np.float32)
    p = np.array(list(cam.position), dtype=np.float32)
    c.position[:] = [float(v) for v in (((p - centre) / scale).astype(np.float32) + np.float32(0.5))]
    c.near_dist = float(np.float32(cam.near_dist) / scale[0])
    return c


@pytest.mark.parametrize("device_paging", [False, True])
def test_scene_blends_tiles_in_render_order(tiles, device_paging):
    gvp, info = tiles
    ctx = vv.Context(0)
    pool = 300 * 1000 * 4
    sc = vv.Scene(ctx, gvp, pool_bytes_per_tile=pool, synchronous=True, device_paging=device_paging,
                  constant_colors=True)
    solo_ctx = vv.Context(0)
    solo = vv.Renderer(solo_ctx, vv.Octree.load_gvx(gvp.replace("root.gvp", info[0]["tree_file"]),
                                                    constant_colors=True),
                       fmt="rgba8", pool_bytes=pool, preload_all=False, alpha_stop=0.99, jitter_seed=7,
                       device_paging=device_paging)
    drawn_total, orders, solo_frames = 0, set(), 0
    for cam in _path(24):
        sc.draw(cam)
        colour = sc.read_color()
        states = sc.tile_states()
        order = sorted((s["drawn_order"], i) for i, s in enumerate(states) if s["drawn_order"] >= 0)
        exp = np.zeros_like(colour)
        for _, i in order:
            tc = sc.tile_renderer(i).read_color()
            exp = sr.blend_over(exp, tc)
        assert np.array_equal(colour, exp), f"blend differs at frame {cam.frame}"
        if any(i == 0 for _, i in order):
            solo.draw(_tile_camera(cam, info[0]["box"]))
            assert np.array_equal(solo.read_color(), sc.tile_renderer(0).read_color()), \
                f"tile 0 differs from its stand-alone renderer at frame {cam.frame}"
            solo.update()
            solo_frames += 1
        sc.update()
        drawn_total += len(order)
        orders.add(tuple(i for _, i in order))
        assert ctx.device_status() == 0
    st = sc.stats()
    assert st["loads"] == 4 and st["load_failures"] == 0
    assert drawn_total > 24 and len(orders) > 2 and solo_frames > 3
    assert np.abs(colour).sum() > 0


def test_batched_scene_matches_per_tile_launches(tiles):
    """VV_SCENE_BATCHED: the drawn tiles' ray casts as one persistent launch
    give the same scene colour and the same page requests per tile."""
    gvp, info = tiles
    out = []
    for batched in (False, True):
        ctx = vv.Context(0)
        sc = vv.Scene(ctx, gvp, pool_bytes_per_tile=300 * 1000 * 4, synchronous=True, device_paging=True,
                      constant_colors=True, batched=batched)
        frames = []
        for cam in _path(16):
            sc.draw(cam)
            colour = sc.read_color()
            sc.update()
            drawn = [i for i, s in enumerate(sc.tile_states()) if s["drawn_order"] >= 0]
            frames.append((colour, {i: sc.tile_renderer(i).last_requests() for i in drawn}))
        assert ctx.device_status() == 0
        out.append(frames)
    multi = 0
    for k, ((c0, r0), (c1, r1)) in enumerate(zip(*out)):
        assert np.array_equal(c0, c1), f"colour differs at frame {k}"
        assert r0.keys() == r1.keys()
        for i in r0:
            assert np.array_equal(r0[i], r1[i]), f"tile {i} requests differ at frame {k}"
        multi += len(r0) > 1
    assert multi > 3
