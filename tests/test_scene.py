"""Paged scenes on the host (VV_SCENE_HOST_ONLY): frustum culling, render
order, load requests, pager order, merging and stale unloading against the
restatement of the reference's cull visitor and DatabasePager, frame by
frame; and the asynchronous pager thread reaching the same states."""
import math
import os

import numpy as np
import pytest

import voxviz_b200 as vv
from oracle import scene_ref as sr

GRID = 6
SIZE = 10.0


def _tile_gvx(path, x0, y0, z0):
    os.makedirs(os.path.dirname(path), exist_ok=True)
    with open(path, "w") as f:
        f.write(f'<GigaVoxelsOctTree MaxDepth="1" X="{x0}" Y="{y0}" Z="{z0}" DeltaX="{SIZE / 8}" '
                f'DeltaY="{SIZE / 8}" DeltaZ="{SIZE / 8}" VolumeXSize="8" VolumeYSize="8" VolumeZSize="8" '
                'BrickXSize="8" BrickYSize="8" BrickZSize="8" Binary="YES" Compressed="NO" >\n'
                '    <Node MipMapX="0" MipMapY="0" MipMapZ="0" Type="LEAF-CONST" ColorR="0" ColorG="0" '
                'ColorB="0" ColorA="0" Depth="0" />\n</GigaVoxelsOctTree>\n')


@pytest.fixture(scope="module")
def grid(tmp_path_factory):
    d = tmp_path_factory.mktemp("grid")
    tiles = []
    missing = {7, 20}
    for i in range(GRID):
        for j in range(GRID):
            k = len(tiles)
            rel = f"grid_{i}_{j}_0/tree.gvx"
            if k not in missing:
                _tile_gvx(str(d / rel), SIZE * i, SIZE * j, 0.0)
            c = (SIZE * i + SIZE / 2, SIZE * j + SIZE / 2, SIZE / 2)
            tiles.append({"center": c, "radius": SIZE / 2 * math.sqrt(3.0), "size_meters": (SIZE,) * 3,
                          "tree_file": rel})
    vv.write_gvp(d / "root.gvp", tiles)
    return str(d / "root.gvp"), tiles, missing


def _path(frames, W=320, H=240):
    cams = []
    for f in range(frames):
        s = f / max(frames - 1, 1)
        pos = (5.0 + 50.0 * s, 3.0 + 20.0 * math.sin(3.0 * s), 8.0 + 6.0 * math.cos(2.0 * s))
        yaw = 0.3 + 2.5 * s
        target = (pos[0] + math.cos(yaw), pos[1] + math.sin(yaw), pos[2] - 0.35)
        look, up = vv.look_at(pos, target)
        cams.append(vv.make_camera(pos, look, up, W, H, frame=f, near=0.5))
    return cams


def _cam_dict(c):
    return {"position": list(c.position), "look": list(c.look), "up": list(c.up), "fov": c.fov_y_deg,
            "near": c.near_dist, "width": c.width, "height": c.height, "frame": c.frame}


@pytest.mark.parametrize("far,stale", [(60.0, 5), (10000.0, 100)])
def test_host_scene_matches_policy(grid, far, stale):
    gvp, tiles, missing = grid
    sc = vv.Scene(None, gvp, host_only=True, synchronous=True, stale_frames=stale, far_dist=far)
    g = vv.read_gvp(gvp)
    ref = sr.SceneRef([{"center": t["center"], "radius": t["radius"]} for t in g["tiles"]], stale_frames=stale,
                      far=far, loadable=lambda i: i not in missing)
    saw = {"drawn": 0, "unloads": 0, "failed": 0, "culled": 0}
    for cam in _path(40):
        sc.draw(cam)
        ref.draw(_cam_dict(cam))
        got, exp = sc.tile_states(), ref.states()
        for i, (a, b) in enumerate(zip(got, exp)):
            for k in ("visible", "drawn_order", "loaded", "pending", "failed", "last_access"):
                assert a[k] == b[k], f"frame {cam.frame} tile {i} {k}: {a[k]} != {b[k]}"
            if a["visible"]:
                assert a["dist_to_near_plane"] == np.float32(b["dist_to_near_plane"])
        sc.update()
        ref.update()
        got, exp = sc.tile_states(), ref.states()
        for i, (a, b) in enumerate(zip(got, exp)):
            for k in ("loaded", "pending", "failed"):
                assert a[k] == b[k], f"after update {cam.frame} tile {i} {k}"
        st = sc.stats()
        saw["drawn"] = max(saw["drawn"], st["drawn"])
        saw["failed"] = st["load_failures"]
        saw["culled"] = max(saw["culled"], sum(1 for s in got if not s["visible"]))
        assert st["loads"] == ref.loads and st["unloads"] == ref.unloads
    assert saw["drawn"] >= 3 and saw["culled"] > 0 and saw["failed"] >= 1
    if stale == 5:
        assert ref.unloads > 0


def test_pager_thread_loads_the_same(grid):
    gvp, tiles, missing = grid
    a = vv.Scene(None, gvp, host_only=True, synchronous=True, stale_frames=5, far_dist=60.0)
    b = vv.Scene(None, gvp, host_only=True, synchronous=False, stale_frames=5, far_dist=60.0)
    for cam in _path(30):
        for sc in (a, b):
            sc.draw(cam)
        b.wait_loads()
        for sc in (a, b):
            sc.update()
        sa, sb = a.tile_states(), b.tile_states()
        assert [(s["loaded"], s["drawn_order"], s["failed"]) for s in sa] == \
               [(s["loaded"], s["drawn_order"], s["failed"]) for s in sb], f"frame {cam.frame}"
    assert b.stats()["loads"] == a.stats()["loads"] > 0


def test_frustum_restatement_known_answers():
    """A camera at the origin looking down +y: spheres straight ahead are in,
    behind the camera, beyond the far plane or far to the side are out; the
    reported distance is to the near plane."""
    look, up = vv.look_at((0.0, 0.0, 0.0), (0.0, 1.0, 0.0))
    cam = vv.make_camera((0.0, 0.0, 0.0), look, up, 400, 300, near=1.0)
    fr = sr.Frustum(list(cam.position), list(cam.look), list(cam.up), cam.fov_y_deg, cam.near_dist, 400, 300,
                    far=100.0)
    assert fr.sphere((0.0, 10.0, 0.0), 1.0) == pytest.approx(9.0, abs=1e-6)
    assert fr.sphere((0.0, -10.0, 0.0), 1.0) is None
    assert fr.sphere((0.0, 150.0, 0.0), 1.0) is None
    assert fr.sphere((0.0, 100.5, 0.0), 1.0) is not None
    assert fr.sphere((50.0, 10.0, 0.0), 1.0) is None
    # half-width of the view at distance 10: 10 * tan(22.5 deg) * 4/3
    hw = 10.0 * math.tan(math.radians(22.5)) * 400 / 300
    assert fr.sphere((hw + 0.9, 10.0, 0.0), 1.0) is not None
    assert fr.sphere((hw + 1.2 / math.cos(math.atan(hw / 10.0)), 10.0, 0.0), 1.0) is None
