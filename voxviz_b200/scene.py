"""Scene set-up helpers: resident pools, seeded views and camera paths.

These build the inputs of the workloads on the host: the fully resident
node and brick pools of an octree (what ``BrickPool::initBricks`` would hold
once every brick is loaded, GigaVoxelsBrickPool.cpp:270-354), seeded
pinhole views above the terrain and a seeded low-altitude camera path.
"""
from __future__ import annotations

import math

import numpy as np

from . import BRICK_BYTES, Octree, fmt_code, look_at, make_camera

RESIDENT = np.uint32(0x80000000)
CONSTANT = np.uint32(0x40000000)


def slot_grid(count: int) -> tuple[int, int, int]:
    """BrickPool::init slot grid for `count` bricks (GigaVoxelsBrickPool.cpp:75-87)."""
    cr = max(1, int(math.pow(float(count), 1.0 / 3.0)))
    sx = sy = sz = cr
    while sx * sy * sz < count:
        sx += 1
    return sx, sy, sz


def resident_scene(octree: Octree, fmt="rgba8", slots=None):
    """Node words with every non-constant brick resident and the matching pool.

    Bricks are placed in node-index order into slots 0, 1, 2, ... (the order
    the renderer's preload uses).  Returns (words, pool, slots, nonconst_xyz).
    """
    f = fmt_code(fmt)
    words = octree.node_words().copy()
    dz, dy, dx, _ = words.shape
    w0 = words[..., 0]
    info = octree.info
    # node index order: block-major, 8 children x fastest inside the 2x2x2 cell
    bx, by = dx // 2, dy // 2
    n = np.arange(info.node_count, dtype=np.int64)
    k, c = n >> 3, n & 7
    gx = 2 * (k % bx) + (c & 1)
    gy = 2 * ((k // bx) % by) + ((c >> 1) & 1)
    gz = 2 * (k // (bx * by)) + (c >> 2)
    valid = np.zeros(info.node_count, dtype=bool)
    # unused nodes 1..7 of block 0 have no level; they are zero words, constant
    # bit clear, but they are never reached.  Mark real nodes by node_info.
    valid[0] = True
    valid[8:] = True
    nc = valid & ((w0[gz, gy, gx] & CONSTANT) == 0)
    nodes_nc = np.nonzero(nc)[0]
    count = len(nodes_nc)
    if slots is None:
        slots = slot_grid(count + 1)
    sx, sy, sz = slots
    assert sx * sy * sz >= count
    xyz = np.stack([gx[nodes_nc], gy[nodes_nc], gz[nodes_nc]], axis=1).astype(np.uint32)
    s = np.arange(count, dtype=np.int64)
    px = (s % sx) * 10 + 1
    py = ((s // sx) % sy) * 10 + 1
    pz = (s // (sx * sy)) * 10 + 1
    ptr = ((px << 20) | (py << 10) | pz).astype(np.uint32)
    words[xyz[:, 2], xyz[:, 1], xyz[:, 0], 0] |= RESIDENT
    words[xyz[:, 2], xyz[:, 1], xyz[:, 0], 1] = ptr
    pool = np.zeros((sx * sy * sz, BRICK_BYTES[f]), dtype=np.uint8)
    if count:
        pool[:count] = octree.produce_bricks(xyz, f)
    return words, pool, (sx, sy, sz), xyz


def terrain_height(heights: np.ndarray, x: float, y: float) -> float:
    """Normalized terrain height at normalized (x, y) (nearest column)."""
    n = heights.shape[0]
    i = min(n - 1, max(0, int(x * n)))
    j = min(n - 1, max(0, int(y * n)))
    return float(heights[j, i]) / n


def seeded_view(seed: int, heights: np.ndarray, width: int, height: int, frame: int = 0, near: float = 0.05):
    """A seeded pinhole camera above the terrain looking at it."""
    rng = np.random.default_rng(seed)
    theta = rng.uniform(0, 2 * math.pi)
    r = rng.uniform(0.45, 0.9)
    z = rng.uniform(0.85, 1.25)
    eye = np.array([0.5 + r * math.cos(theta), 0.5 + r * math.sin(theta), z])
    tx, ty = 0.5 + rng.uniform(-0.15, 0.15), 0.5 + rng.uniform(-0.15, 0.15)
    target = np.array([tx, ty, terrain_height(heights, tx, ty)])
    look, up = look_at(eye, target)
    return make_camera(eye, look, up, width, height, frame=frame, near=near)


def _catmull_rom(p0, p1, p2, p3, t):
    t2, t3 = t * t, t * t * t
    return 0.5 * ((2 * p1) + (-p0 + p2) * t + (2 * p0 - 5 * p1 + 4 * p2 - p3) * t2 + (-p0 + 3 * p1 - 3 * p2 + p3) * t3)


def camera_path(seed: int, heights: np.ndarray, frames: int, width: int, height: int, near: float = 0.005,
                waypoints: int = 6):
    """A seeded low-altitude flight: a Catmull-Rom spline through seeded
    waypoints 1.05-1.3x the local terrain height, looking forward and down."""
    rng = np.random.default_rng(seed)
    pts = []
    ang = rng.uniform(0, 2 * math.pi)
    c = np.array([0.5, 0.5])
    for i in range(waypoints + 3):
        a = ang + i * (2 * math.pi / (waypoints + 1)) + rng.uniform(-0.3, 0.3)
        r = rng.uniform(0.15, 0.32)
        xy = c + r * np.array([math.cos(a), math.sin(a)])
        pts.append(xy)
    pts = np.array(pts)
    cams = []
    segs = len(pts) - 3
    pos = []
    for f in range(frames + 1):
        u = f / frames * segs
        s = min(int(u), segs - 1)
        t = u - s
        xy = _catmull_rom(pts[s], pts[s + 1], pts[s + 2], pts[s + 3], t)
        pos.append(xy)
    alts = rng.uniform(1.05, 1.3, size=frames + 1)
    for f in range(frames):
        xy, nxt = pos[f], pos[f + 1]
        h = max(terrain_height(heights, xy[0], xy[1]), 0.02)
        # clear the terrain a little ahead too
        ha = max(h, terrain_height(heights, nxt[0], nxt[1]))
        z = min(0.98, max(h * alts[f], ha * 1.05))
        eye = np.array([xy[0], xy[1], z])
        fwd = np.array([nxt[0] - xy[0], nxt[1] - xy[1], 0.0])
        if np.linalg.norm(fwd) < 1e-9:
            fwd = np.array([1.0, 0.0, 0.0])
        fwd /= np.linalg.norm(fwd)
        target = eye + fwd + np.array([0.0, 0.0, -0.35])
        look, up = look_at(eye, target)
        cams.append(make_camera(eye, look, up, width, height, frame=f, near=near))
    return cams


def converge_views(renderer, cams, max_passes: int = 64, strict: bool = True):
    """Draw every view and service its page requests until one whole pass
    over the views uploads no brick (the paging fixed point of
    GigaVoxelsRenderer::postDraw + BrickPool::update for that view set).
    Returns the number of passes.  When the pool cannot hold the set, raises
    (strict) or returns (max_passes, bricks uploaded in the last pass)."""
    uploaded = 0
    for p in range(1, max_passes + 1):
        uploaded = 0
        for cam in cams:
            renderer.draw(cam)
            renderer.update()
            uploaded += renderer.stats()["bricks_uploaded"]
        if uploaded == 0:
            return p if strict else (p, 0)
    if strict:
        raise RuntimeError(f"paging did not converge in {max_passes} passes over {len(cams)} views")
    return max_passes, uploaded
