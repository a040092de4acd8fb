"""Dense numpy restatement of the reference octree builder.  TEST INFRASTRUCTURE.

For small volumes this builds everything the way the reference does, from
a dense RGBA8 volume, and the tests compare the product's sparse builder
against it:

* heights / leaf voxels - the synthetic terrain (seeded fBm value noise,
  float32 arithmetic in the same order as the product), solid below the
  surface, colour by 8 height bands
* ``mip_pyramid``        - GenerateMipMaps / GenerateMipMap / GetBoxFilterAverage
                           (VoxViz/GigaVoxels/GigaVoxelsOctTree.cpp:809-960,1030-1194)
* ``compute_node_type``  - Node::computeNodeType (:1490-1609)
* ``copy_mip_to_brick``  - Node::copyMipMapToBrick (:1428-1488) into a
                           zeroed brick (BrickPool::uploadBrick memsets it,
                           GigaVoxelsBrickPool.cpp:736-745)
* ``build_tree``         - BuildOctTree / BuildOctTreeChildren (:1196-1306)
                           with OctTreeNodePool::allocateChildNodeBlock and
                           create3DTexture (GigaVoxelsOctTreeNodePool.cpp:49-223)
"""
from __future__ import annotations

import math

import numpy as np

U32 = np.uint32
F32 = np.float32
BANDS = np.array([[72, 58, 46], [112, 84, 56], [150, 122, 80], [92, 136, 62], [54, 104, 48], [118, 116, 108],
                  [168, 166, 160], [242, 242, 248]], dtype=np.uint32)


def band_colour(b):
    b = np.asarray(b) & 7
    c = BANDS[b]
    return (c[..., 0] | (c[..., 1] << 8) | (c[..., 2] << 16) | (U32(255) << 24)).astype(np.uint32)


def lattice_hash(x, y, seed):
    with np.errstate(over="ignore"):
        x = np.asarray(x, dtype=np.uint32)
        y = np.asarray(y, dtype=np.uint32)
        h = (np.uint32(seed) * U32(0x9E3779B9)).astype(np.uint32)
        h = h ^ (x * U32(0x85EBCA6B))
        h = (h << U32(13)) | (h >> U32(19))
        h = h ^ (y * U32(0xC2B2AE35))
        h = h ^ (h >> U32(16))
        h = h * U32(0x7FEB352D)
        h = h ^ (h >> U32(15))
        h = h * U32(0x846CA68B)
        h = h ^ (h >> U32(16))
    return h.astype(np.uint32)


def _lattice_value(ix, iy, seed):
    return (lattice_hash(ix, iy, seed) >> U32(8)).astype(F32) * F32(1.0 / 16777216.0)


def _smooth(t):
    return (t * t) * (F32(3.0) - F32(2.0) * t)


def value_noise(x, y, seed):
    fx, fy = np.floor(x).astype(F32), np.floor(y).astype(F32)
    ix, iy = fx.astype(np.int32), fy.astype(np.int32)
    sx, sy = _smooth((x - fx).astype(F32)), _smooth((y - fy).astype(F32))
    v00 = _lattice_value(ix, iy, seed)
    v10 = _lattice_value(ix + 1, iy, seed)
    v01 = _lattice_value(ix, iy + 1, seed)
    v11 = _lattice_value(ix + 1, iy + 1, seed)
    a = v00 + (v10 - v00) * sx
    b = v01 + (v11 - v01) * sx
    return (a + (b - a) * sy).astype(F32)


def fbm(u, v, seed, octaves=4, lacunarity=2.0, gain=0.5, base_cells=4):
    s = np.zeros_like(u, dtype=F32)
    amp, norm, freq = F32(1.0), F32(0.0), F32(base_cells)
    for o in range(octaves):
        so = (seed + o * 0x632BE5AB) & 0xFFFFFFFF
        s = (s + amp * value_noise((u * freq).astype(F32), (v * freq).astype(F32), so)).astype(F32)
        norm = F32(norm + amp)
        amp = F32(amp * F32(gain))
        freq = F32(freq * F32(lacunarity))
    return (s / norm).astype(F32)


def heights(seed, depth, **kw):
    n = 8 << depth
    inv = F32(1.0 / n)
    x = np.arange(n, dtype=F32) * inv
    u, v = np.meshgrid(x, x)  # v varies along rows (y), u along columns (x)
    h = fbm(u.astype(F32), v.astype(F32), seed, **kw)
    t = (h * F32(n)).astype(F32)
    return np.clip(np.ceil(t).astype(np.int64), 0, n).astype(np.int32)


def leaf_volume(seed, depth, **kw):
    """Dense RGBA8 volume [z, y, x]."""
    n = 8 << depth
    H = heights(seed, depth, **kw)
    z = np.arange(n)[:, None, None]
    solid = z < H[None, :, :]
    col = band_colour(z >> depth)
    return np.where(solid, np.broadcast_to(col, (n, n, n)), U32(0)).astype(np.uint32)


def _channels(v):
    return [((v >> U32(8 * c)) & U32(255)).astype(np.uint32) for c in range(4)]


def generate_mip_map(cur):
    """GenerateMipMap for a level with even dims (2x2x2 box filter)."""
    d = cur.shape[0] // 2
    out = np.zeros((d, d, d), dtype=np.uint32)
    one_div = F32(1.0) / F32(8.0)  # the static oneDivSampleCount of the first call
    for c, ch in enumerate(_channels(cur)):
        s = ch.reshape(d, 2, d, 2, d, 2).sum(axis=(1, 3, 5)).astype(np.uint32)
        avg = np.floor((s.astype(F32) * one_div + F32(0.5)).astype(F32)).astype(np.uint32)
        out |= avg << U32(8 * c)
    return out


def mip_pyramid(vol, brick_dim=8):
    mips = [vol]
    while mips[-1].shape[0] > brick_dim:
        mips.append(generate_mip_map(mips[-1]))
    return mips


def _region(mip_dim, start, brick_dim=8, border=1):
    """computeNodeType's region along one axis: [start', end')."""
    s = start
    e = s + brick_dim
    if s != 0:
        s -= border
    if e <= mip_dim - border:
        e += border
    if e > mip_dim:
        e = mip_dim
    return s, e


def compute_node_type(mip, x, y, z, brick_dim=8):
    """Returns (is_constant, const_value RGBA8)."""
    d = mip.shape[0]
    sx, ex = _region(d, x, brick_dim)
    sy, ey = _region(d, y, brick_dim)
    sz, ez = _region(d, z, brick_dim)
    cv = int(mip[sz, sy, sx])
    edge = sx == 0 or sy == 0 or sz == 0 or ex == d or ey == d or ez == d
    if edge:
        cv = 0
    reg = mip[sz:ez, sy:ey, sx:ex]
    clear = (reg >> U32(24)) == 0
    if (cv >> 24) == 0:
        ok = np.all(clear | (reg == U32(cv)))
    else:
        ok = np.all(reg == U32(cv))
    return bool(ok), cv


def copy_mip_to_brick(mip, x, y, z, brick_dim=8):
    """Node::copyMipMapToBrick into a zeroed (B+2)^3 brick [z, y, x]."""
    d = mip.shape[0]
    bd = brick_dim + 2
    brick = np.zeros((bd, bd, bd), dtype=np.uint32)
    sx, ex = _region(d, x, brick_dim)
    sy, ey = _region(d, y, brick_dim)
    sz, ez = _region(d, z, brick_dim)
    ox = 1 if sx == 0 else 0
    oy = 1 if sy == 0 else 0
    oz = 1 if sz == 0 else 0
    brick[oz:oz + (ez - sz), oy:oy + (ey - sy), ox:ox + (ex - sx)] = mip[sz:ez, sy:ey, sx:ex]
    return brick


def build_tree(mips, collapse=True, brick_dim=8):
    """BuildOctTree with child blocks allocated depth first.

    Returns dict with node_count, pool_dim, words (dz,dy,dx,2) in texture
    order (no brick resident) and per-node (level, x, y, z) of real nodes.
    """
    L = len(mips) - 1
    nodes = []  # per node index: (level, i, j, k, is_const, cv, child_block)

    def alloc_block():
        b = len(nodes) // 8
        for _ in range(8):
            nodes.append(None)
        return b

    def classify(level, i, j, k):
        m = mips[L - level]
        return compute_node_type(m, i * brick_dim, j * brick_dim, k * brick_dim, brick_dim)

    def children(level, i, j, k, block):
        for c in range(8):
            ci, cj, ck = 2 * i + (c & 1), 2 * j + ((c >> 1) & 1), 2 * k + (c >> 2)
            isc, cv = classify(level + 1, ci, cj, ck)
            idx = 8 * block + c
            nodes[idx] = [level + 1, ci, cj, ck, isc, cv, None]
            if level + 1 < L and not (collapse and isc):
                cb = alloc_block()
                nodes[idx][6] = cb
                children(level + 1, ci, cj, ck, cb)

    root_block = alloc_block()
    isc, cv = classify(0, 0, 0, 0)
    nodes[0] = [0, 0, 0, 0, isc, cv, None]
    if L > 0 and not (collapse and isc):
        cb = alloc_block()
        nodes[0][6] = cb
        children(0, 0, 0, 0, cb)
    assert root_block == 0
    num = len(nodes)
    cr = int(math.pow(float(num), 1.0 / 3.0))
    if cr % 2 != 0:
        cr -= 1
        if cr == 0:
            cr = 2
    dx = dy = dz = cr
    while dx * dy * dz < num:
        dx += 2
    bx, by = dx // 2, dy // 2

    def grid(idx):
        k, c = idx >> 3, idx & 7
        return 2 * (k % bx) + (c & 1), 2 * ((k // bx) % by) + ((c >> 1) & 1), 2 * (k // (bx * by)) + (c >> 2)

    words = np.zeros((dz, dy, dx, 2), dtype=np.uint32)
    real = {}
    for idx, nd in enumerate(nodes):
        if nd is None:
            continue
        level, i, j, k, isc, cv, cb = nd
        w0 = 0x40000000 if isc else 0
        w1 = cv if isc else 0
        if cb is not None:
            x, y, z = grid(8 * cb)
            w0 |= (x << 20) | (y << 10) | z
        gx, gy, gz = grid(idx)
        words[gz, gy, gx] = (w0, w1)
        real[(gx, gy, gz)] = (level, i, j, k)
    return {"node_count": num, "pool_dim": (dx, dy, dz), "words": words, "nodes": real}


# ---- gradients (the lighting path) -----------------------------------------

def leaf_gradients(alpha):
    """VolumeDataSet::convert (VoxViz/VoxVizCore/VolumeDataSet.cpp:144-209):
    per voxel (a(x-1) - a(x+1), a(y-1) - a(y+1), a(z-1) - a(z+1)) with a the
    binary32 alpha/255 and 0 outside, normalised in double when its length
    is positive (QVector3D::length, operator/=), stored as binary32.
    alpha: (z, y, x) float32.  Returns (z, y, x, 3) float32."""
    a = alpha.astype(F32)
    z = np.zeros_like(a)

    def shifted(axis, d):
        out = z.copy()
        src = [slice(None)] * 3
        dst = [slice(None)] * 3
        if d < 0:  # a(x-1) at x
            src[axis] = slice(0, -1)
            dst[axis] = slice(1, None)
        else:      # a(x+1) at x
            src[axis] = slice(1, None)
            dst[axis] = slice(0, -1)
        out[tuple(dst)] = a[tuple(src)]
        return out

    g = np.stack([(shifted(2, -1) - shifted(2, +1)).astype(F32),
                  (shifted(1, -1) - shifted(1, +1)).astype(F32),
                  (shifted(0, -1) - shifted(0, +1)).astype(F32)], axis=-1).astype(np.float64)
    length = np.sqrt(g[..., 0] * g[..., 0] + g[..., 1] * g[..., 1] + g[..., 2] * g[..., 2])
    safe = np.where(length > 0, length, 1.0)
    g = np.where((length > 0)[..., None], g / safe[..., None], 0.0)
    return g.astype(F32)


def qt_normalize(v):
    """QVector3D::normalize (Qt 4.8) on binary32 vectors, in double: left as is
    when |len^2 - 1| <= 1e-12 or len^2 <= 1e-12."""
    d = v.astype(np.float64)
    len2 = (d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1]) + d[..., 2] * d[..., 2]
    keep = (np.abs(len2 - 1.0) <= 1e-12) | (np.abs(len2) <= 1e-12)
    length = np.sqrt(np.where(keep, 1.0, len2))
    out = np.where(keep[..., None], d, d / length[..., None])
    return out.astype(F32)


def gradient_pyramid(leaf):
    """GenerateMipMap / GetBoxFilterAverage for gradients
    (GigaVoxelsOctTree.cpp:809-960): each coarser voxel sums its 2x2x2 block
    in binary32 (z, y, x order, starting from 0), scales by 1/8 and applies
    QVector3D::normalize."""
    levels = [leaf]
    cur = leaf
    while cur.shape[0] > 1:
        a = np.zeros((cur.shape[0] // 2, cur.shape[1] // 2, cur.shape[2] // 2, 3), dtype=F32)
        for dz in (0, 1):
            for dy in (0, 1):
                for dx in (0, 1):
                    a = (a + cur[dz::2, dy::2, dx::2]).astype(F32)
        a = (a * F32(0.125)).astype(F32)
        cur = qt_normalize(a)
        levels.append(cur)
    return levels


def gradient_brick(level_grads, origin, brick_dim=8):
    """copyMipMapToBrick for gradients: texel b = mip voxel origin - 1 + b,
    zero outside (the brick is cleared first).  Returns (10, 10, 10, 3)."""
    n = level_grads.shape[0]
    out = np.zeros((brick_dim + 2,) * 3 + (3,), dtype=F32)
    ox, oy, oz = (int(v) - 1 for v in origin)
    for bz in range(brick_dim + 2):
        for by in range(brick_dim + 2):
            for bx in range(brick_dim + 2):
                x, y, zz = ox + bx, oy + by, oz + bz
                if 0 <= x < n and 0 <= y < n and 0 <= zz < n:
                    out[bz, by, bx] = level_grads[zz, y, x]
    return out
