"""Dataset files in the offline voxelizer's layout, made from the oracle's
terrain, for the reader tests.  TEST INFRASTRUCTURE.

The layout restates the voxelizer's writer: ``writeOctTree`` /
``WriteOctTreeNode`` (VoxViz/Voxelizer/Voxelizer/Voxelizer.cu:2840-3058: one
``Node`` element per node, depth first, ``CONST`` for a constant node with
children and ``LEAF-CONST`` without, colours as ``value / 255.0`` printed by
an ``ostream`` with its default precision, i.e. ``%g``) and
``WriteBinaryBrick`` (VoxelBrickWriter.cu:726-818: a brick keeps a 1-voxel
border where its neighbour exists; at the volume's low face it starts at 0
with border 0 and two extra voxels on the far side; at the high face it
starts two voxels early yet records border 1; a brick that spans its whole
level is 8 wide with border 0).  Brick indices per level follow the bricks'
z-major position, not the depth-first order, so the index indirection is
exercised.
"""
from __future__ import annotations

import os
import struct

import numpy as np

from oracle import terrain_ref as tr


def _axis(off: int, size: int) -> tuple[int, int, int]:
    """WriteBinaryBrick along one axis: (start, end, border)."""
    end = off + 8
    if off != 0 and end < size:       # middle brick
        return off - 1, end + 1, 1
    if off == 0 and end < size:       # low-face brick
        return 0, end + 2, 0
    if off != 0:                      # high-face brick
        return off - 2, end, 1
    return 0, end, 0                  # spans the level


def _normals(x0, x1, y0, y1, z0, z1, level) -> np.ndarray:
    z, y, x = np.meshgrid(np.arange(z0, z1), np.arange(y0, y1), np.arange(x0, x1), indexing="ij")
    out = np.stack([(x * 7 + y * 13 + level) % 256, (y * 5 + z * 11 + 3) % 256, (z * 3 + x * 17 + 101) % 256],
                   axis=-1)
    return out.astype(np.uint8)


def write_voxelizer_style(directory, seed=3, depth=4, collapse=True, origin=(-12.5, 3.25, 100.0),
                          delta=0.1) -> dict:
    """tree.gvx + voxels_<level>.gvb for the oracle terrain of (seed, depth)."""
    os.makedirs(directory, exist_ok=True)
    mips = tr.mip_pyramid(tr.leaf_volume(seed, depth))
    L = len(mips) - 1
    tree = tr.build_tree(mips, collapse)
    words, real = tree["words"], tree["nodes"]

    def node_at(g):
        gx, gy, gz = g
        return words[gz, gy, gx], real[g]

    def children(g):
        w0 = int(words[g[2], g[1], g[0], 0]) & 0x3FFFFFFF & ~0x40000000
        if w0 == 0:
            return []
        x, y, z = (w0 >> 20) & 0x3FF, (w0 >> 10) & 0x3FF, w0 & 0x3FF
        return [(x + (c & 1), y + ((c >> 1) & 1), z + (c >> 2)) for c in range(8)]

    # brick index per level: z-major position order
    per_level: dict[int, list] = {}
    for g, (lv, i, j, k) in real.items():
        if not int(words[g[2], g[1], g[0], 0]) & 0x40000000:
            per_level.setdefault(lv, []).append((k, j, i, g))
    index = {}
    for lv, lst in per_level.items():
        lst.sort()
        for n, (_, _, _, g) in enumerate(lst):
            index[g] = n

    lines = []
    n0 = 8 << L
    lines.append(f'<GigaVoxelsOctTree MaxDepth="{L + 1}" X="{origin[0]:g}" Y="{origin[1]:g}" Z="{origin[2]:g}" '
                 f'DeltaX="{delta:g}" DeltaY="{delta:g}" DeltaZ="{delta:g}" VolumeXSize="{n0}" VolumeYSize="{n0}" '
                 f'VolumeZSize="{n0}" BrickXSize="8" BrickYSize="8" BrickZSize="8" Binary="YES" Compressed="NO" >')

    def emit(g):
        w, (lv, i, j, k) = node_at(g)
        kids = children(g)
        pad = "    " * (lv + 1)
        s = f'{pad}<Node MipMapX="{8 * i}" MipMapY="{8 * j}" MipMapZ="{8 * k}" '
        if int(w[0]) & 0x40000000:
            cv = int(w[1])
            s += f'Type="{"CONST" if kids else "LEAF-CONST"}" '
            for c, name in enumerate(("ColorR", "ColorG", "ColorB", "ColorA")):
                s += f'{name}="{((cv >> (8 * c)) & 255) / 255.0:g}" '
        else:
            s += f'Type="NON-CONST" Brick="{index[g]}" '
        s += f'Depth="{lv}"'
        if kids:
            lines.append(s + ">")
            for c in kids:
                emit(c)
            lines.append(pad + "</Node>")
        else:
            lines.append(s + " />")

    emit((0, 0, 0))
    lines.append("</GigaVoxelsOctTree>")
    with open(os.path.join(directory, "tree.gvx"), "w") as f:
        f.write("\n".join(lines) + "\n")

    for lv, lst in per_level.items():
        m = mips[L - lv]
        S = m.shape[0]
        out = bytearray(struct.pack("<i", 0))
        for (k, j, i, g) in lst:
            x0, x1, bx = _axis(8 * i, S)
            y0, y1, by = _axis(8 * j, S)
            z0, z1, bz = _axis(8 * k, S)
            out += struct.pack("<3Q", x1 - x0, y1 - y0, z1 - z0)
            out += struct.pack("<3I", bx, by, bz)
            col = np.ascontiguousarray(m[z0:z1, y0:y1, x0:x1]).astype("<u4").tobytes()
            nrm = _normals(x0, x1, y0, y1, z0, z1, lv).tobytes()
            out += struct.pack("<iI", 0, len(col)) + col
            out += struct.pack("<iI", 0, len(nrm)) + nrm
        with open(os.path.join(directory, f"voxels_{lv}.gvb"), "wb") as f:
            f.write(bytes(out))
    return {"depth": L, "levels": sorted(per_level), "tree": tree}
