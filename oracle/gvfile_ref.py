"""Restatement of the GigaVoxels dataset reader.  TEST INFRASTRUCTURE.

GigaVoxelsReader (VoxViz/GigaVoxels/GigaVoxelsReader.cpp):

* ``LoadGVX`` (:373-514) reads the ``GigaVoxelsOctTree`` header, then the
  root ``Node`` element, then ``voxels_<depth>.gvb`` for every depth that has
  non-constant nodes;
* ``LoadOctTreeNode`` (:277-371) checks the ``Depth`` attribute, marks the
  node constant (``CONST`` / ``LEAF-CONST``, colour through
  ``Node::setConstantValue``, GigaVoxelsOctTree.cpp:1611-1621, which converts
  the colour but never stores it) or non-constant (``Brick`` index), and,
  unless the node is at the last depth or ``LEAF-CONST``, allocates its child
  block (``OctTreeNodePool::allocateChildNodeBlock``,
  GigaVoxelsOctTreeNodePool.cpp:49-73) and reads the next 8 start elements
  as its children - so node blocks are numbered in depth-first pre-order;
* ``LoadBinaryBricks`` (:106-221): ``int compressed``, then per brick in
  index order ``size_t dims[3]``, ``uint32 border[3]`` and twice (colours,
  gradients) ``int compressed, uint32 size, bytes``; the file must end there;
* ``LoadGVP`` (:35-101): ``OctTrees`` with ``OctTree`` tiles and the bounding
  sphere grown by ``BoundingSphere::expandBy``
  (VoxVizCore/BoundingVolumes.cpp:48-107).

Node words follow ``OctTreeNodePool::create3DTexture``
(GigaVoxelsOctTreeNodePool.cpp:90-223): block b covers the 2x2x2 grid cell
(2(b mod bx), 2(b div bx mod by), 2(b div bx div by)), word0 = child block's
grid cell (10:10:10) | 0x40000000 for constant nodes.

The XML token stream comes from Python's own parser
(``xml.etree.ElementTree.iterparse``), independent of the product's.
"""
from __future__ import annotations

import math
import os
import struct
import xml.etree.ElementTree as ET

import numpy as np

CONSTANT = 0x40000000


class GvxError(Exception):
    """An input the reference rejects (kind 'io') or the product does not
    render (kind 'unsupported')."""

    def __init__(self, msg: str, kind: str = "io"):
        super().__init__(msg)
        self.kind = kind


def to_int(s) -> int:
    """QString::toInt: 0 when absent or not a number."""
    if s is None:
        return 0
    try:
        v = int(s.strip(), 10)
    except ValueError:
        return 0
    return v if -2 ** 31 <= v < 2 ** 31 else 0


def to_float32(s) -> np.float32:
    """QString::toFloat: 0 when absent or not a number."""
    if s is None:
        return np.float32(0.0)
    try:
        return np.float32(float(s.strip()))
    except ValueError:
        return np.float32(0.0)


def colour_byte(s) -> int:
    """static_cast<unsigned char>(value * 255.0f), clamped to [0, 255]."""
    v = np.float32(to_float32(s) * np.float32(255.0))
    if not v > 0:
        return 0
    return 255 if v >= 255 else int(math.floor(float(v)))


class _Stream:
    """Start/end element tokens with the stream reader's two navigation calls."""

    def __init__(self, path):
        self.tokens = []
        try:
            for ev, el in ET.iterparse(path, events=("start", "end")):
                self.tokens.append((ev, el.tag, dict(el.attrib)))
        except ET.ParseError as e:
            raise GvxError(f"XML: {e}") from e
        self.i = 0
        self.name = None
        self.attrs = {}
        self.elements = sum(1 for t in self.tokens if t[0] == "start")

    def next(self):
        if self.i >= len(self.tokens):
            return None
        ev, tag, attrs = self.tokens[self.i]
        self.i += 1
        if ev == "start":
            self.name, self.attrs = tag, attrs
        return ev

    def read_next_start_element(self) -> bool:
        return self.next() == "start"

    def skip_current_element(self) -> None:
        depth = 1
        while depth:
            ev = self.next()
            if ev is None:
                return
            depth += 1 if ev == "start" else -1


def _load_bricks(path, nodes, load_normals):
    """LoadBinaryBricks for one depth: list of brick dicts in index order."""
    if not os.path.exists(path):
        raise GvxError(f"cannot open {path}")
    data = open(path, "rb").read()
    p = 0

    def take(fmt):
        nonlocal p
        n = struct.calcsize(fmt)
        if p + n > len(data):
            raise GvxError(f"{path}: truncated")
        v = struct.unpack_from(fmt, data, p)
        p += n
        return v

    (compressed,) = take("<i")
    out = []
    for node in nodes:
        if node is None:
            break
        dims = take("<3Q")
        border = take("<3I")
        for a in range(3):
            if not 1 <= dims[a] <= 10 or border[a] > 2:
                raise GvxError(f"{path}: dims {dims} / border {border} outside a 10^3 slot", "unsupported")
        count = dims[0] * dims[1] * dims[2]
        b = {"dims": dims, "border": border, "colors": None, "normals": None}
        for part, what, width in ((0, "colors", 4), (1, "gradients", 3)):
            c, size = take("<iI")
            if c != compressed:
                raise GvxError(f"{path}: compression mismatch ({what})")
            if size == 0:
                raise GvxError(f"{path}: size of {what} data is zero")
            if compressed:
                raise GvxError(f"{path}: DXT-compressed bricks", "unsupported")
            if part == 1 and not load_normals:
                if p + size > len(data):
                    raise GvxError(f"{path}: truncated")
                p += size
                continue
            if size != count * width:
                raise GvxError(f"{path}: {what} size {size} != {count * width}")
            if p + size > len(data):
                raise GvxError(f"{path}: tried to read {size} {what} bytes")
            raw = np.frombuffer(data, dtype=np.uint8, count=size, offset=p)
            p += size
            b["colors" if part == 0 else "normals"] = raw.copy()
        out.append(b)
    if p != len(data):
        raise GvxError(f"{path}: data after the last brick")
    return out


def load_gvx(path, constant_colors=False, load_normals=True) -> dict:
    """LoadGVX.  Returns header, node records (pool order), the node words
    (dz, dy, dx, 2) in texture order (no brick resident) and, per grid cell of
    a non-constant node, its brick: dims, border, the 10^3 RGBA8 block
    (stored texels at the block origin, zero elsewhere) and normals."""
    xs = _Stream(path)
    header = None
    nodes = []
    brick_nodes = []
    have_tree = False
    bricks = []
    while xs.read_next_start_element():
        if xs.name == "GigaVoxelsOctTree":
            if header is not None:
                raise GvxError("more than one GigaVoxelsOctTree")
            a = xs.attrs
            header = {
                "origin": [to_float32(a.get(k)) for k in ("X", "Y", "Z")],
                "delta": [to_float32(a.get(k)) for k in ("DeltaX", "DeltaY", "DeltaZ")],
                "volume_size": [to_int(a.get(k)) for k in ("VolumeXSize", "VolumeYSize", "VolumeZSize")],
                "brick_size": [to_int(a.get(k)) for k in ("BrickXSize", "BrickYSize", "BrickZSize")],
                "binary": a.get("Binary") == "YES",
                "compressed": a.get("Compressed") == "YES",
                "max_depth": to_int(a.get("MaxDepth")),
            }
            if header["max_depth"] < 1:
                raise GvxError("MaxDepth < 1")
            if header["max_depth"] > 11:
                raise GvxError("MaxDepth > 11", "unsupported")
            if header["brick_size"] != [8, 8, 8]:
                raise GvxError("brick size", "unsupported")
        elif header is not None and xs.name == "Node":
            if have_tree:
                raise GvxError("more than one root Node")
            have_tree = True
            max_level = header["max_depth"] - 1
            brick_nodes = [[] for _ in range(header["max_depth"])]
            nodes = [None] * 8

            def load_node(cur, level, parent):
                a = xs.attrs
                if to_int(a.get("Depth")) != level:
                    raise GvxError("Depth attribute mismatch")
                rec = {"level": level, "parent": parent, "mip": [to_int(a.get(k)) for k in ("MipMapX", "MipMapY",
                                                                                         "MipMapZ")],
                       "child_block": None, "brick": None, "color": 0}
                typ = a.get("Type") or ""
                if typ in ("CONST", "LEAF-CONST"):
                    rec["type"] = typ
                    ch = [colour_byte(a.get(k)) for k in ("ColorR", "ColorG", "ColorB", "ColorA")]
                    rec["color"] = ch[0] | (ch[1] << 8) | (ch[2] << 16) | (ch[3] << 24)
                else:
                    rec["type"] = "NON-CONST"
                    b = to_int(a.get("Brick"))
                    if b < 0:
                        raise GvxError("negative Brick")
                    if b >= xs.elements:
                        # more bricks than the file has elements: a gap for sure
                        raise GvxError("Brick index beyond the file's element count")
                    lst = brick_nodes[level]
                    if b >= len(lst):
                        lst.extend([None] * (b + 1 - len(lst)))
                    if lst[b] is not None:
                        raise GvxError("Brick index used twice")
                    lst[b] = cur
                    rec["brick"] = b
                nodes[cur] = rec
                if level == max_level or typ == "LEAF-CONST":
                    xs.skip_current_element()
                    return
                block = len(nodes) // 8
                rec["child_block"] = block
                nodes.extend([None] * 8)
                for i in range(8):
                    ev = xs.next()
                    while ev == "end":
                        ev = xs.next()
                    if ev != "start":
                        raise GvxError("fewer than 8 children")
                    if xs.name != "Node":
                        raise GvxError("invalid element")
                    load_node(8 * block + i, level + 1, cur)

            load_node(0, 0, None)
            xs.skip_current_element()
            bricks = [[] for _ in range(header["max_depth"])]
            d = os.path.dirname(path) or "."
            for lv, lst in enumerate(brick_nodes):
                if not lst:
                    continue
                if not header["binary"]:
                    raise GvxError("binary bricks only")
                if header["compressed"]:
                    raise GvxError("DXT-compressed bricks", "unsupported")
                bricks[lv] = _load_bricks(os.path.join(d, f"voxels_{lv}.gvb"), lst, load_normals)
                if len(bricks[lv]) != len(lst):
                    raise GvxError("Brick index gap")
    if not have_tree:
        raise GvxError("no tree")

    # create3DTexture layout
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
    node_bricks = {}
    for idx, r in enumerate(nodes):
        if r is None:
            continue
        w0 = CONSTANT if r["type"] != "NON-CONST" else 0
        w1 = r["color"] if (r["type"] != "NON-CONST" and constant_colors) else 0
        if r["child_block"] is not None:
            x, y, z = grid(8 * r["child_block"])
            w0 |= (x << 20) | (y << 10) | z
        gx, gy, gz = grid(idx)
        words[gz, gy, gx] = (w0, w1)
        if r["type"] == "NON-CONST":
            b = bricks[r["level"]][r["brick"]]
            dims = b["dims"]
            block = np.zeros((10, 10, 10), dtype=np.uint32)
            col = b["colors"].view(np.uint32).reshape(dims[2], dims[1], dims[0])
            block[:dims[2], :dims[1], :dims[0]] = col
            nrm = None
            if b["normals"] is not None:
                n3 = b["normals"].reshape(dims[2], dims[1], dims[0], 3).astype(np.uint32)
                nrm = np.zeros((10, 10, 10), dtype=np.uint32)
                nrm[:dims[2], :dims[1], :dims[0]] = n3[..., 0] | (n3[..., 1] << 8) | (n3[..., 2] << 16)
            node_bricks[(gx, gy, gz)] = {"dims": dims, "border": b["border"], "block": block.reshape(-1),
                                         "normals": None if nrm is None else nrm.reshape(-1),
                                         "level": r["level"], "index": r["brick"]}
    return {"header": header, "nodes": nodes, "words": words, "pool_dim": (dx, dy, dz), "bricks": node_bricks}


def expand_sphere(center, radius, c, r):
    """BoundingSphere::expandBy(center, radius) in double arithmetic."""
    if not r > 0:
        return center, radius
    if not radius > 0:
        return list(c), float(r)
    d = math.sqrt(sum((float(center[a]) - float(c[a])) ** 2 for a in range(3)))
    if d + r <= radius:
        return center, radius
    if d + radius <= r:
        return list(c), float(r)
    nr = (radius + d + r) * 0.5
    ratio = (nr - radius) / d
    return [float(np.float32(float(center[a]) + (float(c[a]) - float(center[a])) * ratio)) for a in range(3)], nr


def load_gvp(path) -> dict:
    """LoadGVP: tiles (tree file joined with the .gvp's directory) and sphere."""
    xs = _Stream(path)
    root = None
    tiles = []
    center, radius = [0.0, 0.0, 0.0], -1.0
    d = os.path.dirname(path) or "."
    while xs.read_next_start_element():
        if xs.name == "OctTrees":
            a = xs.attrs
            root = {"compressed": a.get("Compressed") == "YES",
                    "brick_size": tuple(to_int(a.get(k)) for k in ("BrickXSize", "BrickYSize", "BrickZSize"))}
        elif root is not None and xs.name == "OctTree":
            a = xs.attrs
            c = [float(to_float32(a.get(k))) for k in ("CenterX", "CenterY", "CenterZ")]
            r = float(to_float32(a.get("Radius")))
            tiles.append({"center": tuple(c), "radius": r,
                          "size_meters": tuple(float(to_float32(a.get(k))) for k in ("SizeXMeters", "SizeYMeters",
                                                                                      "SizeZMeters")),
                          "tree_file": d + "/" + (a.get("TreeFile") or "")})
            center, radius = expand_sphere(center, radius, c, r)
            xs.skip_current_element()
    if root is None:
        raise GvxError("no OctTrees element")
    root.update({"tiles": tiles, "sphere_center": tuple(center), "sphere_radius": radius})
    return root
