"""The .gvx / .gvb / .gvp reader and writer against the oracle's restatement
of GigaVoxelsReader, on files in the offline voxelizer's layout: node words,
brick texels, borders and gradients bit-exact, the reference's constant-colour
behaviour, the error cases the reference rejects, and write/read round trips."""
import os
import shutil
import struct

import numpy as np
import pytest

import voxviz_b200 as vv
from voxviz_b200 import _native as N
from oracle import gvfile_ref as gr
from tests import gvx_fixtures as gf


@pytest.fixture(scope="module")
def files(tmp_path_factory):
    out = {}
    for depth in (2, 4, 5):
        d = tmp_path_factory.mktemp(f"vox{depth}")
        gf.write_voxelizer_style(str(d), seed=3, depth=depth)
        out[depth] = str(d)
    return out


def _bricks(o, ref):
    xyz = np.array(sorted(ref["bricks"].keys()), dtype=np.uint32).reshape(-1, 3)
    got = o.produce_bricks(xyz, "rgba8").view(np.uint32)
    exp = np.stack([ref["bricks"][tuple(p)]["block"] for p in xyz.tolist()])
    return xyz, got, exp


@pytest.mark.parametrize("depth", [4, 5])
@pytest.mark.parametrize("constant_colors", [False, True])
def test_reader_matches_oracle(files, depth, constant_colors):
    path = os.path.join(files[depth], "tree.gvx")
    ref = gr.load_gvx(path, constant_colors=constant_colors)
    o = vv.Octree.load_gvx(path, constant_colors=constant_colors)
    assert np.array_equal(o.node_words(), ref["words"])
    xyz, got, exp = _bricks(o, ref)
    assert np.array_equal(got, exp)
    nrm = o.produce_gradients(xyz, "rgba8").view(np.uint32)
    assert np.array_equal(nrm, np.stack([ref["bricks"][tuple(p)]["normals"] for p in xyz.tolist()]))
    # FP32 gradients hold the same unsigned bytes as b / 255
    f32 = o.produce_gradients(xyz[:5], "fp32").view(np.float32).reshape(5, 1000, 4)
    b = nrm[:5]
    for c in range(3):
        assert np.array_equal(f32[..., c], ((b >> (8 * c)) & 255).astype(np.float32) / np.float32(255.0))
    i = o.gvx_info
    h = ref["header"]
    assert i.file_backed == 1 and i.max_depth == h["max_depth"] == depth + 1
    assert list(i.volume_size) == h["volume_size"] and list(i.brick_size) == [8, 8, 8]
    assert np.allclose(list(i.origin), [-12.5, 3.25, 100.0]) and np.allclose(list(i.delta), [0.1] * 3)
    assert i.bricks == len(ref["bricks"]) == o.info.nonconst_count
    assert i.has_gradients == 1
    assert o.info.volume_dim == 8 << depth and i.ray_step_size == np.float32(1.0 / (8 << depth))
    # the voxelizer's edge bricks: border 0 at the low face, 8-wide bricks spanning a level
    borders = {b["border"] for b in ref["bricks"].values()}
    assert (0, 0, 0) in borders and (1, 1, 1) in borders
    assert {b["dims"] for b in ref["bricks"].values()} == {(8, 8, 8), (10, 10, 10)}


def test_constant_colours_follow_the_reference(files):
    """Node::setConstantValue drops the colour: constant nodes load as
    transparent black unless asked; the stored colour is the reader's
    truncation of the writer's %g text."""
    path = os.path.join(files[5], "tree.gvx")
    plain = vv.Octree.load_gvx(path).node_words()
    kept = vv.Octree.load_gvx(path, constant_colors=True).node_words()
    const = (plain[..., 0] & 0x40000000) != 0
    assert const.sum() > 0 and np.all(plain[..., 1][const] == 0)
    assert np.array_equal(plain[..., 0], kept[..., 0])
    t = vv.Octree.terrain(seed=3, depth=5).node_words()
    tv = t[..., 1][const]
    assert (tv != 0).sum() > 0
    exp = np.zeros_like(tv)
    for c in range(4):
        ch = (tv >> np.uint32(8 * c)) & np.uint32(255)
        back = np.array([gr.colour_byte("%g" % (int(v) / 255.0)) for v in ch], dtype=np.uint32)
        exp |= back << np.uint32(8 * c)
    assert np.array_equal(kept[..., 1][const], exp)
    assert (exp != tv).sum() > 0  # some colours lose one unit through the text, as in the reference


@pytest.mark.parametrize("depth,collapse", [(5, True), (4, False)])
def test_terrain_round_trip(tmp_path, depth, collapse):
    t = vv.Octree.terrain(seed=3, depth=depth, collapse=collapse)
    t.save_gvx(tmp_path)
    o = vv.Octree.load_gvx(tmp_path / "tree.gvx", constant_colors=True)
    assert np.array_equal(o.node_words(), t.node_words())
    ref = gr.load_gvx(str(tmp_path / "tree.gvx"), constant_colors=True)
    assert np.array_equal(ref["words"], t.node_words())
    xyz, got, exp = _bricks(o, ref)
    assert np.array_equal(got, exp)
    assert np.array_equal(got, t.produce_bricks(xyz, "rgba8").view(np.uint32))
    assert {b["border"] for b in ref["bricks"].values()} == {(1, 1, 1)}
    if depth <= 6:
        assert np.array_equal(o.produce_gradients(xyz, "rgba8"), t.produce_gradients(xyz, "rgba8"))
    if not collapse:
        types = {r["type"] for r in ref["nodes"] if r is not None}
        assert "CONST" in types


def test_file_round_trip_is_byte_exact(files, tmp_path):
    src = files[4]
    o = vv.Octree.load_gvx(os.path.join(src, "tree.gvx"), constant_colors=True)
    o.save_gvx(tmp_path)
    for name in sorted(os.listdir(src)):
        if name.endswith(".gvb"):
            assert open(os.path.join(src, name), "rb").read() == open(tmp_path / name, "rb").read(), name
    again = vv.Octree.load_gvx(tmp_path / "tree.gvx", constant_colors=True)
    assert np.array_equal(again.node_words(), o.node_words())


def test_skip_gradients(files):
    path = os.path.join(files[4], "tree.gvx")
    o = vv.Octree.load_gvx(path, gradients=False)
    ref = gr.load_gvx(path, load_normals=False)
    assert o.gvx_info.has_gradients == 0
    xyz, got, exp = _bricks(o, ref)
    assert np.array_equal(got, exp)
    with pytest.raises(vv.VVError):
        o.produce_gradients(xyz[:1], "rgba8")
    with pytest.raises(vv.VVError):
        o.heights()


# ---- error cases: each is rejected by both readers with the same kind --------

def _edit_text(d, old, new, count=1):
    p = os.path.join(d, "tree.gvx")
    s = open(p).read()
    assert old in s, old
    open(p, "w").write(s.replace(old, new, count))


def _edit_gvb(d, level, fn):
    p = os.path.join(d, f"voxels_{level}.gvb")
    b = bytearray(open(p, "rb").read())
    b = fn(b)
    if b is None:
        os.remove(p)
    else:
        open(p, "wb").write(bytes(b))


def _case_missing(d):
    _edit_gvb(d, 1, lambda b: None)


def _case_trailing(d):
    _edit_gvb(d, 1, lambda b: b + b"\0")


def _case_truncated(d):
    _edit_gvb(d, 2, lambda b: b[:-10])


def _case_grad_compression(d):
    def f(b):
        csize = struct.unpack_from("<I", b, 44)[0]
        struct.pack_into("<i", b, 48 + csize, 1)
        return b
    _edit_gvb(d, 1, f)


def _case_zero_size(d):
    def f(b):
        struct.pack_into("<I", b, 44, 0)
        return b
    _edit_gvb(d, 1, f)


def _case_dims(d):
    def f(b):
        struct.pack_into("<Q", b, 4, 11)
        return b
    _edit_gvb(d, 1, f)


def _case_border(d):
    def f(b):
        struct.pack_into("<I", b, 28, 3)
        return b
    _edit_gvb(d, 1, f)


CASES = {
    "missing .gvb": (_case_missing, N.VV_ERR_IO),
    "data after the last brick": (_case_trailing, N.VV_ERR_IO),
    "truncated .gvb": (_case_truncated, N.VV_ERR_IO),
    "gradient compression mismatch": (_case_grad_compression, N.VV_ERR_IO),
    "zero colour size": (_case_zero_size, N.VV_ERR_IO),
    "dims beyond the slot": (_case_dims, N.VV_ERR_ARG),
    "border beyond the slot": (_case_border, N.VV_ERR_ARG),
    "Depth mismatch": (lambda d: _edit_text(d, 'Depth="1"', 'Depth="2"'), N.VV_ERR_IO),
    "brick size 16": (lambda d: _edit_text(d, 'BrickXSize="8"', 'BrickXSize="16"'), N.VV_ERR_ARG),
    "compressed header": (lambda d: _edit_text(d, 'Compressed="NO"', 'Compressed="YES"'), N.VV_ERR_ARG),
    "text bricks": (lambda d: _edit_text(d, 'Binary="YES"', 'Binary="NO"'), N.VV_ERR_IO),
    "MaxDepth 0": (lambda d: _edit_text(d, 'MaxDepth="3"', 'MaxDepth="0"'), N.VV_ERR_IO),
    "MaxDepth 12": (lambda d: _edit_text(d, 'MaxDepth="3"', 'MaxDepth="12"'), N.VV_ERR_ARG),
    "not a Node": (lambda d: _edit_text(d, "\n            <Node ", "\n            <Nodes "), N.VV_ERR_IO),
    "mismatched end tag": (lambda d: _edit_text(d, "</Node>", "</Nod>"), N.VV_ERR_IO),
    "unterminated attribute": (lambda d: _edit_text(d, 'Depth="2" />', 'Depth="2 />'), N.VV_ERR_IO),
    "Brick index twice": (lambda d: _edit_text(d, 'Brick="1"', 'Brick="0"'), N.VV_ERR_IO),
    "Brick index gap": (lambda d: _edit_text(d, 'Brick="1"', 'Brick="100"'), N.VV_ERR_IO),
    "negative Brick": (lambda d: _edit_text(d, 'Brick="1"', 'Brick="-1"'), N.VV_ERR_IO),
    # rejected before the index list is sized by it (it would take 8 GB)
    "huge Brick index": (lambda d: _edit_text(d, 'Brick="1"', 'Brick="2000000000"'), N.VV_ERR_IO),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_rejected_inputs(files, tmp_path, name):
    d = str(tmp_path / "ds")
    shutil.copytree(files[2], d)
    mutate, code = CASES[name]
    mutate(d)
    path = os.path.join(d, "tree.gvx")
    with pytest.raises(gr.GvxError) as ref_err:
        gr.load_gvx(path)
    assert ref_err.value.kind == ("io" if code == N.VV_ERR_IO else "unsupported")
    with pytest.raises(vv.VVError) as err:
        vv.Octree.load_gvx(path)
    assert err.value.code == code, str(err.value)


def test_text_after_the_tree_is_not_read(files, tmp_path):
    """LoadGVX stops at the root Node's end tag: like the reference's stream
    reader, the product never reads what follows it."""
    d = str(tmp_path / "ds")
    shutil.copytree(files[2], d)
    _edit_text(d, "</GigaVoxelsOctTree>", "</GigaVoxelsOctTre>")
    o = vv.Octree.load_gvx(os.path.join(d, "tree.gvx"))
    assert np.array_equal(o.node_words(), vv.Octree.load_gvx(os.path.join(files[2], "tree.gvx")).node_words())


def test_missing_file(tmp_path):
    with pytest.raises(vv.VVError) as err:
        vv.Octree.load_gvx(tmp_path / "none.gvx")
    assert err.value.code == N.VV_ERR_IO


# ---- XML forms the stream reader accepts -------------------------------------

def test_xml_forms(tmp_path):
    """Declaration, comments, single quotes, character references and a
    LEAF-CONST node written with children (skipped) parse as the oracle's
    XML parser reads them; a CONST node at an inner depth gets children."""
    leaf = ("<Node MipMapX='{x}' MipMapY='0' MipMapZ='0' Type='LEAF-CONST' ColorR='0.5' ColorG='&#48;.25' "
            "ColorB='1' ColorA='0.75' Depth='2'/>")
    kids = "".join(leaf.format(x=8 * i) for i in range(8))
    text = f"""<?xml version="1.0"?>
<!-- a hand-made tree -->
<GigaVoxelsOctTree MaxDepth='3' X='0' Y='0' Z='0' DeltaX='0.03125' DeltaY='0.03125' DeltaZ='0.03125'
   VolumeXSize='32' VolumeYSize='32' VolumeZSize='32' BrickXSize='8' BrickYSize='8' BrickZSize='8'
   Binary='YES' Compressed='NO'>
  <Node MipMapX='0' MipMapY='0' MipMapZ='0' Type='CONST' ColorR='0' ColorG='0' ColorB='0' ColorA='0' Depth='0'>
    <Node MipMapX='0' MipMapY='0' MipMapZ='0' Type='LEAF-CONST' ColorR='1' ColorG='0' ColorB='0' ColorA='1' Depth='1'>
      {kids}
    </Node>
    <!-- inner comment -->
    <Node MipMapX='8' MipMapY='0' MipMapZ='0' Type='CONST' ColorR='0.2' ColorG='0.4' ColorB='0.6' ColorA='0.8' Depth='1'>
      {kids}
    </Node>
    {"".join(f"<Node MipMapX='0' MipMapY='8' MipMapZ='{8 * i}' Type='LEAF-CONST' ColorR='0' ColorG='0' ColorB='0' ColorA='0' Depth='1'/>" for i in range(6))}
  </Node>
</GigaVoxelsOctTree>
"""
    p = tmp_path / "tree.gvx"
    p.write_text(text)
    for cc in (False, True):
        ref = gr.load_gvx(str(p), constant_colors=cc)
        o = vv.Octree.load_gvx(p, constant_colors=cc)
        assert np.array_equal(o.node_words(), ref["words"])
    assert o.info.node_count == 24  # root block, its children, the CONST child's children
    assert o.info.nonconst_count == 0


def test_volume_size_sets_ray_step(tmp_path):
    text = ("<GigaVoxelsOctTree MaxDepth='1' VolumeXSize='100' VolumeYSize='120' VolumeZSize='90' "
            "BrickXSize='8' BrickYSize='8' BrickZSize='8' Binary='YES'>"
            "<Node Type='LEAF-CONST' ColorA='0' Depth='0'/></GigaVoxelsOctTree>")
    p = tmp_path / "tree.gvx"
    p.write_text(text)
    o = vv.Octree.load_gvx(p)
    assert o.info.volume_dim == 120
    assert o.gvx_info.ray_step_size == np.float32(1.0) / np.float32(120.0)
    look, up = vv.look_at((0.5, -1.5, 0.5), (0.5, 0.5, 0.5))
    cam = vv.make_camera((0.5, -1.5, 0.5), look, up, 64, 48)
    u = vv.compute_uniforms(o.info, cam, (4, 4, 4))
    assert u.ray_step_size == np.float32(np.float32(1.0 / 120.0) * np.float32(0.5))


# ---- .gvp ------------------------------------------------------------------

def test_gvp_round_trip(tmp_path):
    tiles = [{"center": (10.0, 20.0, 5.0), "radius": 7.5, "size_meters": (3.2, 3.2, 3.2), "tree_file": "grid_0_0_0/tree.gvx"},
             {"center": (25.0, 20.0, 5.0), "radius": 7.5, "size_meters": (3.2, 3.2, 3.2), "tree_file": "grid_1_0_0/tree.gvx"},
             {"center": (11.0, 21.0, 5.5), "radius": 1.0, "size_meters": (3.2, 3.2, 3.2), "tree_file": "a&b/tree.gvx"},
             {"center": (-40.0, 2.0, 9.0), "radius": 60.0, "size_meters": (3.2, 3.2, 3.2), "tree_file": "big/tree.gvx"}]
    p = tmp_path / "root.gvp"
    vv.write_gvp(p, tiles)
    got = vv.read_gvp(p)
    ref = gr.load_gvp(str(p))
    assert got["compressed"] is False and got["brick_size"] == (8, 8, 8) == ref["brick_size"]
    assert len(got["tiles"]) == 4
    for g, r, t in zip(got["tiles"], ref["tiles"], tiles):
        assert g["center"] == tuple(np.float32(c) for c in t["center"]) == r["center"]
        assert g["radius"] == r["radius"] and g["size_meters"] == r["size_meters"]
        assert g["tree_file"] == r["tree_file"] == str(tmp_path) + "/" + t["tree_file"]
    assert got["sphere_radius"] == pytest.approx(ref["sphere_radius"], rel=1e-12)
    assert np.allclose(got["sphere_center"], ref["sphere_center"], rtol=0, atol=1e-5)
    # the last tile contains the others' sphere: the result is that tile
    assert got["sphere_radius"] == pytest.approx(60.0) or got["sphere_radius"] > 60.0


def test_gvp_without_root(tmp_path):
    p = tmp_path / "x.gvp"
    p.write_text("<Other/>")
    with pytest.raises(vv.VVError) as err:
        vv.read_gvp(p)
    assert err.value.code == N.VV_ERR_IO
    with pytest.raises(gr.GvxError):
        gr.load_gvp(str(p))
