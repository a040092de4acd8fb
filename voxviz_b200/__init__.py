"""voxviz_b200 - B200-native GigaVoxels sparse-octree ray caster.

Python binding over the C ABI of ``include/voxviz_b200.h``.  Every call goes
through ``libvoxviz_b200.so``; there is no Python or CPU fallback for the hot
path (a missing library raises).

The objects mirror the reference's host API:

* :class:`Octree` - ``gv::GigaVoxelsOctTree`` built from a synthetic terrain
  (VoxViz/GigaVoxels/GigaVoxelsOctTree.h:34-516) or read from ``.gvx`` /
  ``.gvb`` files (``GigaVoxelsReader``, VoxViz/GigaVoxels/GigaVoxelsReader.cpp);
  :func:`read_gvp` reads a ``.gvp`` index of paged trees
* :class:`Context` - device pools and the draw entry point
  (node pool: GigaVoxelsOctTreeNodePool.h, brick pool: GigaVoxelsBrickPool.h)
* :class:`Renderer` - the ``"gv"`` ``vox::Renderer`` frame protocol
  (VoxViz/VoxVizCore/Renderer.h:20-110, GigaVoxelsRenderer.cpp)
* :class:`Scene` - a paged scene of ``.gvx`` tiles listed by a ``.gvp``
  (the cull visitor of GigaVoxelsRenderer.cpp and GigaVoxelsDatabasePager)
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np

from . import _native as N
from ._native import (BRICK_BYTES, FMT_NAMES, TEXEL_BYTES, VV_FMT_BF16, VV_FMT_DXT1, VV_FMT_DXT5, VV_FMT_FP16, VV_FMT_FP32, VV_FMT_RGBA8,  # noqa: F401
                      VV_PASS_ALL, VV_PASS_COLOR_RGBA8, VV_PASS_COMPACT, VV_PASS_RAYCAST, VV_PASS_SELECT, Camera,
                      FrameOut,
                      NodePatch, OctreeInfo, Uniforms, VVError)

__all__ = ["Octree", "Context", "Renderer", "Batch", "Scene", "batch_variants", "make_camera", "look_at",
           "read_gvp", "write_gvp",
           "compute_uniforms", "make_jitter", "pixel_size", "lib", "VVError", "Uniforms", "Camera", "FMT_NAMES",
           "TEXEL_BYTES", "BRICK_BYTES"]


def lib() -> C.CDLL:
    return N.load()


def _check(rc: int, ctx=None, what: str = "") -> None:
    if rc != N.VV_OK:
        L = lib()
        msg = L.vv_last_error(ctx).decode() if ctx is not None else L.vv_last_error(None).decode()
        base = L.vv_status_string(rc).decode()
        raise VVError(rc, f"{what}: {base}" + (f" ({msg})" if msg else ""))


def _ptr(a: np.ndarray) -> int:
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


def fmt_code(fmt) -> int:
    return FMT_NAMES[fmt] if isinstance(fmt, str) else int(fmt)


# ---------------------------------------------------------------- camera ---

def look_at(eye: Sequence[float], target: Sequence[float], world_up=(0.0, 0.0, 1.0)):
    """Unit look and up vectors for a camera at eye looking at target (Z up,
    as vox::Camera's m_worldUp, Camera.cpp:22)."""
    e = np.asarray(eye, dtype=np.float64)
    look = np.asarray(target, dtype=np.float64) - e
    look /= np.linalg.norm(look)
    wu = np.asarray(world_up, dtype=np.float64)
    left = np.cross(wu, look)
    if np.linalg.norm(left) < 1e-9:
        left = np.cross(np.array([0.0, 1.0, 0.0]), look)
    left /= np.linalg.norm(left)
    up = np.cross(look, left)
    up /= np.linalg.norm(up)
    return look, up


def make_camera(position, look, up, width: int, height: int, frame: int = 0, fov_y_deg: float = 45.0,
                near: float = 1e-3) -> Camera:
    c = Camera()
    c.position[:] = [float(v) for v in position]
    c.look[:] = [float(v) for v in look]
    c.up[:] = [float(v) for v in up]
    c.fov_y_deg = fov_y_deg
    c.near_dist = near
    c.width = width
    c.height = height
    c.frame = frame
    return c


def pixel_size(cam: Camera) -> float:
    return float(lib().vv_camera_pixel_size(C.byref(cam)))


def make_jitter(seed: int, size: int = 32) -> np.ndarray:
    out = np.empty(size * size, dtype=np.uint8)
    _check(lib().vv_make_jitter(seed, size, _ptr(out)), what="make_jitter")
    return out


def compute_uniforms(info: OctreeInfo, cam: Camera, slots: Sequence[int], lod_scalar: float = 1.0,
                     alpha_stop: float = 0.99) -> Uniforms:
    u = Uniforms()
    _check(lib().vv_compute_uniforms(C.byref(info), C.byref(cam), int(slots[0]), int(slots[1]), int(slots[2]),
                                     lod_scalar, alpha_stop, C.byref(u)), what="compute_uniforms")
    return u


# ---------------------------------------------------------------- octree ---

class Octree:
    """A terrain octree (host data model, ``gv::GigaVoxelsOctTree``)."""

    def __init__(self, handle: int):
        self._h = C.c_void_p(handle)

    @classmethod
    def terrain(cls, seed: int = 1, depth: int = 5, collapse: bool = True, octaves: int = 4,
                lacunarity: float = 2.0, gain: float = 0.5, base_cells: int = 4, threads: int = 0,
                device: int | None = None) -> "Octree":
        """The seeded fBm terrain octree, built on the host cores or, with
        ``device``, on that CUDA device (the same tree)."""
        d = N.TerrainDesc(seed=seed, depth=depth, octaves=octaves, lacunarity=lacunarity, gain=gain,
                          base_cells=base_cells, collapse_constant=1 if collapse else 0, threads=threads)
        h = C.c_void_p()
        if device is None:
            _check(lib().vv_octree_build_terrain(C.byref(d), C.byref(h)), what="octree build")
        else:
            _check(lib().vv_octree_build_terrain_gpu(C.byref(d), int(device), C.byref(h)), what="octree build (GPU)")
        return cls(h.value)

    @classmethod
    def load_gvx(cls, path, constant_colors: bool = False, gradients: bool = True) -> "Octree":
        """``GigaVoxelsReader::LoadOctTreeFile``: a tree.gvx and its voxels_<level>.gvb.

        constant_colors=False renders constant nodes as the reference does
        (transparent: ``Node::setConstantValue`` drops the colour); True keeps
        their colours.  gradients=False skips the gradient payloads.
        """
        flags = (N.VV_GVX_CONSTANT_COLORS if constant_colors else 0) | (0 if gradients else N.VV_GVX_SKIP_GRADIENTS)
        h = C.c_void_p()
        _check(lib().vv_octree_load_gvx(str(path).encode(), flags, C.byref(h)), what="load gvx")
        return cls(h.value)

    def save_gvx(self, directory, gradients: bool = True) -> None:
        """Write tree.gvx and voxels_<level>.gvb into an existing directory."""
        _check(lib().vv_octree_save_gvx(self._h, str(directory).encode(), 0 if gradients else N.VV_GVX_SKIP_GRADIENTS),
               what="save gvx")

    @property
    def gvx_info(self) -> N.GvxInfo:
        i = N.GvxInfo()
        _check(lib().vv_octree_gvx_info(self._h, C.byref(i)), what="gvx info")
        return i

    def close(self) -> None:
        if self._h:
            lib().vv_octree_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    @property
    def info(self) -> OctreeInfo:
        i = OctreeInfo()
        _check(lib().vv_octree_get_info(self._h, C.byref(i)), what="octree info")
        return i

    def node_words(self) -> np.ndarray:
        """Node pool in reference texture order: shape (dz, dy, dx, 2) uint32."""
        i = self.info
        dx, dy, dz = i.pool_dim
        out = np.zeros((dz, dy, dx, 2), dtype=np.uint32)
        _check(lib().vv_octree_node_words(self._h, _ptr(out)), what="node words")
        return out

    def node_info(self, x: int, y: int, z: int) -> N.NodeInfo:
        ni = N.NodeInfo()
        _check(lib().vv_octree_node_info(self._h, x, y, z, C.byref(ni)), what="node info")
        return ni

    def produce_bricks(self, xyz: np.ndarray, fmt="rgba8") -> np.ndarray:
        f = fmt_code(fmt)
        xyz = np.ascontiguousarray(xyz, dtype=np.uint32).reshape(-1, 3)
        n = xyz.shape[0]
        out = np.zeros((n, BRICK_BYTES[f]), dtype=np.uint8)
        _check(lib().vv_octree_produce_bricks(self._h, _ptr(xyz), n, f, _ptr(out)), what="produce bricks")
        return out

    def produce_gradients(self, xyz: np.ndarray, fmt="fp32") -> np.ndarray:
        """Gradient bricks of the nodes at grid positions xyz (trees of depth <= 6)."""
        f = fmt_code(fmt)
        xyz = np.ascontiguousarray(xyz, dtype=np.uint32).reshape(-1, 3)
        n = xyz.shape[0]
        out = np.zeros((n, BRICK_BYTES[f]), dtype=np.uint8)
        _check(lib().vv_octree_produce_gradients(self._h, _ptr(xyz), n, f, _ptr(out)), what="produce gradients")
        return out

    def mip_level(self, level: int) -> np.ndarray:
        d = (8 << self.info.depth) >> level
        out = np.zeros((d, d, d), dtype=np.uint32)
        _check(lib().vv_octree_mip_level(self._h, level, _ptr(out), out.size), what="mip level")
        return out

    def heights(self) -> np.ndarray:
        d = 8 << self.info.depth
        out = np.zeros((d, d), dtype=np.int32)
        _check(lib().vv_octree_heights(self._h, _ptr(out)), what="heights")
        return out


def read_gvp(path) -> dict:
    """``LoadGVP``: the paged-tree index (tiles with their bounding spheres)."""
    info = N.GvpInfo()
    _check(lib().vv_gvp_read(str(path).encode(), C.byref(info), None, 0), what="read gvp")
    tiles = (N.GvpTile * max(info.tiles, 1))()
    _check(lib().vv_gvp_read(str(path).encode(), C.byref(info), tiles, info.tiles), what="read gvp")
    return {
        "compressed": bool(info.compressed),
        "brick_size": tuple(info.brick_size),
        "sphere_center": tuple(info.sphere_center),
        "sphere_radius": info.sphere_radius,
        "tiles": [{"center": tuple(t.center), "radius": t.radius, "size_meters": tuple(t.size_meters),
                   "tree_file": t.tree_file.decode()} for t in tiles[:info.tiles]],
    }


def write_gvp(path, tiles: Sequence[dict], compressed: bool = False, brick_size=(8, 8, 8)) -> None:
    """Write a .gvp index; each tile dict has center, radius, size_meters and
    tree_file (relative to the .gvp's directory)."""
    info = N.GvpInfo(compressed=1 if compressed else 0)
    info.brick_size[:] = list(brick_size)
    arr = (N.GvpTile * max(len(tiles), 1))()
    for a, t in zip(arr, tiles):
        a.center[:] = list(t["center"])
        a.radius = t["radius"]
        a.size_meters[:] = list(t["size_meters"])
        a.tree_file = str(t["tree_file"]).encode()
    _check(lib().vv_gvp_write(str(path).encode(), C.byref(info), arr, len(tiles)), what="write gvp")


# --------------------------------------------------------------- context ---

class Context:
    """A device context (``vv_ctx``): node pools, the brick pool, the draw."""

    def __init__(self, device: int = 0):
        p = N.Params(device=device, flags=0)
        h = C.c_void_p()
        _check(lib().vv_ctx_create(C.byref(p), C.byref(h)), what="ctx create")
        self._h = h

    @property
    def slots(self) -> tuple[int, int, int]:
        """Brick-pool slots per axis (0,0,0 before vv_brickpool_create)."""
        s, f = (C.c_int32 * 3)(), C.c_int32()
        self._ck(lib().vv_brickpool_info(self._h, s, C.byref(f)), "brick pool info")
        return int(s[0]), int(s[1]), int(s[2])

    @property
    def fmt(self) -> int:
        s, f = (C.c_int32 * 3)(), C.c_int32()
        self._ck(lib().vv_brickpool_info(self._h, s, C.byref(f)), "brick pool info")
        return int(f.value)

    def node_dims(self, tree: int = 0) -> tuple[int, int, int]:
        d = (C.c_int32 * 3)()
        self._ck(lib().vv_nodepool_info(self._h, tree, d), "node pool info")
        return int(d[0]), int(d[1]), int(d[2])

    def close(self) -> None:
        if self._h:
            lib().vv_ctx_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def _ck(self, rc: int, what: str) -> None:
        _check(rc, self._h, what)

    def set_stream(self, stream_ptr: int) -> None:
        self._ck(lib().vv_ctx_set_stream(self._h, C.c_void_p(stream_ptr)), "set stream")

    def synchronize(self) -> None:
        self._ck(lib().vv_ctx_synchronize(self._h), "synchronize")

    def device_status(self, clear: bool = True) -> int:
        s = C.c_int32()
        self._ck(lib().vv_ctx_device_status(self._h, C.byref(s), 1 if clear else 0), "device status")
        return s.value

    def upload_nodes(self, words: np.ndarray, tree: int = 0) -> None:
        w = np.ascontiguousarray(words, dtype=np.uint32)
        dz, dy, dx = w.shape[:3]
        self._ck(lib().vv_nodepool_upload(self._h, tree, _ptr(w), dx, dy, dz), "node upload")

    def download_nodes(self, tree: int = 0) -> np.ndarray:
        dx, dy, dz = self.node_dims(tree)
        if dx == 0:
            raise VVError(N.VV_ERR_STATE, "node pool not uploaded")
        out = np.zeros((dz, dy, dx, 2), dtype=np.uint32)
        self._ck(lib().vv_nodepool_download(self._h, tree, _ptr(out)), "node download")
        return out

    def patch_nodes(self, patches: np.ndarray, tree: int = 0) -> None:
        """patches: (n, 5) uint32 rows x, y, z, word0, word1."""
        p = np.ascontiguousarray(patches, dtype=np.uint32).reshape(-1, 5)
        self._ck(lib().vv_nodepool_patch(self._h, tree, _ptr(p), p.shape[0]), "node patch")

    def create_brickpool(self, slots: Sequence[int], fmt="rgba8") -> None:
        f = fmt_code(fmt)
        self._ck(lib().vv_brickpool_create(self._h, int(slots[0]), int(slots[1]), int(slots[2]), f), "brick pool")

    def upload_bricks(self, slot_ids: np.ndarray, texels: np.ndarray) -> None:
        s = np.ascontiguousarray(slot_ids, dtype=np.uint32)
        t = np.ascontiguousarray(texels)
        if t.nbytes != s.size * BRICK_BYTES[self.fmt]:
            raise VVError(N.VV_ERR_ARG, "texels must hold one brick per slot id in the pool's format")
        self._ck(lib().vv_upload_bricks(self._h, _ptr(s), s.size, _ptr(t)), "brick upload")

    def download_bricks(self) -> np.ndarray:
        sx, sy, sz = self.slots
        n = sx * sy * sz
        if n == 0:
            raise VVError(N.VV_ERR_STATE, "brick pool not created")
        out = np.zeros((n, BRICK_BYTES[self.fmt]), dtype=np.uint8)
        self._ck(lib().vv_brickpool_download(self._h, _ptr(out)), "brick download")
        return out

    def update_cell_masks(self) -> None:
        """Rebuild the pool's empty-cell masks from its contents (after writing
        texels through an attached buffer or the device pointer)."""
        self._ck(lib().vv_brickpool_update_cell_masks(self._h), "cell masks")

    def download_cell_masks(self) -> np.ndarray:
        """(slots, 32) uint32: bit (z*9+y)*9+x set when the 2x2x2 texel cell at
        (x,y,z) is zero in every bit."""
        sx, sy, sz = self.slots
        out = np.zeros((sx * sy * sz, 32), dtype=np.uint32)
        self._ck(lib().vv_brickpool_download_cell_masks(self._h, _ptr(out)), "cell mask download")
        return out

    def create_gradpool(self, fmt="fp32") -> None:
        """Gradient pool with the brick pool's slots (lighting)."""
        self._ck(lib().vv_gradpool_create(self._h, fmt_code(fmt)), "gradient pool")

    def upload_gradients(self, slot_ids: np.ndarray, texels: np.ndarray) -> None:
        s = np.ascontiguousarray(slot_ids, dtype=np.uint32)
        t = np.ascontiguousarray(texels)
        self._ck(lib().vv_upload_gradients(self._h, _ptr(s), s.size, _ptr(t)), "gradient upload")

    def set_jitter(self, table: np.ndarray) -> None:
        t = np.ascontiguousarray(table, dtype=np.uint8)
        size = int(round(np.sqrt(t.size)))
        self._ck(lib().vv_set_jitter(self._h, _ptr(t), size), "jitter")

    def set_raycast_mode(self, mode) -> None:
        """vv_ctx_set_raycast_mode: "tiles" (default, one thread per pixel),
        "refill" (lane-refill persistent warps) or "staged" (the tiles with
        each warp's shared brick slot copied to shared memory; RGBA8 pools).
        All give the same results.  True / False mean "refill" / "tiles"."""
        modes = {"tiles": N.VV_RAYCAST_TILES, "refill": N.VV_RAYCAST_REFILL, "staged": N.VV_RAYCAST_STAGED}
        if isinstance(mode, bool):
            m = N.VV_RAYCAST_REFILL if mode else N.VV_RAYCAST_TILES
        elif isinstance(mode, str):
            if mode not in modes:
                raise ValueError(f"unknown ray-cast mode {mode!r}")
            m = modes[mode]
        else:
            m = int(mode)
        self._ck(lib().vv_ctx_set_raycast_mode(self._h, m), "raycast mode")

    def set_compaction(self, per_level: bool) -> None:
        """vv_ctx_set_compaction: the selection + histopyramid + compaction in
        three launches (default) or one launch per pyramid level (same
        results)."""
        self._ck(lib().vv_ctx_set_compaction(self._h, N.VV_COMPACT_PER_LEVEL if per_level else N.VV_COMPACT_FUSED),
                 "compaction mode")

    def set_profiling(self, on: bool = True) -> None:
        self._ck(lib().vv_ctx_set_profiling(self._h, 1 if on else 0), "profiling")

    def last_times(self) -> tuple[float, float]:
        """(ray-cast ms, selection+compaction ms) of the last profiled draw."""
        a, b = C.c_float(), C.c_float()
        self._ck(lib().vv_ctx_last_times(self._h, C.byref(a), C.byref(b)), "last times")
        return a.value, b.value

    def footprint(self, u: Uniforms, tree: int = 0) -> tuple[int, int]:
        """(distinct node-pool entries, distinct brick slots) one draw reads."""
        n, b = C.c_int64(), C.c_int64()
        self._ck(lib().vv_measure_footprint(self._h, tree, C.byref(u), C.byref(n), C.byref(b)), "footprint")
        return n.value, b.value

    def footprint_union(self, us: Sequence[Uniforms], tree: int = 0) -> tuple[int, int]:
        """The footprint of the union of several draws' reads."""
        arr = (Uniforms * len(us))(*us)
        n, b = C.c_int64(), C.c_int64()
        self._ck(lib().vv_measure_footprint_views(self._h, tree, arr, len(us), C.byref(n), C.byref(b)), "footprint")
        return n.value, b.value

    def render(self, u: Uniforms, color=0, usage=0, mask=0, requests=0, request_count=0, request_cap=0,
               compress_max_push=4, passes=VV_PASS_ALL, tree: int = 0) -> None:
        """One draw; every buffer argument is a device pointer (int) or 0."""
        o = FrameOut(color=color or None, usage=usage or None, mask=mask or None, requests=requests or None,
                     request_count=request_count or None, request_cap=request_cap,
                     compress_max_push=compress_max_push, passes=passes)
        self._ck(lib().vv_render(self._h, tree, C.byref(u), C.byref(o)), "render")

    # ---- differentiable ray cast (device pointers throughout) ----

    def attach_bricks(self, texels_ptr: int, slots: Sequence[int], fmt="fp32") -> None:
        """Use caller-owned device memory (1000 texels per slot) as the brick pool."""
        self._ck(lib().vv_brickpool_attach(self._h, C.c_void_p(texels_ptr), int(slots[0]), int(slots[1]),
                                           int(slots[2]), fmt_code(fmt)), "brick pool attach")

    def brickpool_ptr(self) -> tuple[int, int]:
        """(device pointer, bytes) of the current brick pool."""
        p, n = C.c_void_p(), C.c_size_t()
        self._ck(lib().vv_brickpool_device_ptr(self._h, C.byref(p), C.byref(n)), "brick pool pointer")
        return int(p.value or 0), int(n.value)

    @staticmethod
    def ckpt_bytes(width: int, height: int, per_ray: int) -> int:
        return int(lib().vv_ckpt_bytes(width, height, per_ray))

    def forward_ckpt(self, u: Uniforms, color: int, ckpt: int, per_ray: int, tree: int = 0) -> None:
        self._ck(lib().vv_render_forward_ckpt(self._h, tree, C.byref(u), C.c_void_p(color), C.c_void_p(ckpt),
                                              per_ray), "forward with checkpoints")

    def backward(self, u: Uniforms, dl_dcolor: int, ckpt: int, per_ray: int, grad_texels: int,
                 tree: int = 0) -> None:
        self._ck(lib().vv_backward(self._h, tree, C.byref(u), C.c_void_p(dl_dcolor), C.c_void_p(ckpt), per_ray,
                                   C.c_void_p(grad_texels)), "backward")

    def backward_ex(self, u: Uniforms, dl_dcolor: int, ckpt: int, per_ray: int, grad: int, f64: bool = False,
                    slot_map: int = 0, rows_used: int = 0, rows_cap: int = 0, tree: int = 0,
                    warp_sum: bool = False, spread: bool = False, keep: bool = False) -> None:
        """vv_backward_ex: binary64 accumulation, a sparse gradient (rows
        claimed per touched slot through `slot_map`), warp sums before the
        atomics and/or the atomics spread over copies of the rows (binary32
        rows; with `keep` the copies' sums wait for the next spread call
        without it)."""
        flags = ((N.VV_GRAD_F64 if f64 else 0) | (N.VV_GRAD_WARP_SUM if warp_sum else 0) |
                 (N.VV_GRAD_SPREAD if spread else 0) | (N.VV_GRAD_SPREAD_KEEP if keep else 0))
        g = N.GradDesc(grad=grad, flags=flags, rows_cap=rows_cap, slot_map=slot_map or None,
                       rows_used=rows_used or None)
        self._ck(lib().vv_backward_ex(self._h, tree, C.byref(u), C.c_void_p(dl_dcolor), C.c_void_p(ckpt), per_ray,
                                      C.byref(g)), "backward")


# --------------------------------------------------------------- batches ---

def batch_variants() -> list[tuple[int, int, int]]:
    """The compiled (tile_w, tile_h, steps) variants of the batched launch."""
    n = lib().vv_batch_variants(None, 0)
    arr = (N.BatchConfig * n)()
    lib().vv_batch_variants(arr, n)
    return [(c.tile_w, c.tile_h, c.steps) for c in arr]


class Batch:
    """Many views of many octrees rendered by one persistent launch.

    ``views`` holds (context, tree, uniforms, colour device pointer, usage
    device pointer) tuples; the launch runs on ``ctx``'s stream."""

    def __init__(self, ctx: Context, views: Sequence[tuple]):
        self.ctx = ctx
        self.n = len(views)
        self._arr = (N.BatchView * self.n)()
        self._keep = []
        for i, (vctx, tree, u, color, usage) in enumerate(views):
            self._arr[i].ctx = vctx.handle
            self._arr[i].tree = tree
            self._arr[i].u = u
            self._arr[i].color = color or None
            self._arr[i].usage = usage or None
            self._keep.append(vctx)
        self.config = N.BatchConfig(tile_w=16, tile_h=16, steps=1, ctas_per_sm=0)

    def set_uniforms(self, i: int, u: Uniforms) -> None:
        self._arr[i].u = u

    def render(self, config: tuple[int, int, int] | None = None, ctas_per_sm: int = 0) -> None:
        cfg = self.config if config is None else N.BatchConfig(tile_w=config[0], tile_h=config[1],
                                                               steps=config[2], ctas_per_sm=ctas_per_sm)
        _check(lib().vv_render_batch(self.ctx.handle, self._arr, self.n, C.byref(cfg)), self.ctx.handle,
               "batched render")

    def autotune(self, reps: int = 3) -> dict:
        """Time every compiled variant on this batch; keep and return the fastest."""
        variants = batch_variants()
        ms = (C.c_float * len(variants))()
        best = N.BatchConfig()
        _check(lib().vv_batch_autotune(self.ctx.handle, self._arr, self.n, reps, C.byref(best), ms),
               self.ctx.handle, "batch autotune")
        self.config = best
        return {"best": (best.tile_w, best.tile_h, best.steps),
                "ms": {f"{w}x{h}/s{s}": round(float(t), 4) for (w, h, s), t in zip(variants, ms)}}


# -------------------------------------------------------------- renderer ---

class Renderer:
    """The ``"gv"`` renderer plugin: init, draw, update (postDraw + update)."""

    def __init__(self, ctx: Context, octree: Octree, fmt="rgba8", pool_bytes: int = 0, preload_all: bool = True,
                 request_cap: int = 0, lod_scalar: float = 1.0, alpha_stop: float = 0.99, jitter_seed: int = 7,
                 producer_threads: int = 0, device_paging: bool = False, color_rgba8: bool = False):
        d = N.RendererDesc(fmt=fmt_code(fmt), pool_bytes=pool_bytes, preload_all=1 if preload_all else 0,
                           request_cap=request_cap, lod_scalar=lod_scalar, alpha_stop=alpha_stop,
                           jitter_seed=jitter_seed, max_width=0, max_height=0, producer_threads=producer_threads,
                           device_paging=1 if device_paging else 0, color_rgba8=1 if color_rgba8 else 0)
        self.color_rgba8 = bool(color_rgba8)
        h = C.c_void_p()
        _check(lib().vv_renderer_create(ctx.handle, octree.handle, C.byref(d), C.byref(h)), ctx.handle,
               "renderer create")
        self._h = h
        self.ctx = ctx
        self.octree = octree
        self.fmt = fmt_code(fmt)

    def close(self) -> None:
        if self._h:
            lib().vv_renderer_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, rc: int, what: str) -> None:
        _check(rc, self.ctx.handle, what)

    def draw(self, cam: Camera) -> None:
        self._ck(lib().vv_renderer_draw(self._h, C.byref(cam)), "draw")

    def update(self) -> None:
        self._ck(lib().vv_renderer_update(self._h), "update")

    def service(self, requests: int, count: int, cap: int) -> None:
        """Page-request service for a compacted list drawn elsewhere (device pointers)."""
        self._ck(lib().vv_renderer_service(self._h, C.c_void_p(requests), C.c_void_p(count), cap), "service")

    def set_deferred(self, on: bool = True) -> None:
        self._ck(lib().vv_renderer_set_deferred(self._h, 1 if on else 0), "set deferred")

    def stage_uploads(self) -> None:
        self._ck(lib().vv_renderer_stage_uploads(self._h), "stage uploads")

    def enqueue_uploads(self) -> None:
        self._ck(lib().vv_renderer_enqueue_uploads(self._h), "enqueue uploads")

    def stats(self) -> dict:
        s = N.RendererStats()
        self._ck(lib().vv_renderer_get_stats(self._h, C.byref(s)), "stats")
        return {k: getattr(s, k) for k, _ in N.RendererStats._fields_}

    def frame_buffers(self) -> dict:
        ptrs = [C.c_void_p() for _ in range(5)]
        self._ck(lib().vv_renderer_frame_buffers(self._h, *[C.byref(p) for p in ptrs]), "frame buffers")
        return dict(zip(["color", "usage", "mask", "requests", "request_count"], [p.value for p in ptrs]))

    def read_color(self, out: np.ndarray | None = None) -> np.ndarray:
        """Last frame's colour (H,W,4): float32, or uint8 for an RGBA8 renderer;
        into `out` (e.g. pinned) if given."""
        if out is None:
            u = self.last_uniforms()
            out = np.zeros((u.height, u.width, 4), dtype=np.uint8 if getattr(self, "color_rgba8", False)
                           else np.float32)
        self._ck(lib().vv_renderer_read_color(self._h, _ptr(out)), "read color")
        return out

    def read_color_async(self, out: np.ndarray) -> None:
        """Queue the last frame's colour read-back into `out` (pinned, (H,W,4)
        float32); it completes at wait_readback()."""
        assert out.dtype == np.float32 and out.flags["C_CONTIGUOUS"]
        self._ck(lib().vv_renderer_read_color_async(self._h, _ptr(out)), "read color async")

    def wait_readback(self) -> None:
        self._ck(lib().vv_renderer_wait_readback(self._h), "wait readback")

    def read_lists(self):
        """(usage (H,W,12), mask (H,W)) of the last frame, uint32."""
        u = self.last_uniforms()
        usage = np.zeros((u.height, u.width, 12), dtype=np.uint32)
        mask = np.zeros((u.height, u.width), dtype=np.uint32)
        self._ck(lib().vv_renderer_read_lists(self._h, _ptr(usage), _ptr(mask)), "read lists")
        return usage, mask

    def last_requests(self) -> np.ndarray:
        n = C.c_int32()
        self._ck(lib().vv_renderer_last_requests(self._h, None, 0, C.byref(n)), "requests")
        out = np.zeros((n.value, 4), dtype=np.uint32)
        self._ck(lib().vv_renderer_last_requests(self._h, _ptr(out), n.value, C.byref(n)), "requests")
        return out

    def residency(self):
        n = C.c_int64()
        self._ck(lib().vv_renderer_residency(self._h, None, None, 0, C.byref(n)), "residency")
        xyz = np.zeros((n.value, 3), dtype=np.uint32)
        slot = np.zeros(n.value, dtype=np.uint32)
        self._ck(lib().vv_renderer_residency(self._h, _ptr(xyz), _ptr(slot), n.value, C.byref(n)), "residency")
        return xyz, slot

    def lru_order(self) -> np.ndarray:
        """The brick pool's slots, least recently used first."""
        n = C.c_int64(0)
        self._ck(lib().vv_renderer_lru_order(self._h, None, 0, C.byref(n)), "lru order")
        out = np.zeros(n.value, dtype=np.uint32)
        self._ck(lib().vv_renderer_lru_order(self._h, _ptr(out), n.value, C.byref(n)), "lru order")
        return out

    def last_uniforms(self) -> Uniforms:
        u = Uniforms()
        self._ck(lib().vv_renderer_last_uniforms(self._h, C.byref(u)), "uniforms")
        return u


class _CtxRef:
    def __init__(self, handle):
        self.handle = C.c_void_p(handle)


class _TileRenderer(Renderer):
    """A loaded tile's renderer, owned by its scene."""

    def __init__(self, handle: int, scene: "Scene"):
        self._h = C.c_void_p(handle)
        self.ctx = _CtxRef(lib().vv_renderer_ctx(self._h))
        self._scene = scene

    def close(self) -> None:
        self._h = C.c_void_p()


class Scene:
    """Paged tiles of a .gvp: frustum culling, pager, back-to-front blending
    (``vv_scene_*``).  Cameras are in world coordinates."""

    def __init__(self, ctx: Context | None, gvp_path, fmt="rgba8", pool_bytes_per_tile: int = 0,
                 request_cap: int = 0, lod_scalar: float = 1.0, alpha_stop: float = 0.99, jitter_seed: int = 7,
                 device_paging: bool = False, constant_colors: bool = False, gradients: bool = True,
                 stale_frames: int = 100, far_dist: float = 10000.0, host_only: bool = False,
                 synchronous: bool = False, batched: bool = False):
        d = N.SceneDesc(fmt=fmt_code(fmt), pool_bytes_per_tile=pool_bytes_per_tile, request_cap=request_cap,
                        lod_scalar=lod_scalar, alpha_stop=alpha_stop, jitter_seed=jitter_seed,
                        device_paging=1 if device_paging else 0,
                        load_flags=(N.VV_GVX_CONSTANT_COLORS if constant_colors else 0)
                        | (0 if gradients else N.VV_GVX_SKIP_GRADIENTS),
                        stale_frames=stale_frames, far_dist=far_dist,
                        flags=(N.VV_SCENE_HOST_ONLY if host_only else 0) | (N.VV_SCENE_SYNCHRONOUS if synchronous else 0)
                        | (N.VV_SCENE_BATCHED if batched else 0))
        h = C.c_void_p()
        ch = ctx.handle if ctx is not None else None
        _check(lib().vv_scene_create(ch, str(gvp_path).encode(), C.byref(d), C.byref(h)), ch, "scene create")
        self._h = h
        self.ctx = ctx
        self._size = None

    def close(self) -> None:
        if self._h:
            lib().vv_scene_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, rc: int, what: str) -> None:
        _check(rc, self.ctx.handle if self.ctx is not None else None, what)

    def draw(self, cam: Camera) -> None:
        self._size = (cam.height, cam.width)
        self._ck(lib().vv_scene_draw(self._h, C.byref(cam)), "scene draw")

    def update(self) -> None:
        self._ck(lib().vv_scene_update(self._h), "scene update")

    def wait_loads(self) -> None:
        self._ck(lib().vv_scene_wait_loads(self._h), "scene wait loads")

    def read_color(self) -> np.ndarray:
        out = np.zeros(self._size + (4,), dtype=np.float32)
        self._ck(lib().vv_scene_read_color(self._h, _ptr(out)), "scene read color")
        return out

    def tile_states(self) -> list[dict]:
        n = self.stats()["tiles"]
        arr = (N.SceneTileState * max(n, 1))()
        self._ck(lib().vv_scene_tile_states(self._h, arr, n), "scene tile states")
        return [{f: getattr(t, f) for f, _ in N.SceneTileState._fields_} for t in arr[:n]]

    def stats(self) -> dict:
        s = N.SceneStats()
        self._ck(lib().vv_scene_get_stats(self._h, C.byref(s)), "scene stats")
        return {f: getattr(s, f) for f, _ in N.SceneStats._fields_}

    def tile_renderer(self, tile: int) -> Renderer | None:
        h = lib().vv_scene_tile_renderer(self._h, tile)
        return _TileRenderer(h, self) if h else None
