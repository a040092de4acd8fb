"""ctypes view of ``include/voxviz_b200.h`` (the library's C ABI).

The structures here mirror the header field for field; ``check_layout``
compares their sizes with the values the library itself reports.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libvoxviz_b200.so"

VV_OK, VV_ERR_ARG, VV_ERR_OOM, VV_ERR_CUDA, VV_ERR_TIMEOUT, VV_ERR_BOUNDS, VV_ERR_STATE, VV_ERR_NODEV, VV_ERR_IO = range(9)
VV_GVX_CONSTANT_COLORS, VV_GVX_SKIP_GRADIENTS = 1, 2
VV_SCENE_HOST_ONLY, VV_SCENE_SYNCHRONOUS, VV_SCENE_BATCHED = 1, 2, 4
VV_FMT_RGBA8, VV_FMT_FP16, VV_FMT_BF16, VV_FMT_FP32, VV_FMT_DXT5, VV_FMT_DXT1 = range(6)
VV_PASS_RAYCAST, VV_PASS_SELECT, VV_PASS_COMPACT, VV_PASS_ALL = 1, 2, 4, 7
VV_PASS_COLOR_RGBA8 = 8
FMT_NAMES = {"rgba8": VV_FMT_RGBA8, "fp16": VV_FMT_FP16, "bf16": VV_FMT_BF16, "fp32": VV_FMT_FP32,
             "dxt5": VV_FMT_DXT5, "dxt1": VV_FMT_DXT1}
TEXEL_BYTES = {VV_FMT_RGBA8: 4, VV_FMT_FP16: 8, VV_FMT_BF16: 8, VV_FMT_FP32: 16}
# bytes of one stored brick (pool slot): 1000 texels, or 90 S3TC blocks
BRICK_BYTES = {VV_FMT_RGBA8: 4000, VV_FMT_FP16: 8000, VV_FMT_BF16: 8000, VV_FMT_FP32: 16000, VV_FMT_DXT5: 1440,
               VV_FMT_DXT1: 720}

f3 = C.c_float * 3
i3 = C.c_int32 * 3


class Uniforms(C.Structure):
    _fields_ = [
        ("ray_step_size", C.c_float),
        ("brick_step_vector", f3),
        ("camera_position", f3),
        ("camera_up", f3),
        ("camera_left", f3),
        ("vol_extent_min", f3),
        ("vol_extent_max", f3),
        ("brick_dimension", f3),
        ("root_voxel_half_size", C.c_float),
        ("brick_pool_dimension", f3),
        ("pixel_size", C.c_float),
        ("lod_scalar", C.c_float),
        ("alpha_stop", C.c_float),
        ("oct_tree_depth_minus_one", C.c_int32),
        ("max_nodes_to_push", C.c_int32),
        ("root_node_is_constant", C.c_int32),
        ("jitter_tex_size", C.c_int32),
        ("width", C.c_int32),
        ("height", C.c_int32),
        ("camera_inside", C.c_int32),
        ("max_segments", C.c_int32),
        ("near_origin", f3),
        ("near_dx", f3),
        ("near_dy", f3),
        ("light_position", f3),
        ("compute_lighting", C.c_int32),
        ("gradients_unsigned", C.c_int32),
    ]


class NodePatch(C.Structure):
    _fields_ = [("x", C.c_uint32), ("y", C.c_uint32), ("z", C.c_uint32), ("word0", C.c_uint32), ("word1", C.c_uint32)]


class FrameOut(C.Structure):
    _fields_ = [
        ("color", C.c_void_p),
        ("usage", C.c_void_p),
        ("mask", C.c_void_p),
        ("requests", C.c_void_p),
        ("request_count", C.c_void_p),
        ("request_cap", C.c_int32),
        ("compress_max_push", C.c_int32),
        ("passes", C.c_int32),
    ]


class Params(C.Structure):
    _fields_ = [("device", C.c_int32), ("flags", C.c_int32), ("reserved", C.c_int64 * 4)]


class TerrainDesc(C.Structure):
    _fields_ = [
        ("seed", C.c_uint32),
        ("depth", C.c_int32),
        ("octaves", C.c_int32),
        ("lacunarity", C.c_float),
        ("gain", C.c_float),
        ("base_cells", C.c_int32),
        ("collapse_constant", C.c_int32),
        ("threads", C.c_int32),
    ]


class OctreeInfo(C.Structure):
    _fields_ = [
        ("depth", C.c_int32),
        ("volume_dim", C.c_int32),
        ("node_count", C.c_int64),
        ("pool_dim", i3),
        ("nonconst_count", C.c_int64),
        ("root_is_constant", C.c_int32),
        ("root_word0", C.c_uint32),
        ("root_word1", C.c_uint32),
    ]


class GvxInfo(C.Structure):
    _fields_ = [
        ("file_backed", C.c_int32),
        ("max_depth", C.c_int32),
        ("origin", C.c_float * 3),
        ("delta", C.c_float * 3),
        ("volume_size", i3),
        ("brick_size", i3),
        ("bricks", C.c_int64),
        ("has_gradients", C.c_int32),
        ("ray_step_size", C.c_float),
    ]


class GvpTile(C.Structure):
    _fields_ = [
        ("center", C.c_float * 3),
        ("radius", C.c_float),
        ("size_meters", C.c_float * 3),
        ("tree_file", C.c_char * 1024),
    ]


class GvpInfo(C.Structure):
    _fields_ = [
        ("compressed", C.c_int32),
        ("brick_size", i3),
        ("tiles", C.c_int32),
        ("sphere_center", C.c_float * 3),
        ("sphere_radius", C.c_double),
    ]


class SceneDesc(C.Structure):
    _fields_ = [
        ("fmt", C.c_int32),
        ("pool_bytes_per_tile", C.c_int64),
        ("request_cap", C.c_int32),
        ("lod_scalar", C.c_float),
        ("alpha_stop", C.c_float),
        ("jitter_seed", C.c_uint32),
        ("device_paging", C.c_int32),
        ("load_flags", C.c_int32),
        ("stale_frames", C.c_int32),
        ("far_dist", C.c_float),
        ("flags", C.c_int32),
        ("reserved", C.c_int32 * 4),
    ]


class SceneTileState(C.Structure):
    _fields_ = [
        ("loaded", C.c_int32),
        ("pending", C.c_int32),
        ("visible", C.c_int32),
        ("drawn_order", C.c_int32),
        ("failed", C.c_int32),
        ("dist_to_near_plane", C.c_float),
        ("last_access", C.c_int64),
    ]


class SceneStats(C.Structure):
    _fields_ = [
        ("tiles", C.c_int32), ("loaded", C.c_int32), ("pending", C.c_int32), ("drawn", C.c_int32),
        ("loads", C.c_int64), ("unloads", C.c_int64), ("load_failures", C.c_int64),
        ("load_ms_avg", C.c_float), ("load_ms_max", C.c_float),
    ]


class NodeInfo(C.Structure):
    _fields_ = [
        ("valid", C.c_int32),
        ("level", C.c_int32),
        ("origin", i3),
        ("is_constant", C.c_int32),
        ("has_children", C.c_int32),
        ("parent", i3),
    ]


class Camera(C.Structure):
    _fields_ = [
        ("position", f3),
        ("look", f3),
        ("up", f3),
        ("fov_y_deg", C.c_float),
        ("near_dist", C.c_float),
        ("width", C.c_int32),
        ("height", C.c_int32),
        ("frame", C.c_int32),
    ]


class RendererDesc(C.Structure):
    _fields_ = [
        ("fmt", C.c_int32),
        ("pool_bytes", C.c_int64),
        ("preload_all", C.c_int32),
        ("request_cap", C.c_int32),
        ("lod_scalar", C.c_float),
        ("alpha_stop", C.c_float),
        ("jitter_seed", C.c_uint32),
        ("max_width", C.c_int32),
        ("max_height", C.c_int32),
        ("producer_threads", C.c_int32),
        ("device_paging", C.c_int32),
        ("color_rgba8", C.c_int32),
    ]


class RendererStats(C.Structure):
    _fields_ = [
        ("frame", C.c_int64),
        ("requests", C.c_int64),
        ("active_pixels", C.c_int64),
        ("bricks_uploaded", C.c_int64),
        ("bricks_uploaded_total", C.c_int64),
        ("resident_bricks", C.c_int64),
        ("evictions_total", C.c_int64),
        ("pool_slots", C.c_int32),
        ("ms_readback", C.c_float),
        ("ms_policy", C.c_float),
        ("ms_produce", C.c_float),
        ("ms_upload", C.c_float),
        ("ms_visit", C.c_float),
        ("unique_nodes", C.c_int32),
    ]


class GradDesc(C.Structure):
    _fields_ = [("grad", C.c_void_p), ("flags", C.c_int32), ("rows_cap", C.c_int32), ("slot_map", C.c_void_p),
                ("rows_used", C.c_void_p)]


VV_GRAD_F64, VV_GRAD_WARP_SUM, VV_GRAD_SPREAD, VV_GRAD_SPREAD_KEEP = 1, 2, 4, 8
VV_RAYCAST_TILES, VV_RAYCAST_REFILL, VV_RAYCAST_STAGED = 0, 1, 2
VV_COMPACT_FUSED, VV_COMPACT_PER_LEVEL = 0, 1


class BatchView(C.Structure):
    _fields_ = [
        ("ctx", C.c_void_p),
        ("tree", C.c_int32),
        ("pad", C.c_int32),
        ("u", Uniforms),
        ("color", C.c_void_p),
        ("usage", C.c_void_p),
    ]


class BatchConfig(C.Structure):
    _fields_ = [("tile_w", C.c_int32), ("tile_h", C.c_int32), ("steps", C.c_int32), ("ctas_per_sm", C.c_int32)]


P = C.c_void_p
u32p = C.POINTER(C.c_uint32)
i32p = C.POINTER(C.c_int32)

# name: (restype, argtypes)
SIGNATURES = {
    "vv_abi_version": (C.c_int, []),
    "vv_status_string": (C.c_char_p, [C.c_int]),
    "vv_ctx_create": (C.c_int, [C.POINTER(Params), C.POINTER(P)]),
    "vv_ctx_destroy": (C.c_int, [P]),
    "vv_last_error": (C.c_char_p, [P]),
    "vv_ctx_set_stream": (C.c_int, [P, P]),
    "vv_ctx_synchronize": (C.c_int, [P]),
    "vv_ctx_device_status": (C.c_int, [P, i32p, C.c_int32]),
    "vv_nodepool_upload": (C.c_int, [P, C.c_int32, P, C.c_int32, C.c_int32, C.c_int32]),
    "vv_nodepool_patch": (C.c_int, [P, C.c_int32, P, C.c_int32]),
    "vv_nodepool_download": (C.c_int, [P, C.c_int32, P]),
    "vv_brickpool_create": (C.c_int, [P, C.c_int32, C.c_int32, C.c_int32, C.c_int32]),
    "vv_upload_bricks": (C.c_int, [P, P, C.c_int32, P]),
    "vv_upload_bricks_device": (C.c_int, [P, P, C.c_int32, P]),
    "vv_gradpool_create": (C.c_int, [P, C.c_int32]),
    "vv_upload_gradients": (C.c_int, [P, P, C.c_int32, P]),
    "vv_gradpool_download": (C.c_int, [P, P]),
    "vv_octree_produce_gradients": (C.c_int, [P, P, C.c_int32, C.c_int32, P]),
    "vv_brickpool_download": (C.c_int, [P, P]),
    "vv_brickpool_update_cell_masks": (C.c_int, [P]),
    "vv_brickpool_download_cell_masks": (C.c_int, [P, P]),
    "vv_brickpool_info": (C.c_int, [P, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "vv_nodepool_info": (C.c_int, [P, C.c_int32, C.POINTER(C.c_int32)]),
    "vv_brickpool_device_ptr": (C.c_int, [P, C.POINTER(P), C.POINTER(C.c_size_t)]),
    "vv_set_jitter": (C.c_int, [P, P, C.c_int32]),
    "vv_render": (C.c_int, [P, C.c_int32, C.POINTER(Uniforms), C.POINTER(FrameOut)]),
    "vv_compact_requests_noalloc": (C.c_int, [P, P, C.c_int32, C.c_int32, P, P, C.c_int32, C.c_int32, P]),
    "vv_ctx_set_profiling": (C.c_int, [P, C.c_int32]),
    "vv_ctx_set_raycast_mode": (C.c_int, [P, C.c_int32]),
    "vv_ctx_set_compaction": (C.c_int, [P, C.c_int32]),
    "vv_ckpt_bytes": (C.c_size_t, [C.c_int32, C.c_int32, C.c_int32]),
    "vv_render_forward_ckpt": (C.c_int, [P, C.c_int32, C.POINTER(Uniforms), P, P, C.c_int32]),
    "vv_backward": (C.c_int, [P, C.c_int32, C.POINTER(Uniforms), P, P, C.c_int32, P]),
    "vv_backward_ex": (C.c_int, [P, C.c_int32, C.POINTER(Uniforms), P, P, C.c_int32, C.POINTER(GradDesc)]),
    "vv_brickpool_attach": (C.c_int, [P, P, C.c_int32, C.c_int32, C.c_int32, C.c_int32]),
    "vv_batch_variants": (C.c_int32, [C.POINTER(BatchConfig), C.c_int32]),
    "vv_render_batch": (C.c_int, [P, C.POINTER(BatchView), C.c_int32, C.POINTER(BatchConfig)]),
    "vv_batch_autotune": (C.c_int, [P, C.POINTER(BatchView), C.c_int32, C.c_int32, C.POINTER(BatchConfig),
                                    C.POINTER(C.c_float)]),
    "vv_ctx_last_times": (C.c_int, [P, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "vv_measure_footprint": (C.c_int, [P, C.c_int32, C.POINTER(Uniforms), C.POINTER(C.c_int64),
                                       C.POINTER(C.c_int64)]),
    "vv_measure_footprint_views": (C.c_int, [P, C.c_int32, C.POINTER(Uniforms), C.c_int32, C.POINTER(C.c_int64),
                                             C.POINTER(C.c_int64)]),
    "vv_octree_build_terrain": (C.c_int, [C.POINTER(TerrainDesc), C.POINTER(P)]),
    "vv_octree_build_terrain_gpu": (C.c_int, [C.POINTER(TerrainDesc), C.c_int32, C.POINTER(P)]),
    "vv_octree_destroy": (None, [P]),
    "vv_octree_get_info": (C.c_int, [P, C.POINTER(OctreeInfo)]),
    "vv_octree_node_words": (C.c_int, [P, P]),
    "vv_octree_node_info": (C.c_int, [P, C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(NodeInfo)]),
    "vv_octree_produce_bricks": (C.c_int, [P, P, C.c_int32, C.c_int32, P]),
    "vv_octree_mip_level": (C.c_int, [P, C.c_int32, P, C.c_size_t]),
    "vv_octree_heights": (C.c_int, [P, P]),
    "vv_octree_load_gvx": (C.c_int, [C.c_char_p, C.c_int32, C.POINTER(P)]),
    "vv_octree_save_gvx": (C.c_int, [P, C.c_char_p, C.c_int32]),
    "vv_octree_gvx_info": (C.c_int, [P, C.POINTER(GvxInfo)]),
    "vv_gvp_read": (C.c_int, [C.c_char_p, C.POINTER(GvpInfo), C.POINTER(GvpTile), C.c_int32]),
    "vv_gvp_write": (C.c_int, [C.c_char_p, C.POINTER(GvpInfo), C.POINTER(GvpTile), C.c_int32]),
    "vv_scene_create": (C.c_int, [P, C.c_char_p, C.POINTER(SceneDesc), C.POINTER(P)]),
    "vv_scene_destroy": (None, [P]),
    "vv_scene_draw": (C.c_int, [P, C.POINTER(Camera)]),
    "vv_scene_update": (C.c_int, [P]),
    "vv_scene_wait_loads": (C.c_int, [P]),
    "vv_scene_read_color": (C.c_int, [P, P]),
    "vv_scene_tile_states": (C.c_int, [P, C.POINTER(SceneTileState), C.c_int32]),
    "vv_scene_get_stats": (C.c_int, [P, C.POINTER(SceneStats)]),
    "vv_scene_tile_renderer": (P, [P, C.c_int32]),
    "vv_compute_uniforms": (C.c_int, [C.POINTER(OctreeInfo), C.POINTER(Camera), C.c_int32, C.c_int32, C.c_int32,
                                      C.c_float, C.c_float, C.POINTER(Uniforms)]),
    "vv_camera_pixel_size": (C.c_float, [C.POINTER(Camera)]),
    "vv_make_jitter": (C.c_int, [C.c_uint32, C.c_int32, P]),
    "vv_renderer_create": (C.c_int, [P, P, C.POINTER(RendererDesc), C.POINTER(P)]),
    "vv_renderer_destroy": (None, [P]),
    "vv_renderer_draw": (C.c_int, [P, C.POINTER(Camera)]),
    "vv_renderer_update": (C.c_int, [P]),
    "vv_renderer_draw_passes": (C.c_int, [P, C.POINTER(Camera), C.c_int32]),
    "vv_renderer_post_draw": (C.c_int, [P]),
    "vv_renderer_service": (C.c_int, [P, P, P, C.c_int32]),
    "vv_renderer_set_deferred": (C.c_int, [P, C.c_int32]),
    "vv_renderer_stage_uploads": (C.c_int, [P]),
    "vv_renderer_enqueue_uploads": (C.c_int, [P]),
    "vv_renderer_get_stats": (C.c_int, [P, C.POINTER(RendererStats)]),
    "vv_renderer_frame_buffers": (C.c_int, [P, C.POINTER(P), C.POINTER(P), C.POINTER(P), C.POINTER(P), C.POINTER(P)]),
    "vv_renderer_read_color": (C.c_int, [P, P]),
    "vv_renderer_read_color_async": (C.c_int, [P, P]),
    "vv_renderer_wait_readback": (C.c_int, [P]),
    "vv_renderer_read_lists": (C.c_int, [P, P, P]),
    "vv_renderer_last_requests": (C.c_int, [P, P, C.c_int32, i32p]),
    "vv_renderer_residency": (C.c_int, [P, P, P, C.c_int64, C.POINTER(C.c_int64)]),
    "vv_renderer_lru_order": (C.c_int, [P, P, C.c_int64, C.POINTER(C.c_int64)]),
    "vv_renderer_last_uniforms": (C.c_int, [P, C.POINTER(Uniforms)]),
    "vv_renderer_ctx": (P, [P]),
}

_lib = None


def load(path: str | os.PathLike | None = None) -> C.CDLL:
    """Load the native library and declare every entry point."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(
            f"{p} is missing: build it with `python -m voxviz_b200.build` (there is no fallback path)")
    lib = C.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


class VVError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"vv status {code}: {msg}")
        self.code = code
