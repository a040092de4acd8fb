"""The C ABI: the library loads, exports every function the header
declares, and the ctypes structures have the header's layout."""
import re
import subprocess
import ctypes as C
from pathlib import Path

import pytest

import voxviz_b200 as vv
from voxviz_b200 import _native as N

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "voxviz_b200.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(vv_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_function():
    lib = vv.lib()
    names = declared_functions()
    assert len(names) >= 40
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(N.SIGNATURES), set(names) ^ set(N.SIGNATURES)
    assert lib.vv_abi_version() == 1


STRUCTS = {
    "vv_uniforms": N.Uniforms, "vv_node_patch": N.NodePatch, "vv_frame_out": N.FrameOut, "vv_params": N.Params,
    "vv_terrain_desc": N.TerrainDesc, "vv_octree_info": N.OctreeInfo, "vv_node_info": N.NodeInfo,
    "vv_camera": N.Camera, "vv_renderer_desc": N.RendererDesc, "vv_renderer_stats": N.RendererStats,
    "vv_batch_view": N.BatchView, "vv_batch_config": N.BatchConfig,
}


def test_struct_layout_matches_header(tmp_path):
    src = tmp_path / "sizes.c"
    body = "\n".join(f'printf("{k} %zu %zu\\n", sizeof({k}), _Alignof({k}));' for k in STRUCTS)
    src.write_text(f'#include <stdio.h>\n#include "{HEADER}"\nint main(void){{ {body} return 0; }}\n')
    exe = tmp_path / "sizes"
    subprocess.run(["gcc", "-std=c11", str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    for line in filter(None, out):
        name, size, align = line.split()
        assert C.sizeof(STRUCTS[name]) == int(size), name
        assert C.alignment(STRUCTS[name]) == int(align), name


def test_errors_are_status_codes_not_crashes():
    lib = vv.lib()
    assert lib.vv_ctx_create(None, None) == N.VV_ERR_ARG
    assert lib.vv_render(None, 0, None, None) == N.VV_ERR_ARG
    assert lib.vv_octree_build_terrain(None, None) == N.VV_ERR_ARG
    d = N.TerrainDesc(seed=1, depth=11, octaves=4, lacunarity=2.0, gain=0.5, base_cells=4)
    h = C.c_void_p()
    assert lib.vv_octree_build_terrain(C.byref(d), C.byref(h)) == N.VV_ERR_ARG
    assert lib.vv_status_string(N.VV_ERR_TIMEOUT) == b"device loop bound reached"
    with pytest.raises(vv.VVError):
        vv.Octree.terrain(depth=-1)
