"""The C++ data-model API (include/voxviz_b200.hpp: GigaVoxelsOctTree,
OctTreeNodePool, BrickPool, GigaVoxelsRenderer with the reference's method
names) and the vox::Renderer adapter a maintainer would add to the
reference (tests/cpp/gigavoxels_b200_adapter.h over the stand-in
tests/cpp/vox_renderer.h), compiled with g++ and driven by
tests/cpp/data_model_check.cpp.

* CPU: OctTreeNodePool rebuilt from a terrain octree in the allocation order
  of GigaVoxelsOctTree::build lays out, with create3DTexture's grid rule
  (GigaVoxelsOctTreeNodePool.cpp:90-223), exactly the library's node words.
* GPU: the host data model (processNodeUsageList = NodeUsageListProcessor::run,
  BrickPool::update, OctTreeNodePool::update) services a paged camera path
  with eviction frame by frame identically to the library's device-side
  renderer (requests, residency, LRU order, node words), and the plugin
  driven through vox::Renderer* (draw, postDraw, update) renders the same
  frames as the renderer's own draw + update.
"""
import json
import os
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
CUDA = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))


@pytest.fixture(scope="module")
def check_exe(tmp_path_factory):
    from voxviz_b200 import build as vb

    lib = vb.build()
    exe = tmp_path_factory.mktemp("cpp") / "data_model_check"
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-Wno-unused-parameter",
           "-I", str(ROOT / "include"), "-I", str(ROOT / "tests" / "cpp"), "-I", str(CUDA / "include"),
           str(ROOT / "tests" / "cpp" / "data_model_check.cpp"), "-o", str(exe),
           "-L", str(lib.parent), "-lvoxviz_b200", f"-Wl,-rpath,{lib.parent}",
           "-L", str(CUDA / "lib64"), "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return exe


def _run(exe, *args, timeout=600):
    r = subprocess.run([str(exe), *map(str, args)], capture_output=True, text=True, timeout=timeout)
    assert r.returncode == 0, r.stdout + r.stderr
    return [json.loads(line) for line in r.stdout.splitlines() if line.startswith("{")]


@pytest.mark.parametrize("depth", [3, 4, 5, 6])
@pytest.mark.parametrize("collapse", [0, 1])
def test_node_pool_layout_matches_builder(check_exe, depth, collapse):
    (out,) = _run(check_exe, "layout", depth, collapse)
    assert out["dims_equal"] and out["words_equal"], out
    assert out["levels"] == depth + 1


def _cams(tmp_path, depth, frames, w, h):
    import voxviz_b200 as vv
    from voxviz_b200 import scene
    from tests import helpers

    o = helpers.octree(seed=3, depth=depth)
    cams = scene.camera_path(5, o.heights(), frames, w, h)
    p = tmp_path / "cams.bin"
    p.write_bytes(b"".join(bytes(c) for c in cams))
    assert isinstance(cams[0], vv.Camera)
    return p


@pytest.mark.gpu
def test_host_data_model_services_like_the_renderer(check_exe, tmp_path):
    cams = _cams(tmp_path, 6, 12, 256, 160)
    out = _run(check_exe, "paging", 6, cams, 700)
    summary = out[-1]
    assert summary["check"] == "paging_summary"
    assert summary["equal_frames"] == summary["frames"] == 12, out
    assert summary["evictions"] > 0, "the pool never filled: eviction was not exercised"
    assert summary["requests"] > 0


@pytest.mark.gpu
def test_vox_renderer_adapter_frames(check_exe, tmp_path):
    cams = _cams(tmp_path, 5, 8, 192, 128)
    (out,) = _run(check_exe, "adapter", 5, cams)
    assert out["algorithm"] == "gv"
    assert out["equal_frames"] == out["frames"] == 8, out
