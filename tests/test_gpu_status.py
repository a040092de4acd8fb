"""Device-side error reporting: loop bounds and index checks end in a status
code the host reads, never in a fault or a hang."""
import numpy as np
import pytest

import voxviz_b200 as vv
from oracle import gv_oracle as go
from tests import helpers

pytestmark = pytest.mark.gpu


def test_loop_bound_sets_timeout_status_and_matches_oracle():
    sc = helpers.Scene(seed=1, depth=4)
    g = helpers.GpuScene(sc)
    u = sc.uniforms(sc.view(3, 64, 64))
    u.max_segments = 6  # far below what the rays need
    got = g.render(u)
    assert got["status"] == vv._native.VV_ERR_TIMEOUT
    ref = helpers.oracle_frame(u, sc.oracle_scene())
    assert ref["status"] == vv._native.VV_ERR_TIMEOUT
    assert np.array_equal(got["usage"], ref["usage"])
    assert np.abs(got["color"] - ref["color"]).max() <= 1 / 255
    # the context stays usable
    u.max_segments = 0
    assert g.render(u)["status"] == 0


def test_out_of_range_patch_and_slot_are_reported():
    sc = helpers.Scene(seed=1, depth=3)
    g = helpers.GpuScene(sc)
    before = g.ctx.download_nodes()
    g.ctx.patch_nodes(np.array([[5000, 0, 0, 1, 2]], dtype=np.uint32))
    g.ctx.synchronize()
    assert g.ctx.device_status() == vv._native.VV_ERR_BOUNDS
    assert np.array_equal(g.ctx.download_nodes(), before)
    total = sc.slots[0] * sc.slots[1] * sc.slots[2]
    g.ctx.upload_bricks(np.array([total + 3], dtype=np.uint32), np.zeros((1, 4000), dtype=np.uint8))
    assert g.ctx.device_status() == vv._native.VV_ERR_BOUNDS
    assert g.ctx.device_status() == 0  # cleared on read
