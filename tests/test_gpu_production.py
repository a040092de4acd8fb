"""GPU brick production (device copy of the column-run mip pyramid) writes
exactly the bricks the host builder produces, in every pool format."""
import numpy as np
import pytest

import voxviz_b200 as vv
from tests import helpers

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("fmt", ["rgba8", "fp16", "bf16", "fp32"])
@pytest.mark.parametrize("depth,collapse", [(4, False), (6, True)])
def test_device_production_matches_host_builder(fmt, depth, collapse):
    o = helpers.octree(seed=9, depth=depth, collapse=collapse)
    ctx = vv.Context(0)
    r = vv.Renderer(ctx, o, fmt=fmt, preload_all=True, device_paging=True)
    pool = ctx.download_bricks()
    xyz, slot = r.residency()
    assert len(slot) == o.info.nonconst_count
    assert np.array_equal(pool[slot], o.produce_bricks(xyz, fmt))
    assert ctx.device_status() == 0
