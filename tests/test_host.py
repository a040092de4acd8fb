"""Host-side logic: uniform derivation, pixel size, jitter, camera paths and
the paging policy restatement."""
import math

import numpy as np
import pytest

import voxviz_b200 as vv
from voxviz_b200 import scene
from oracle.paging_ref import PagingRef


def _glu_pixel_size(cam):
    """Camera::getPixelSize with explicit matrices and gluUnProject (Camera.cpp:128-196)."""
    n, f = float(cam.near_dist), 10000.0
    ymax = n * math.tan(np.float32(cam.fov_y_deg * math.pi / 360.0))
    xmax = ymax * float(np.float32(cam.width) / np.float32(cam.height))
    P = np.array([[n / xmax, 0, 0, 0], [0, n / ymax, 0, 0], [0, 0, (-f - n) / (f - n), -2 * f * n / (f - n)],
                  [0, 0, -1, 0]])
    eye = np.array(cam.position[:], np.float64)
    look = np.array(cam.look[:], np.float64)
    up = np.array(cam.up[:], np.float64)
    s = np.cross(look, up)
    s /= np.linalg.norm(s)
    u2 = np.cross(s, look)
    M = np.eye(4)
    M[0, :3], M[1, :3], M[2, :3] = s, u2, -look
    M[:3, 3] = -M[:3, :3] @ eye
    inv = np.linalg.inv(P @ M)

    def unproject(wx, wy):
        v = inv @ np.array([2 * wx / cam.width - 1, 2 * wy / cam.height - 1, -1.0, 1.0])
        return v[:3] / v[3]

    a = unproject(cam.width * 0.5, cam.height * 0.5) - eye
    b = unproject(cam.width * 0.5 + 1, cam.height * 0.5 + 1) - eye
    return 1.0 - np.dot(a / np.linalg.norm(a), b / np.linalg.norm(b))


@pytest.mark.parametrize("w,h", [(512, 512), (1920, 1080), (333, 777)])
def test_pixel_size_matches_unprojection(w, h):
    look, up = vv.look_at([0.2, 0.3, 1.5], [0.5, 0.5, 0.4])
    cam = vv.make_camera([0.2, 0.3, 1.5], look, up, w, h, near=0.01)
    assert vv.pixel_size(cam) == pytest.approx(_glu_pixel_size(cam), rel=1e-4)


def test_uniforms_follow_draw_volume():
    o = vv.Octree.terrain(seed=1, depth=5)
    look, up = vv.look_at([1.2, -0.4, 1.1], [0.5, 0.5, 0.45])
    cam = vv.make_camera([1.2, -0.4, 1.1], look, up, 512, 512, frame=3)
    u = vv.compute_uniforms(o.info, cam, (27, 24, 24), 1.0, 0.99)
    assert u.ray_step_size == np.float32(0.5 / 256)
    assert u.oct_tree_depth_minus_one == 5
    assert u.max_nodes_to_push == 24          # 12 * (frame % 2 + 1)
    assert u.root_voxel_half_size == np.float32(1 / 16)
    assert list(u.brick_pool_dimension) == [270.0, 240.0, 240.0]
    # BrickStepVector = (1/poolDim) * (rayStep * 2^L / (1/8))
    for a, pd in enumerate((270.0, 240.0, 240.0)):
        expect = np.float32(np.float32(1.0) / np.float32(pd)) * np.float32(np.float32(0.5 / 256) * np.float32(32) / np.float32(0.125))
        assert u.brick_step_vector[a] == expect
    assert u.camera_inside == 0
    assert list(u.vol_extent_min) == [0.0, 0.0, 0.0] and list(u.vol_extent_max) == [1.0, 1.0, 1.0]
    # the centre pixel's near-plane point lies on the look axis
    d = np.array(u.near_origin[:]) + 256 * np.array(u.near_dx[:]) + 256 * np.array(u.near_dy[:])
    assert np.allclose(d / np.linalg.norm(d), look, atol=1e-6)


def test_jitter_values_in_range_and_seeded():
    a, b = vv.make_jitter(7), vv.make_jitter(7)
    assert np.array_equal(a, b) and a.min() >= 1 and a.max() <= 255 and a.size == 1024
    assert not np.array_equal(a, vv.make_jitter(8))
    assert len(np.unique(a)) > 200


def test_camera_path_stays_above_terrain():
    o = vv.Octree.terrain(seed=4, depth=6)
    H = o.heights()
    cams = scene.camera_path(9, H, 64, 320, 180)
    assert len(cams) == 64
    for c in cams:
        x, y, z = c.position
        assert 0 < x < 1 and 0 < y < 1
        assert z > scene.terrain_height(H, x, y)
        assert abs(np.linalg.norm(np.array(c.look[:])) - 1) < 1e-5


def test_paging_policy_known_answer():
    # root (non-constant, children block at (2,0,0)) and 8 children, 3 slots
    words = np.zeros((2, 2, 4, 2), dtype=np.uint32)
    words[0, 0, 0, 0] = (2 << 20)
    for k in range(8):
        x, y, z = 2 + (k & 1), (k >> 1) & 1, k >> 2
        words[z, y, x, 0] = 0x40000000 if k % 2 else 0   # odd children constant
    sim = PagingRef(words, (3, 1, 1))
    sim.init(False)
    assert sim.residency() == {(0, 0, 0): 0}
    ident = lambda n: ((n[0] + 1) << 20) | ((n[1] + 1) << 10) | (n[2] + 1)
    req = np.array([[ident((2, 0, 0)), ident((3, 0, 0)), ident((2, 0, 0)), 0],
                    [ident((2, 1, 0)), 0, 0, 0]], dtype=np.uint32)
    up = sim.update(req)
    assert up == [(2, 0, 0), (2, 1, 0)]               # constant (3,0,0) skipped, duplicate dropped
    assert sim.residency() == {(0, 0, 0): 0, (2, 0, 0): 1, (2, 1, 0): 2}
    up = sim.update(np.array([[ident((2, 0, 1)), 0, 0, 0]], dtype=np.uint32))
    # LRU front is slot 1: (2,1,0) was uploaded after (2,0,0); the root was touched
    assert up == [(2, 0, 1)] and sim.residency()[(2, 0, 1)] == 1
    assert not words[0, 0, 2, 0] & 0x80000000
    assert sim.words[0, 0, 2, 0] & 0x80000000 == 0 and sim.words[1, 0, 2, 0] & 0x80000000
