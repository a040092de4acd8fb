"""Restatement of the paged-scene policy.  TEST INFRASTRUCTURE.

* ``Frustum`` - vox::Frustum::setFromCamera (VoxViz/VoxVizCore/Frustum.cpp:
  13-120) for the projection of ComputePerspective / ComputeFrustum
  (Camera.cpp:44-89) and FlyCamera's view matrix (Camera.cpp:365-395), in
  double, with the matrix product and plane extraction as written there;
  ``sphere`` is sphereInFrustum (:122-135): outside if the centre is at or
  below -radius for any plane, else the near plane's signed distance.
* ``SceneRef.draw`` - the cull visitor (GigaVoxelsRenderer.cpp:667-798):
  visible tiles are stamped with the frame; loaded ones are inserted into
  the render list before the first entry with a smaller distance (distance
  minus radius), the others are requested once (requestLoadOctTree,
  GigaVoxelsDatabasePager.cpp:340-372).
* ``SceneRef.update`` - synchronous pager: requests sorted by last access
  (latest first) then distance (SortByDistAndFrameIndex, :226-236), loaded
  in that order (a failed load stays on the request list and is not retried),
  merged (mergeHandledRequests, :378-415), then tiles unseen for more than
  ``stale_frames`` frames unloaded (:425-453, unsigned difference).
"""
from __future__ import annotations

import math

import numpy as np


class Frustum:
    def __init__(self, position, look, up, fov_y_deg, near, width, height, far=10000.0):
        look = np.asarray(look, dtype=np.float64)
        up = np.asarray(up, dtype=np.float64)
        look = look / np.linalg.norm(look)
        up = up / np.linalg.norm(up)
        left = np.cross(up, look)
        left = left / np.linalg.norm(left)
        e = np.asarray(position, dtype=np.float64)
        u, v, n = -left, up, -look
        modl = [u[0], v[0], n[0], 0.0, u[1], v[1], n[1], 0.0, u[2], v[2], n[2], 0.0,
                -float(e @ u), -float(e @ v), -float(e @ n), 1.0]
        aspect = float(np.float32(width) / np.float32(height))
        ymax = float(near) * float(np.tan(np.float32(fov_y_deg * math.pi / 360.0)))
        xmax = ymax * aspect
        proj = [0.0] * 16
        proj[0] = 2.0 * near / (2.0 * xmax)
        proj[5] = 2.0 * near / (2.0 * ymax)
        proj[10] = (-far - near) / (far - near)
        proj[11] = -1.0
        proj[14] = (-2.0 * near * far) / (far - near)
        clip = [0.0] * 16
        for i in range(4):
            for j in range(4):
                clip[4 * i + j] = (modl[4 * i] * proj[j] + modl[4 * i + 1] * proj[4 + j] + modl[4 * i + 2] * proj[8 + j]
                                   + modl[4 * i + 3] * proj[12 + j])
        planes = []
        for col, sgn in ((0, -1.0), (0, 1.0), (1, 1.0), (1, -1.0), (2, -1.0), (2, 1.0)):
            p = [clip[4 * k + 3] + sgn * clip[4 * k + col] for k in range(4)]
            t = math.sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2])
            planes.append([x / t for x in p])
        self.planes = planes

    def sphere(self, c, r):
        d = 0.0
        for p in self.planes:
            d = p[0] * float(c[0]) + p[1] * float(c[1]) + p[2] * float(c[2]) + p[3]
            if d <= -float(r):
                return None
        return float(np.float32(d))


class SceneRef:
    def __init__(self, tiles, stale_frames=100, far=10000.0, loadable=lambda t: True):
        """tiles: dicts with center, radius (float32 values); loadable(i) says
        whether tile i's tree file loads."""
        self.tiles = tiles
        self.n = len(tiles)
        self.stale = stale_frames
        self.far = far
        self.loadable = loadable
        self.last_access = [0] * self.n
        self.on_list = [False] * self.n
        self.loaded = [False] * self.n
        self.failed = [False] * self.n
        self.visible = [False] * self.n
        self.order = [-1] * self.n
        self.dist = [0.0] * self.n
        self.requests = []
        self.frame = 0
        self.loads = self.unloads = 0

    def draw(self, cam):
        self.frame = int(cam["frame"]) & 0xFFFFFFFFFFFFFFFF
        fr = Frustum(cam["position"], cam["look"], cam["up"], cam["fov"], cam["near"], cam["width"], cam["height"],
                     self.far)
        render = []
        for i, t in enumerate(self.tiles):
            self.visible[i] = False
            self.order[i] = -1
            d = fr.sphere(t["center"], t["radius"])
            if d is None:
                continue
            self.visible[i] = True
            self.last_access[i] = self.frame
            if not self.loaded[i]:
                self.dist[i] = d
                if not self.failed[i] and not self.on_list[i]:
                    self.on_list[i] = True
                    self.requests.append((i, d))
                continue
            self.dist[i] = float(np.float32(np.float32(d) - np.float32(t["radius"])))
            k = 0
            while k < len(render) and not (self.dist[render[k]] < self.dist[i]):
                k += 1
            render.insert(k, i)
        for k, i in enumerate(render):
            self.order[i] = k
        return render

    def update(self):
        reqs = sorted(self.requests, key=lambda r: (-self.last_access[r[0]], r[1]))
        self.requests = []
        handled = []
        for i, _ in reqs:
            if self.loaded[i]:
                self.on_list[i] = False
                continue
            if not self.loadable(i):
                self.failed[i] = True
                continue
            handled.append(i)
        for i in handled:
            self.loaded[i] = True
            self.on_list[i] = False
            self.loads += 1
        for i in range(self.n):
            if self.loaded[i] and ((self.frame - self.last_access[i]) & 0xFFFFFFFFFFFFFFFF) > self.stale:
                self.loaded[i] = False
                self.unloads += 1

    def states(self):
        return [{"loaded": int(self.loaded[i]), "pending": int(self.on_list[i]), "visible": int(self.visible[i]),
                 "drawn_order": self.order[i], "failed": int(self.failed[i]), "last_access": self.last_access[i],
                 "dist_to_near_plane": self.dist[i]} for i in range(self.n)]


def blend_over(dst: np.ndarray, src: np.ndarray) -> np.ndarray:
    """glBlendFunc(GL_SRC_ALPHA, GL_ONE_MINUS_SRC_ALPHA), FP32, products
    rounded separately."""
    a = src[..., 3:4].astype(np.float32)
    ia = (np.float32(1.0) - a).astype(np.float32)
    return ((src * a).astype(np.float32) + (dst * ia).astype(np.float32)).astype(np.float32)
