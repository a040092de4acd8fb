"""Shared set-up for the parity tests: scenes, device buffers, oracle runs."""
from __future__ import annotations

import numpy as np

import voxviz_b200 as vv
from voxviz_b200 import scene

_OCTREES: dict = {}


def octree(seed=1, depth=5, collapse=True) -> vv.Octree:
    key = (seed, depth, collapse)
    if key not in _OCTREES:
        _OCTREES[key] = vv.Octree.terrain(seed=seed, depth=depth, collapse=collapse)
    return _OCTREES[key]


class Scene:
    """A fully resident scene: node words, brick pool, jitter, slots."""

    def __init__(self, seed=1, depth=5, collapse=True, fmt="rgba8", jitter_seed=7):
        self.octree = octree(seed, depth, collapse)
        self.fmt = vv.fmt_code(fmt)
        self.words, self.pool, self.slots, self.xyz = scene.resident_scene(self.octree, self.fmt)
        self.jitter = vv.make_jitter(jitter_seed)
        self.heights = self.octree.heights()

    def uniforms(self, cam, lod=1.0, alpha=0.99) -> vv.Uniforms:
        return vv.compute_uniforms(self.octree.info, cam, self.slots, lod, alpha)

    def view(self, view_seed, w, h, frame=0):
        return scene.seeded_view(view_seed, self.heights, w, h, frame=frame)

    def oracle_scene(self, pool=None, fmt=None):
        from oracle import gv_oracle as go
        return go.Scene(self.words, self.pool if pool is None else pool, self.slots,
                        self.fmt if fmt is None else fmt, self.jitter)


class GpuScene:
    """The same scene uploaded to a device context, with torch output buffers."""

    def __init__(self, sc: Scene, ctx: vv.Context | None = None):
        self.sc = sc
        self.ctx = ctx or vv.Context(0)
        self.ctx.upload_nodes(sc.words)
        self.ctx.create_brickpool(sc.slots, sc.fmt)
        n = sc.xyz.shape[0]
        self.ctx.upload_bricks(np.arange(n, dtype=np.uint32), sc.pool[:n])
        self.ctx.set_jitter(sc.jitter)

    def render(self, u: vv.Uniforms, max_push=4, cap=None, passes=vv.VV_PASS_ALL):
        import torch
        H, W = u.height, u.width
        dev = torch.device("cuda", 0)
        color = torch.zeros((H, W, 4), dtype=torch.float32, device=dev)
        usage = torch.zeros((H, W, 12), dtype=torch.int32, device=dev)
        mask = torch.zeros((H, W), dtype=torch.int32, device=dev)
        cap = W * H if cap is None else cap
        req = torch.zeros((max(cap, 1), 4), dtype=torch.int32, device=dev)
        cnt = torch.zeros(1, dtype=torch.int32, device=dev)
        self.ctx.render(u, color.data_ptr(), usage.data_ptr(), mask.data_ptr(), req.data_ptr(), cnt.data_ptr(),
                        cap, max_push, passes)
        self.ctx.synchronize()
        status = self.ctx.device_status(clear=True)
        n = int(cnt.item())
        out = {
            "color": color.cpu().numpy(),
            "usage": usage.cpu().numpy().view(np.uint32),
            "mask": mask.cpu().numpy().view(np.uint32),
            "count": n,
            "requests": req.cpu().numpy().view(np.uint32)[:min(n, cap)],
            "status": status,
        }
        return out


def oracle_frame(u, oscene, max_push=4, cap=None, precision=32):
    from oracle import gv_oracle as go
    color, usage, st = go.raycast(u, oscene, precision)
    mask = go.select(usage)
    cap = u.width * u.height if cap is None else cap
    req, total = go.compress(usage, mask, max_push, cap)
    return {"color": color, "usage": usage, "mask": mask, "requests": req, "count": total, "status": st}
