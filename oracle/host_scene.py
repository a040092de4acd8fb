"""Host-only resident scene for the CPU reference runs.  TEST INFRASTRUCTURE.

The CPU reference arm of bench.py must not touch the CUDA library's device
paths, so it reproduces on the host what the page-request loop converges
to: render a sample with the oracle, decode every node id the rays recorded
(the raw NodeUsageList entries of GigaVoxelsNoLighting.frag:454-488), make
the non-constant ones resident (brick produced by the octree builder, next
free slot), and repeat until no new node is requested.
"""
from __future__ import annotations

import numpy as np

from . import gv_oracle as go

RESIDENT = np.uint32(0x80000000)
CONSTANT = np.uint32(0x40000000)


class HostScene:
    def __init__(self, octree, slots, fmt: int, jitter: np.ndarray):
        from voxviz_b200 import TEXEL_BYTES

        self.octree = octree
        self.slots = tuple(slots)
        self.fmt = fmt
        self.words = octree.node_words()
        n = slots[0] * slots[1] * slots[2]
        self.pool = np.zeros((n, 1000 * TEXEL_BYTES[fmt]), dtype=np.uint8)
        self.next_slot = 0
        self.jitter = np.ascontiguousarray(jitter, dtype=np.uint8)
        self.scene = go.Scene(self.words, self.pool, self.slots, fmt, self.jitter)
        w0 = self.words[0, 0, 0, 0]
        if not w0 & CONSTANT:
            self._make_resident(np.array([[0, 0, 0]], dtype=np.uint32))

    def _make_resident(self, xyz: np.ndarray) -> int:
        xyz = np.asarray(xyz, dtype=np.uint32).reshape(-1, 3)
        if xyz.size == 0:
            return 0
        n = xyz.shape[0]
        if self.next_slot + n > self.pool.shape[0]:
            raise RuntimeError("host brick pool full")
        s = np.arange(self.next_slot, self.next_slot + n, dtype=np.int64)
        sx, sy, _ = self.slots
        ptr = ((((s % sx) * 10 + 1) << 20) | ((((s // sx) % sy) * 10 + 1) << 10) | ((s // (sx * sy)) * 10 + 1))
        self.pool[self.next_slot:self.next_slot + n] = self.octree.produce_bricks(xyz, self.fmt)
        self.words[xyz[:, 2], xyz[:, 1], xyz[:, 0], 1] = ptr.astype(np.uint32)
        self.words[xyz[:, 2], xyz[:, 1], xyz[:, 0], 0] |= RESIDENT
        self.next_slot += n
        return n

    def converge(self, uniforms_list, rows=None, threads: int = 0, max_iter: int = 16) -> int:
        """Make resident every node the given draws request; returns bricks made resident."""
        total = 0
        for _ in range(max_iter):
            new = set()
            for u in uniforms_list:
                _, usage, _ = go.raycast(u, self.scene, 32, rows=rows, threads=threads)
                ids = np.unique(usage[usage != 0])
                x = ((ids >> 20) & 1023).astype(np.int64) - 1
                y = ((ids >> 10) & 1023).astype(np.int64) - 1
                z = (ids & 1023).astype(np.int64) - 1
                w0 = self.words[z, y, x, 0]
                need = ((w0 & CONSTANT) == 0) & ((w0 & RESIDENT) == 0)
                for a, b, c in zip(x[need], y[need], z[need]):
                    new.add((int(a), int(b), int(c)))
            if not new:
                break
            total += self._make_resident(np.array(sorted(new), dtype=np.uint32))
        return total
