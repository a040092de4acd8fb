"""Restatement of the page-request service policy.  TEST INFRASTRUCTURE.

NodeUsageListProcessor::run (VoxViz/GigaVoxels/GigaVoxelsOctTree.cpp:430-657)
decodes the compacted list, keeps each node once, touches resident bricks
and queues non-constant, non-resident nodes; BrickPool::update
(VoxViz/GigaVoxels/GigaVoxelsBrickPool.cpp:561-682) uploads each queued node
into the least recently used slot and also its parent when the parent is
non-constant and not resident; GigaVoxelsOctTree::update touches the root
every frame (GigaVoxelsOctTree.cpp:1821-1850).

The reference runs this on worker threads with tryLock, so its order is not
reproducible.  The policy both sides implement is the synchronous one:
unique nodes in first-seen order of the list, touches in that order, then the
root, then uploads in that order; the LRU list starts with the empty slots in
slot-id order.  This module derives the tree from the node words alone.
"""
from __future__ import annotations

from collections import OrderedDict

import numpy as np

RESIDENT = 0x80000000
CONSTANT = 0x40000000


class PagingRef:
    def __init__(self, words: np.ndarray, slots: tuple[int, int, int], borders: dict | None = None):
        """borders: grid cell -> (bx, by, bz), where a brick's 8^3 voxels
        start in its slot (BrickPool::uploadBrick sets the node pointer to
        slot origin + border, GigaVoxelsBrickPool.cpp:800-808); (1, 1, 1)
        for cells not listed."""
        self.words = np.array(words, dtype=np.uint32, copy=True)  # (dz, dy, dx, 2)
        self.borders = borders or {}
        self.sx, self.sy, self.sz = slots
        self.total = self.sx * self.sy * self.sz
        self.lru: OrderedDict[int, None] = OrderedDict((s, None) for s in range(self.total))
        self.slot_node: dict[int, tuple] = {}
        self.node_slot: dict[tuple, int] = {}
        self._derive_tree()

    def _derive_tree(self) -> None:
        """Parent of every node reachable from the root (flat grid index,
        -1 for the root and for cells no reachable node points at), level by
        level from the root's child pointer (NodeTree::getNode,
        GigaVoxelsOctTree.cpp:56-73, walks the same pointers)."""
        dz, dy, dx, _ = self.words.shape
        self.dims = (dx, dy, dz)
        n = dx * dy * dz
        w0 = self.words[..., 0].reshape(-1)
        self.parent_flat = np.full(n, -1, dtype=np.int64)
        self.valid_flat = np.zeros(n, dtype=bool)
        self.valid_flat[0] = True
        offs = np.array([(k & 1) + ((k >> 1) & 1) * dx + (k >> 2) * dx * dy for k in range(8)], dtype=np.int64)
        level = np.array([0], dtype=np.int64)
        while level.size:
            c = w0[level]
            has = (c & np.uint32(0x3FFFFFFF)) != 0
            par = level[has]
            c = c[has].astype(np.int64)
            base = ((c >> 20) & 1023) + ((c >> 10) & 1023) * dx + (c & 1023) * dx * dy
            ch = (base[:, None] + offs[None, :]).reshape(-1)
            self.parent_flat[ch] = np.repeat(par, 8)
            self.valid_flat[ch] = True
            level = ch

    def _flat(self, n) -> int:
        return n[0] + n[1] * self.dims[0] + n[2] * self.dims[0] * self.dims[1]

    def _cell(self, f: int) -> tuple:
        dx, dy, _ = self.dims
        return (f % dx, (f // dx) % dy, f // (dx * dy))

    def is_constant(self, n) -> bool:
        return bool(int(self.words[n[2], n[1], n[0], 0]) & CONSTANT)

    def _upload(self, n) -> None:
        s = next(iter(self.lru))
        old = self.slot_node.get(s)
        if old is not None:
            del self.node_slot[old]
            self.words[old[2], old[1], old[0], 0] &= np.uint32(~RESIDENT & 0xFFFFFFFF)
        self.slot_node[s] = n
        self.node_slot[n] = s
        x, y, z = s % self.sx, (s // self.sx) % self.sy, s // (self.sx * self.sy)
        bx, by, bz = self.borders.get(n, (1, 1, 1))
        self.words[n[2], n[1], n[0], 1] = ((x * 10 + bx) << 20) | ((y * 10 + by) << 10) | (z * 10 + bz)
        self.words[n[2], n[1], n[0], 0] |= np.uint32(RESIDENT)
        self.lru.move_to_end(s)
        self.uploaded.append(n)

    def set_state(self, lru_order, xyz, slot) -> None:
        """Start from a given paging state: the LRU order (slots, least
        recently used first) and the resident nodes' slots.  The node words
        passed to the constructor must already carry that residency."""
        order = [int(s) for s in np.asarray(lru_order).reshape(-1)]
        if sorted(order) != list(range(self.total)):
            raise ValueError("the LRU order is not a permutation of the slots")
        self.lru = OrderedDict((s, None) for s in order)
        self.slot_node, self.node_slot = {}, {}
        for p, s in zip(np.asarray(xyz).reshape(-1, 3), np.asarray(slot).reshape(-1)):
            n = (int(p[0]), int(p[1]), int(p[2]))
            self.slot_node[int(s)] = n
            self.node_slot[n] = int(s)

    def lru_order(self) -> np.ndarray:
        return np.fromiter(self.lru.keys(), dtype=np.uint32, count=len(self.lru))

    def init(self, preload_all: bool) -> None:
        self.uploaded = []
        if preload_all:
            raise NotImplementedError("the paging checks start from the root brick only")
        if not self.is_constant((0, 0, 0)):
            self._upload((0, 0, 0))

    def distinct_nodes(self, requests: np.ndarray) -> list:
        """The compacted list's node ids decoded (the +1 of
        AddToNodeUsageList removed), zeros and cells outside the tree dropped,
        each node once in first-seen order."""
        v = np.asarray(requests, dtype=np.uint32).reshape(-1)
        v = v[v != 0].astype(np.int64)
        x, y, z = ((v >> 20) & 1023) - 1, ((v >> 10) & 1023) - 1, (v & 1023) - 1
        dx, dy, dz = self.dims
        ok = (x >= 0) & (x < dx) & (y >= 0) & (y < dy) & (z >= 0) & (z < dz)
        f = (x + y * dx + z * dx * dy)[ok]
        f = f[self.valid_flat[f]]
        _, first = np.unique(f, return_index=True)
        return [self._cell(int(c)) for c in f[np.sort(first)]]

    def update(self, requests: np.ndarray) -> list:
        """Service one frame's compacted list (n x 4 words); returns uploads."""
        self.uploaded = []
        queue = []
        for n in self.distinct_nodes(requests):
            if n in self.node_slot:
                self.lru.move_to_end(self.node_slot[n])
            elif not self.is_constant(n):
                queue.append(n)
        if (0, 0, 0) in self.node_slot:
            self.lru.move_to_end(self.node_slot[(0, 0, 0)])
        for n in queue:
            if n in self.node_slot:
                continue
            self._upload(n)
            pf = int(self.parent_flat[self._flat(n)])
            if pf >= 0:
                p = self._cell(pf)
                if not self.is_constant(p) and p not in self.node_slot:
                    self._upload(p)
        return list(self.uploaded)

    def residency(self) -> dict:
        return dict(self.node_slot)
