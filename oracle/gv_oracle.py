"""ctypes binding of the CPU oracle (liboracle_gv.so).  TEST INFRASTRUCTURE.

Only tests/, the smoke check and the cpu_baseline leg of bench.py use this
module; the product never loads it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "build" / "liboracle_gv.so"


class OracleScene(C.Structure):
    _fields_ = [
        ("nodes", C.c_void_p),
        ("node_dim", C.c_int32 * 3),
        ("bricks", C.c_void_p),
        ("fmt", C.c_int32),
        ("slots", C.c_int32 * 3),
        ("jitter", C.c_void_p),
        ("grads", C.c_void_p),
        ("grad_fmt", C.c_int32),
    ]


_lib = None


def build() -> Path:
    """Compile the oracle with its Makefile (no-op when up to date)."""
    r = subprocess.run(["make", "-s", "-C", str(HERE)], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)
    return LIB


def load() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not LIB.exists():
        build()
    lib = C.CDLL(str(LIB))
    from voxviz_b200._native import Uniforms
    lib.oracle_raycast.restype = C.c_int
    lib.oracle_raycast.argtypes = [C.POINTER(Uniforms), C.POINTER(OracleScene), C.c_int, C.c_int, C.c_int,
                                   C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_int32)]
    lib.oracle_raycast_trace.restype = C.c_int
    lib.oracle_raycast_trace.argtypes = [C.POINTER(Uniforms), C.POINTER(OracleScene), C.c_int, C.c_int, C.c_int,
                                         C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_int32)]
    lib.oracle_dxt_decode.restype = C.c_int
    lib.oracle_dxt_decode.argtypes = [C.c_void_p, C.c_int, C.c_longlong, C.c_void_p]
    lib.oracle_max_iterations.restype = C.c_int
    lib.oracle_max_iterations.argtypes = [C.POINTER(Uniforms)]
    lib.oracle_backward.restype = C.c_int
    lib.oracle_backward.argtypes = [C.POINTER(Uniforms), C.POINTER(OracleScene), C.c_void_p, C.c_void_p, C.c_int,
                                    C.c_int]
    lib.oracle_backward_bound.restype = C.c_int
    lib.oracle_backward_bound.argtypes = [C.POINTER(Uniforms), C.POINTER(OracleScene), C.c_void_p, C.c_void_p,
                                          C.c_void_p, C.c_int, C.c_int]
    lib.oracle_fixed_path.restype = C.c_int
    lib.oracle_fixed_path.argtypes = [C.POINTER(Uniforms), C.POINTER(OracleScene), C.POINTER(OracleScene), C.c_int,
                                      C.c_int, C.c_void_p, C.c_int]
    lib.oracle_select.restype = C.c_int
    lib.oracle_select.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p]
    lib.oracle_compress.restype = C.c_int
    lib.oracle_compress.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p,
                                    C.POINTER(C.c_uint32)]
    _lib = lib
    return lib


def _p(a: np.ndarray) -> int:
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


class Scene:
    """Node words (dz,dy,dx,2), brick pool (slots, bytes), format and jitter."""

    def __init__(self, words: np.ndarray, pool: np.ndarray, slots, fmt: int, jitter: np.ndarray,
                 grads: np.ndarray | None = None, grad_fmt: int = 3):
        self.words = np.ascontiguousarray(words, dtype=np.uint32)
        self.pool = np.ascontiguousarray(pool)
        self.jitter = np.ascontiguousarray(jitter, dtype=np.uint8)
        self.grads = None if grads is None else np.ascontiguousarray(grads)
        self.s = OracleScene()
        self.s.nodes = _p(self.words)
        dz, dy, dx = self.words.shape[:3]
        self.s.node_dim[:] = [dx, dy, dz]
        self.s.bricks = _p(self.pool)
        self.s.fmt = int(fmt)
        self.s.slots[:] = [int(v) for v in slots]
        self.s.jitter = _p(self.jitter)
        self.s.grads = _p(self.grads) if self.grads is not None else None
        self.s.grad_fmt = int(grad_fmt)


def raycast(u, scene: Scene, precision: int = 32, rows=None, threads: int = 0, want_usage: bool = True):
    """Returns (color (H,W,4) float32/float64, usage (H,W,12) uint32, status)."""
    lib = load()
    W, H = u.width, u.height
    r0, r1 = (0, H) if rows is None else rows
    color = np.zeros((H, W, 4), dtype=np.float64 if precision == 64 else np.float32)
    usage = np.zeros((H, W, 12), dtype=np.uint32) if want_usage else None
    st = C.c_int32(0)
    rc = lib.oracle_raycast(C.byref(u), C.byref(scene.s), precision, r0, r1, _p(color),
                            _p(usage) if usage is not None else None, threads, C.byref(st))
    if rc != 0:
        raise RuntimeError(f"oracle_raycast failed: {rc}")
    return color, usage, st.value


def raycast_trace(u, scene: Scene, precision: int = 32, rows=None, threads: int = 0):
    """Returns (color, trace (H,W) uint64, status): the ray cast's colour and
    a hash per pixel of its control flow (see oracle_raycast_trace); rows
    outside `rows` keep the trace of an empty pixel (0)."""
    lib = load()
    W, H = u.width, u.height
    r0, r1 = (0, H) if rows is None else rows
    color = np.zeros((H, W, 4), dtype=np.float64 if precision == 64 else np.float32)
    trace = np.zeros((H, W), dtype=np.uint64)
    st = C.c_int32(0)
    rc = lib.oracle_raycast_trace(C.byref(u), C.byref(scene.s), precision, r0, r1, _p(color), None, _p(trace),
                                  threads, C.byref(st))
    if rc != 0:
        raise RuntimeError(f"oracle_raycast_trace failed: {rc}")
    return color, trace, st.value


def flip_pixels(u, scene: Scene, rows=None, threads: int = 0):
    """Pixels whose binary64 ray cast takes other decisions than the binary32
    one (a descent, LOD choice, step count or early termination flips).
    Returns (flips (H,W) bool, fp64 colour, fp32 colour)."""
    c32, t32, _ = raycast_trace(u, scene, 32, rows, threads)
    c64, t64, _ = raycast_trace(u, scene, 64, rows, threads)
    return t32 != t64, c64, c32


def backward(u, scene: Scene, dl_dcolor: np.ndarray, rows=None, grad: np.ndarray | None = None,
             grad_abs: np.ndarray | None = None) -> np.ndarray:
    """dL/d(texel) in float64, shape (slots, 1000, 4), of the binary32 ray
    cast; with grad_abs (same shape) also the per-texel magnitude of the
    summed terms (see oracle_backward_bound)."""
    lib = load()
    r0, r1 = (0, u.height) if rows is None else rows
    g = np.ascontiguousarray(dl_dcolor, dtype=np.float32)
    assert g.shape == (u.height, u.width, 4)
    n = int(np.prod(list(scene.s.slots)))
    if grad is None:
        grad = np.zeros((n, 1000, 4), dtype=np.float64)
    rc = lib.oracle_backward_bound(C.byref(u), C.byref(scene.s), _p(g), _p(grad),
                                   _p(grad_abs) if grad_abs is not None else None, r0, r1)
    if rc != 0:
        raise RuntimeError(f"oracle_backward failed: {rc}")
    return grad


def fixed_path(u, traj: Scene, vals: Scene | None = None, rows=None, threads: int = 0,
               out: np.ndarray | None = None) -> np.ndarray:
    """(H,W,4) float64: the binary32 sample sequence of `traj` composited in
    binary64 with the texels of `vals` (default: traj's own)."""
    lib = load()
    r0, r1 = (0, u.height) if rows is None else rows
    color = np.zeros((u.height, u.width, 4), dtype=np.float64) if out is None else out
    rc = lib.oracle_fixed_path(C.byref(u), C.byref(traj.s), C.byref((vals or traj).s), r0, r1, _p(color), threads)
    if rc != 0:
        raise RuntimeError(f"oracle_fixed_path failed: {rc}")
    return color


def select(usage: np.ndarray) -> np.ndarray:
    lib = load()
    H, W = usage.shape[:2]
    u = np.ascontiguousarray(usage, dtype=np.uint32)
    mask = np.zeros((H, W), dtype=np.uint32)
    lib.oracle_select(_p(u), W, H, _p(mask))
    return mask


def compress(usage: np.ndarray, mask: np.ndarray, max_push: int, cap: int):
    """Returns (list (n,4) uint32 in key order, total active pixels)."""
    lib = load()
    H, W = usage.shape[:2]
    u = np.ascontiguousarray(usage, dtype=np.uint32)
    m = np.ascontiguousarray(mask, dtype=np.uint32)
    out = np.zeros((max(cap, 1), 4), dtype=np.uint32)
    tot = C.c_uint32(0)
    lib.oracle_compress(_p(u), _p(m), W, H, max_push, cap, _p(out), C.byref(tot))
    n = min(tot.value, cap)
    return out[:n].copy(), tot.value


def dxt_decode(blocks: np.ndarray, fmt: int) -> np.ndarray:
    """(bricks, 1000) uint32 RGBA8 texels of DXT5 (1440 B) or DXT1 (720 B) slots."""
    b = np.ascontiguousarray(blocks, dtype=np.uint8)
    n = b.shape[0]
    out = np.zeros((n, 1000), dtype=np.uint32)
    rc = load().oracle_dxt_decode(_p(b), int(fmt), n, _p(out))
    if rc != 0:
        raise RuntimeError(f"oracle_dxt_decode failed: {rc}")
    return out


def max_iterations(u) -> int:
    return load().oracle_max_iterations(C.byref(u))


def cpu_count() -> int:
    return len(os.sched_getaffinity(0))
